"""Oracle (test infrastructure only): the SO(3) grid search and the frequency-marched
Newton refinement, restated in numpy.

Follows, line by line in meaning:
  * SOFFT d-table and evaluation      src/matcha/core/SOFFT.py:30-98
  * top-k over the grid               src/matcha/core/Matcha.py:27-58
  * grid index -> Euler angles        src/matcha/core/SOFFT.py:100-124
  * Newton march                      src/matcha/core/Matcha.py:150-205, 239-403
  * coefficient bank / derivatives    src/matcha/core/WignerDGradients.py:155-302
  * reduce over candidates            src/matcha/core/Matcha.py:19-24

``dtype`` selects float32 (the reference's arithmetic) or float64 (an exact
restatement).  ``compat_top_block`` reproduces the reference's top-degree block at
the final march stage, whose m'=-Lmax row and m=-Lmax column come out as zero
(WignerDMatrices.py:573-576 never writes the conjugate power of index ell_max).
Only tests, the smoke check and the CPU baseline may import this module.
"""
from __future__ import annotations

import numpy as np

from . import wigner as W


# ---------------------------------------------------------------- SO(3) grid
def sofft_tables(L0: int, K: int):
    """d-table (n_beta, dsize(L0)) and flat scatter targets for l < L0 (SOFFT.py:30-64)."""
    n = 2 * L0 * K
    betas = np.linspace(0.0, np.pi, n, endpoint=True)
    dtab = W.small_d_all(L0, betas)  # (n, dsize(L0))
    ls, mps, ms = W.lmm(L0 - 1)
    lin = (mps % n) * n + (ms % n)
    return dtab, lin, n


def sofft_eval(sigma: np.ndarray, L0: int, K: int, dtype=np.float64) -> np.ndarray:
    """f[b, beta, alpha, gamma] = Re ifft2_{alpha,gamma}( scatter(d * sigma) )  (SOFFT.py:67-98)."""
    dtab, lin, n = sofft_tables(L0, K)
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    nk = W.dsize(L0 - 1)
    B = sigma.shape[0]
    temp = dtab[None, :, :nk].astype(cdt) * sigma[:, None, :nk].astype(cdt)  # (B, nb, nk)
    F = np.zeros((B, n, n * n), dtype=cdt)
    for b in range(B):
        for j in range(n):
            np.add.at(F[b, j], lin, temp[b, j])
    f = np.fft.ifft2(F.reshape(B, n, n, n), axes=(2, 3)).real
    return f.astype(dtype)


def topk_grid(f: np.ndarray, k: int):
    """Top-k flat indices per batch, descending, as (beta, alpha, gamma) index triples (Matcha.py:27-58)."""
    B = f.shape[0]
    flat = f.reshape(B, -1)
    idx = np.argsort(-flat, axis=1, kind="stable")[:, :k]
    n1, n2 = f.shape[2], f.shape[3]
    x = idx // (n1 * n2)
    y = (idx // n2) % n1
    z = idx % n2
    return np.stack([x, y, z], axis=-1), np.take_along_axis(flat, idx, axis=1)


def ids_to_angles(ids: np.ndarray, n: int, dtype=np.float64):
    """(SOFFT.py:100-124): beta = i pi/(n-1), alpha = i 2pi/n, gamma = i 2pi/n."""
    betas = (ids[..., 0] * (np.pi / (n - 1))).astype(dtype)
    alphas = (ids[..., 1] * (2 * np.pi / n)).astype(dtype)
    gammas = (ids[..., 2] * (2 * np.pi / n)).astype(dtype)
    return alphas, betas, gammas


# ---------------------------------------------------------------- derivatives
def _row_factors(ell_max: int):
    """Per-entry factors of WignerDGradients.py:45-79, indexed by the flat D index.

    c1 = -sqrt((l+m')(l-m'+1))/2, c2 = sqrt((l-m')(l+m'+1))/2,
    tn2 = sqrt((l+m')(l-m'+1)(l+m'-1)(l-m'+2))/4, t0 = -((l+m')(l-m'+1)+(l+m'+1)(l-m'))/4,
    tp2 = sqrt((l+m'+1)(l-m')(l+m'+2)(l-m'-1))/4, where m' is the row index.
    """
    ls, mps, ms = W.lmm(ell_max)
    l = ls.astype(np.float64)
    mp = mps.astype(np.float64)
    c1 = -0.5 * np.sqrt(np.maximum((l + mp) * (l - mp + 1), 0.0))
    c2 = 0.5 * np.sqrt(np.maximum((l - mp) * (l + mp + 1), 0.0))
    tn2 = np.sqrt(np.maximum((l + mp) * (l - mp + 1) * (l + mp - 1) * (l - mp + 2), 0.0)) / 4
    t0 = -((l + mp) * (l - mp + 1) + (l + mp + 1) * (l - mp)) / 4
    tp2 = np.sqrt(np.maximum((l + mp + 1) * (l - mp) * (l + mp + 2) * (l - mp - 1), 0.0)) / 4
    return c1, c2, tn2, t0, tp2


def _shift_rows(D: np.ndarray, ell_max: int, delta: int) -> np.ndarray:
    """Return S with S[..., idx(l,m',m)] = D[..., idx(l,m'+delta,m)] (0 outside the block)."""
    ls, mps, ms = W.lmm(ell_max)
    out = np.zeros_like(D)
    valid = np.abs(mps + delta) <= ls
    src = np.array([W.dindex(l, mp + delta, m) if v else 0 for l, mp, m, v in zip(ls, mps, ms, valid)])
    out[..., valid] = D[..., src[valid]]
    return out


def derivatives(D: np.ndarray, sigma: np.ndarray, alpha: np.ndarray, ell_max: int):
    """Euler gradient (3) and Hessian (3x3) of f = Re sum D sigma (WignerDGradients.py:155-302).

    D: (B, C, dsize(ell_max)) complex, sigma: (B, dsize(ell_max)), alpha: (B, C).
    Equivalent to the reference's 15-column bank contraction followed by its alpha-phase
    mixing; written with row-shifted D instead of the scattered bank.
    """
    _, mps, ms = W.lmm(ell_max)
    c1, c2, tn2, t0, tp2 = _row_factors(ell_max)
    s = sigma[:, None, :]
    ea = np.exp(1j * alpha)[..., None]
    Dm1 = _shift_rows(D, ell_max, -1) * ea      # e^{+i a} D[m'-1]
    Dp1 = _shift_rows(D, ell_max, +1) / ea      # e^{-i a} D[m'+1]
    Dm2 = _shift_rows(D, ell_max, -2) * ea * ea
    Dp2 = _shift_rows(D, ell_max, +2) / (ea * ea)
    imp = 1j * mps
    im = 1j * ms
    Db = c1 * Dm1 + c2 * Dp1
    Dbb = t0 * D + tn2 * Dm2 + tp2 * Dp2
    ga = np.sum(D * imp * s, -1).real
    gb = np.sum(Db * s, -1).real
    gg = np.sum(D * im * s, -1).real
    haa = np.sum(D * imp * imp * s, -1).real
    hgg = np.sum(D * im * im * s, -1).real
    hag = np.sum(D * imp * im * s, -1).real
    hab = np.sum(Db * imp * s, -1).real
    hbg = np.sum(Db * im * s, -1).real
    hbb = np.sum(Dbb * s, -1).real
    g = np.stack([ga, gb, gg], -1)
    H = np.stack([np.stack([haa, hab, hag], -1),
                  np.stack([hab, hbb, hbg], -1),
                  np.stack([hag, hbg, hgg], -1)], -2)
    return g, H


def derivatives_bank(D, sigma, alpha, ell_max):
    """The reference's own formulation: 15-column bank, contraction, alpha-phase mixing.

    Kept to pin ``derivatives`` against WignerDGradients.py:155-302 step by step.
    """
    ls, mps, ms = W.lmm(ell_max)
    c1, c2, tn2, t0, tp2 = _row_factors(ell_max)
    n = W.dsize(ell_max)
    j = 1j
    coeff = sigma
    bank = np.zeros((sigma.shape[0], 15, n), dtype=np.complex128)
    bank[:, 0] = coeff
    bank[:, 1] = j * mps * coeff
    bank[:, 2] = j * ms * coeff
    bank[:, 3] = (j * mps) ** 2 * coeff
    bank[:, 4] = (j * ms) ** 2 * coeff
    bank[:, 5] = (j * mps) * (j * ms) * coeff
    for i in range(n):
        l, mp, m = ls[i], mps[i], ms[i]
        if mp - 1 >= -l:
            bank[:, 6, W.dindex(l, mp - 1, m)] += coeff[:, i] * c1[i]
        if mp + 1 <= l:
            bank[:, 7, W.dindex(l, mp + 1, m)] += coeff[:, i] * c2[i]
        if mp - 2 >= -l:
            bank[:, 12, W.dindex(l, mp - 2, m)] += coeff[:, i] * tn2[i]
        if mp + 2 <= l:
            bank[:, 14, W.dindex(l, mp + 2, m)] += coeff[:, i] * tp2[i]
    bank[:, 13] = t0 * coeff
    bank[:, 8] = j * mps * bank[:, 6]
    bank[:, 9] = j * mps * bank[:, 7]
    bank[:, 10] = j * ms * bank[:, 6]
    bank[:, 11] = j * ms * bank[:, 7]
    Y = np.einsum("bnc,bkc->bnk", D, bank)
    pp = np.exp(1j * alpha)
    pn = np.exp(-1j * alpha)
    p2p = np.exp(2j * alpha)
    p2n = np.exp(-2j * alpha)
    beta_out = pp * Y[..., 6] + pn * Y[..., 7]
    gb_out = pp * Y[..., 10] + pn * Y[..., 11]
    ab = pp * (1j * Y[..., 6] + Y[..., 8]) + pn * (-1j * Y[..., 7] + Y[..., 9])
    bb = Y[..., 13] + p2p * Y[..., 12] + p2n * Y[..., 14]
    g = np.stack([Y[..., 1], beta_out, Y[..., 2]], -1).real
    H = np.stack([np.stack([Y[..., 3], ab, Y[..., 5]], -1),
                  np.stack([ab, bb, gb_out], -1),
                  np.stack([Y[..., 5], gb_out, Y[..., 4]], -1)], -2).real
    return g, H


# ---------------------------------------------------------------- Newton march
def wigner_D_stage(alpha, beta, gamma, Li: int, Lmax: int, compat_top_block: bool, dtype):
    """D truncated to degree Li as the reference's WignerDMatrices.D(truncate=Li) returns it."""
    D = W.wigner_D(np.asarray(alpha, np.float64), np.asarray(beta, np.float64),
                   np.asarray(gamma, np.float64), Li)
    if compat_top_block and Li == Lmax:
        ls, mps, ms = W.lmm(Li)
        bad = (ls == Li) & ((mps == -Li) | (ms == -Li))
        D[..., bad] = 0.0
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    return D.astype(cdt)


def march_schedule(Li, Lmax):
    """Matcha.py:76 and :381-386: sorted(Li) + [Lmax], skipping Li >= Lmax unless last."""
    sched = sorted(int(x) for x in Li) + [int(Lmax)]
    out = []
    for i, l in enumerate(sched):
        if l >= Lmax and i != len(sched) - 1:
            continue
        out.append(l)
    return out


def optimize(alphas, betas, gammas, sigma, Li, Lmax, num_steps=1, compat_top_block=False,
             dtype=np.float64, trace=None, step_type="newton"):
    """One march stage (Matcha.py:239-367) with Newton steps (or, step_type "gradient", the
    ascent step -lr * gradient with base lr 5e-7, Matcha.py:14-15, :91, :344-345) and
    accept/reject (:150-205)."""
    rdt = dtype
    n = W.dsize(Li)
    s = sigma[:, :n].astype(np.complex64 if dtype == np.float32 else np.complex128)
    a = np.array(alphas, dtype=rdt)
    b = np.array(betas, dtype=rdt)
    g = np.array(gammas, dtype=rdt)
    D = wigner_D_stage(a, b, g, Li, Lmax, compat_top_block, dtype)
    best = np.einsum("bcn,bn->bc", D, s).real.astype(rdt)
    lr = np.full(a.shape, 1.0 if step_type == "newton" else 5e-7, dtype=rdt)
    for _ in range(num_steps):
        grad, H = derivatives(D.astype(np.complex128), s.astype(np.complex128), a.astype(np.float64), Li)
        step = np.zeros_like(grad)
        if step_type == "gradient":
            step = -grad
        else:
            for bi in range(a.shape[0]):
                for ci in range(a.shape[1]):
                    try:
                        step[bi, ci] = np.linalg.solve(H[bi, ci].astype(rdt), grad[bi, ci].astype(rdt))
                    except np.linalg.LinAlgError:
                        step[bi, ci] = 0.0
        step = (lr[..., None] * step).astype(rdt)
        ta = (a - step[..., 0]).astype(rdt)
        tb = (b - step[..., 1]).astype(rdt)
        tg = (g - step[..., 2]).astype(rdt)
        Dt = wigner_D_stage(ta, tb, tg, Li, Lmax, compat_top_block, dtype)
        ev = np.einsum("bcn,bn->bc", Dt, s).real.astype(rdt)
        upd = ev > best
        if trace is not None:
            trace.append(dict(Li=Li, grad=grad, H=H, step=step, ev=ev, upd=upd))
        lr = np.where(upd, lr * rdt(1.1), lr * rdt(0.5)).astype(rdt)
        a = np.where(upd, ta, a)
        b = np.where(upd, tb, b)
        g = np.where(upd, tg, g)
        D = np.where(upd[..., None], Dt, D)
        best = np.where(upd, ev, best)
    return a, b, g, best


def search_orientations(sigma, Li, Lmax, L0=None, K=2, candidates=10, num_steps=1,
                        compat_top_block=False, dtype=np.float64, return_grid=False, return_candidates=False,
                        step_type="newton"):
    """Matcha.search_orientations (Matcha.py:369-403) on numpy input ``sigma`` (B, >=dsize(Lmax)).
    ``return_candidates`` appends the march's final (alpha, beta, gamma, score) of every
    candidate, (B, C) each, before the reduction over candidates (Matcha.py:19-24)."""
    sched = march_schedule(Li, Lmax)
    if L0 is None:
        L0 = min(sched)
    f = sofft_eval(sigma, L0, K, dtype=dtype)
    ids, _ = topk_grid(f, candidates)
    n = 2 * L0 * K
    a, b, g = ids_to_angles(ids, n, dtype=dtype)
    for Li_ in sched:
        a, b, g, best = optimize(a, b, g, sigma, Li_, Lmax, num_steps, compat_top_block, dtype,
                                 step_type=step_type)
    idx = np.argmax(best, axis=-1)
    take = lambda x: np.take_along_axis(x, idx[:, None], 1)[:, 0]
    out = (take(a), take(b), take(g), take(best))
    if return_candidates:
        out = out + ((a, b, g, best),)
    if return_grid:
        return out, f, ids
    return out
