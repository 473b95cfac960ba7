"""Oracle (test infrastructure only): one alignment alternation on the CPU.

Chains the restatements of this package in the order of
src/matcha/align_subtomograms.py:254-285 (get_sigma -> search_orientations ->
update_rotation_estimate -> search_shifts) for a handful of subtomograms.  It is the
CPU baseline the benchmark reports beside the GPU numbers, and a checker for the
GPU pipeline; nothing in the product imports it.

``FoldedFLE`` evaluates the same discrete adjoint as ``fle.evaluate_t`` but folds each
volume over the 8 sign images of the positive octant first, which keeps the 64^3 basis
at 1/8 of the dense size (float64, built once per configuration).
"""
from __future__ import annotations

import numpy as np
from scipy.spatial.transform import Rotation as R
from scipy.special import spherical_jn

from . import fle as F
from . import matcha as M
from . import shift as S


class FoldedFLE:
    """a = h B^H f through the octant folding; exact to float64 rounding."""

    def __init__(self, tables, N1: int, radius: float, dense: bool = True):
        """``dense=False`` skips the basis columns (n_rep x ne complex: 66 GB at 128^3, L = 64);
        only ``evaluate_t_streamed`` is available then."""
        self.tables = tables
        N = N1 + (N1 % 2)
        R_ = N // 2
        g = np.arange(-R_, R_ + N % 2)
        x, y, z = np.meshgrid(g, g, g, indexing="ij")
        inside = (np.sqrt(x ** 2 + y ** 2 + z ** 2) / radius) <= 1 + 1e-13
        if N > N1:
            inside[N1:], inside[:, N1:], inside[:, :, N1:] = False, False, False
        reps = np.unique(np.abs(np.stack([x[inside], y[inside], z[inside]], 1)), axis=0)
        self.reps = reps
        self.N1, self.R = N1, R_
        # flat voxel index of each sign image (bit0 flips x, bit1 y, bit2 z); -1 absent/duplicate
        img = np.full((reps.shape[0], 8), -1, dtype=np.int64)
        for s in range(8):
            sg = np.array([-1 if s & (1 << d) else 1 for d in range(3)])
            c = reps * sg + R_
            ok = np.all((c >= 0) & (c < N1), axis=1)
            for d in range(3):
                if s & (1 << d):
                    ok &= reps[:, d] != 0
            img[ok, s] = (c[ok, 0] * N1 + c[ok, 1]) * N1 + c[ok, 2]
        self.img = img
        r = np.sqrt((reps ** 2).sum(1)) / radius
        th = np.arctan2(np.sqrt(reps[:, 0] ** 2 + reps[:, 1] ** 2), reps[:, 2])
        ph = np.arctan2(reps[:, 1], reps[:, 0])
        self.r, self.th, self.ph = r, th, ph
        tb = tables
        self.pos = np.nonzero(tb.ms >= 0)[0]
        self.partner = {}
        for i in range(tb.ne):
            self.partner[(int(tb.ls[i]), int(tb.ks[i]), int(tb.ms[i]))] = i
        if not dense:
            return
        cols = np.zeros((reps.shape[0], self.pos.size), dtype=np.complex128)
        ylm = _sph_harm_table(tb.lmax, th, ph)
        radial = {}
        for j, i in enumerate(self.pos):
            l, m, k = int(tb.ls[i]), int(tb.ms[i]), int(tb.ks[i])
            if (l, k) not in radial:
                radial[(l, k)] = spherical_jn(l, tb.lmds[i] * r)
            cols[:, j] = tb.h * tb.cs[i] * radial[(l, k)] * np.conj(ylm[(l, m)])
        self.cols = cols
        # parity of Re / Im of each column under the flips of x, y, z
        m = tb.ms[self.pos]
        l = tb.ls[self.pos]
        self.par_re = np.stack([(-1.0) ** m, np.ones_like(m, dtype=float), (-1.0) ** (l + m)], 1)
        self.par_im = np.stack([-(-1.0) ** m, -np.ones_like(m, dtype=float), (-1.0) ** (l + m)], 1)

    def _channel(self, vols, par):
        """sum over images of f(image) * prod over flipped axes of par -> (b, n_rep) per column class."""
        b = vols.shape[0]
        v = vols.reshape(b, -1)
        out = {}
        for key in {tuple(p) for p in par}:
            acc = np.zeros((b, self.reps.shape[0]))
            for s in range(8):
                idx = self.img[:, s]
                ok = idx >= 0
                w = np.prod([key[d] if s & (1 << d) else 1.0 for d in range(3)])
                acc[:, ok] += w * v[:, idx[ok]]
            out[key] = acc
        return out

    def evaluate_t(self, vols):
        vols = np.asarray(vols, dtype=np.float64)
        b = vols.shape[0]
        tb = self.tables
        ch_re = self._channel(vols, self.par_re)
        ch_im = self._channel(vols, self.par_im)
        re = np.zeros((b, self.pos.size))
        im = np.zeros((b, self.pos.size))
        for key, A in ch_re.items():
            sel = np.all(self.par_re == key, axis=1)
            re[:, sel] = A @ self.cols[:, sel].real
        for key, A in ch_im.items():
            sel = np.all(self.par_im == key, axis=1)
            im[:, sel] = A @ self.cols[:, sel].imag
        a = np.zeros((b, tb.ne), dtype=np.complex128)
        a[:, self.pos] = re + 1j * im
        for i in range(tb.ne):
            m = int(tb.ms[i])
            if m < 0:
                j = self.partner[(int(tb.ls[i]), int(tb.ks[i]), -m)]
                a[:, i] = (-1.0) ** m * np.conj(a[:, j])
        return a


    def evaluate_t_streamed(self, vols):
        """``evaluate_t`` one degree at a time, holding no basis: the associated Legendre
        functions advance in l by the same normalised recurrences as ``_sph_harm_table`` (all
        orders m <= l of degrees l - 1 and l - 2 kept), the radial functions of degree l are
        made for that degree only, and each (l, m) contracts the 8 sign-image channels with
        its Re / Im parity.  Same float64 sums as the dense form, in another order."""
        vols = np.asarray(vols, dtype=np.float64)
        b = vols.shape[0]
        tb = self.tables
        keys = [(sx, sy, sz) for sx in (1.0, -1.0) for sy in (1.0, -1.0) for sz in (1.0, -1.0)]
        ch = self._channel(vols, keys)
        x = np.cos(self.th)
        sn = np.sqrt(np.maximum(0.0, 1.0 - x * x))
        lmax = int(tb.lmax)
        # per degree: its coefficient indices with m >= 0, grouped by k
        by_l = {}
        for i in self.pos:
            by_l.setdefault(int(tb.ls[i]), []).append(int(i))
        a = np.zeros((b, tb.ne), dtype=np.complex128)
        p1 = {}  # P_{l-1}^m
        p2 = {}  # P_{l-2}^m
        for l in range(lmax + 1):
            cur = {}
            for m in range(l + 1):
                if m == l:
                    cur[m] = (np.full_like(x, 1.0 / np.sqrt(4 * np.pi)) if l == 0
                              else -np.sqrt((2 * m + 1) / (2 * m)) * sn * p1[m - 1])
                elif m == l - 1:
                    cur[m] = np.sqrt(2 * m + 3) * x * p1[m]
                else:
                    aa = np.sqrt((4 * l * l - 1) / (l * l - m * m))
                    bb = np.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
                    cur[m] = aa * (x * p1[m] - bb * p2[m])
            p2, p1 = p1, cur
            idx = by_l.get(l, [])
            if not idx:
                continue
            ks = sorted({int(tb.ks[i]) for i in idx})
            radial = {}
            for k in ks:
                i0 = next(i for i in idx if int(tb.ks[i]) == k)
                radial[k] = tb.h * tb.cs[i0] * spherical_jn(l, tb.lmds[i0] * self.r)
            Rk = np.stack([radial[k] for k in ks], 0)  # (n_k, n_rep)
            for m in range(l + 1):
                cols = [self.partner[(l, k, m)] for k in ks if (l, k, m) in self.partner]
                kk = [j for j, k in enumerate(ks) if (l, k, m) in self.partner]
                if not cols:
                    continue
                yc = cur[m] * np.exp(-1j * m * self.ph)  # conj(Y_l^m)
                sre = (-1.0) ** m
                slm = (-1.0) ** (l + m)
                key_re = (sre, 1.0, slm)
                key_im = (-sre, -1.0, slm)
                re = (ch[key_re] * yc.real) @ Rk[kk].T
                im = (ch[key_im] * yc.imag) @ Rk[kk].T
                a[:, cols] = re + 1j * im
        for i in range(tb.ne):
            m = int(tb.ms[i])
            if m < 0:
                j = self.partner[(int(tb.ls[i]), int(tb.ks[i]), -m)]
                a[:, i] = (-1.0) ** m * np.conj(a[:, j])
        return a


def _sph_harm_table(lmax, theta, phi):
    """Y_l^m(theta, phi) for 0 <= m <= l <= lmax: orthonormal, Condon-Shortley phase, by the
    standard normalised associated-Legendre recurrences (checked against scipy's sph_harm_y
    in the tests)."""
    x = np.cos(theta)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    out = {}
    pmm = np.full_like(x, 1.0 / np.sqrt(4 * np.pi))
    for m in range(lmax + 1):
        if m > 0:
            pmm = -np.sqrt((2 * m + 1) / (2 * m)) * s * pmm
        e = np.exp(1j * m * phi)
        p2, p1 = np.zeros_like(x), pmm
        out[(m, m)] = pmm * e
        for l in range(m + 1, lmax + 1):
            if l == m + 1:
                p = np.sqrt(2 * m + 3) * x * pmm
            else:
                a = np.sqrt((4 * l * l - 1) / (l * l - m * m))
                b = np.sqrt(((l - 1) ** 2 - m * m) / (4 * (l - 1) ** 2 - 1))
                p = a * (x * p1 - b * p2)
            p2, p1 = p1, p
            out[(l, m)] = p * e
    return out


def update_rotation_estimate(alpha, beta, gamma, tracker):
    """src/matcha/utils/rotation_ops.py:23-34 with (w, x, y, z) float64 trackers."""
    cb, sb = np.cos(0.5 * beta), np.sin(0.5 * beta)
    q = np.stack([cb * np.cos(0.5 * (alpha + gamma)), -sb * np.sin(0.5 * (alpha - gamma)),
                  sb * np.cos(0.5 * (alpha - gamma)), cb * np.sin(0.5 * (alpha + gamma))], -1)
    q[:, [1, 3]] = q[:, [3, 1]]
    qc = q * np.array([1, -1, -1, -1])
    t = np.asarray(tracker, dtype=np.float64)
    w1, v1 = t[:, :1], t[:, 1:]
    w2, v2 = qc[:, :1], qc[:, 1:]
    out = np.concatenate([w1 * w2 - (v1 * v2).sum(1, keepdims=True), w1 * v2 + w2 * v1 + np.cross(v1, v2)], 1)
    return out / np.linalg.norm(out, axis=1, keepdims=True)


def align_batch(fle: FoldedFLE, a_template, ref_fourier, vols, subtomos, tracker, shift_zyx, L, Li, K=2,
                candidates=10, num_steps=1, uf=8, shift_radius=5, dtype=np.float32):
    """One alternation for a few subtomograms: returns the same quantities as the GPU step."""
    a = fle.evaluate_t(vols)
    sigma = F.compute_sigma(fle.tables, a_template, a)
    al, be, ga, score, cand = M.search_orientations(sigma, list(Li) + [L], L, K=K, candidates=candidates,
                                                    num_steps=num_steps, dtype=dtype, return_candidates=True)
    tr = update_rotation_estimate(al.astype(np.float64), be.astype(np.float64), ga.astype(np.float64), tracker)
    ang = S.euler_zyz_deg_from_quat_conj(tr)
    shifts, scores = [], []
    for i in range(vols.shape[0]):
        s, sc = S.estimate_shift_like_relion(ref_fourier, subtomos[i], shift_zyx[i], ang[i], uf, shift_radius)
        shifts.append(s)
        scores.append(sc)
    return dict(alpha=al, beta=be, gamma=ga, rotation_score=score, bh_norms=np.linalg.norm(a, axis=1),
                tracker=tr, shift=np.array(shifts), shift_score=np.array(scores),
                candidates=dict(zip(("alpha", "beta", "gamma", "score"), cand)))


def rotation_matrix_of_tracker(tr):
    """Matrix the shift match uses for a tracker (ShiftMatcher.py:503, :913)."""
    return R.from_euler("ZYZ", S.euler_zyz_deg_from_quat_conj(tr), degrees=True).as_matrix()


def run_alternations(fle: FoldedFLE, a_template, ref_fourier, subtomos, tracker, local_shifts, prior_shifts,
                     base_shifts, L, Li, radius, num_alternations, **kw):
    """BatchProcessor._run_alternations (src/matcha/align_subtomograms.py:316-361) for a few
    subtomograms: each alternation prepares the batch at the current shift and orientation
    (oracle.prepare, align_subtomograms.py:240-252), aligns it (align_batch) with the shift
    match at the current shift, and adds the found shift to the local shifts.  Returns one
    dict per alternation; the tracker and local shifts are not modified in place."""
    from . import prepare as P

    tr = np.asarray(tracker, dtype=np.float64).copy()
    local = np.asarray(local_shifts, dtype=np.float64).copy()
    outs = []
    for _ in range(num_alternations):
        current = (np.asarray(prior_shifts) + np.asarray(base_shifts) + local).astype(np.float32)
        data = P.prepare(subtomos, current, tr, radius)
        o = align_batch(fle, a_template, ref_fourier, data, np.asarray(subtomos, dtype=np.float64), tr,
                        current.astype(np.float64), L, Li, **kw)
        tr = o["tracker"]
        local = local + o["shift"]
        o["local_shifts"] = local.copy()
        o["shift_prior"] = current
        outs.append(o)
    return outs
