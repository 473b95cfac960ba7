"""Generate the golden fixtures under tests/golden from the reference's own code.

Run where a checkout of the reference exists, named by MATCHA_REFERENCE_ROOT:

    MATCHA_REFERENCE_ROOT=<checkout> python tests/golden/make_golden.py [wigner|grad|search|shift|fle|sigma|all]

What each fixture holds and which reference code produced it:

* ``wigner_ref.npz``   -- ``WignerDMatrices.D`` (src/matcha/core/WignerDMatrices.py:1291-1375),
  the reference's Numba kernels executed by Numba's CPU simulator, for two angle
  triples at ell_max=6 with truncate=5 (exact blocks) and truncate=6 (the top block
  the reference returns when truncate == ell_max).
* ``grad_ref.npz``     -- ``WignerDGradients.set_so3_coeffs`` + ``get_derivatives``
  (src/matcha/core/WignerDGradients.py:155-302) on a seeded sigma and D.
* ``shift_ref.npz``    -- ``load_reference_full`` and ``estimate_shift_like_relion``
  (src/matcha/core/ShiftMatcher.py:456-472, 619-674) with the masks of
  src/matcha/utils/setup_utils.py:239-270, on three seeded 32^3 subtomograms.
* ``search_ref.npz``   -- ``Matcha.search_orientations`` (src/matcha/core/Matcha.py:369-403) and
  ``SOFFT.eval`` (src/matcha/core/SOFFT.py:67-98), run as reference code on the CPU.
  Two inputs the reference takes from packages absent here are supplied by the
  oracle: the SOFFT d-table (``spherical.Wigner(L).d``, the same small-d at
  alpha=gamma=0) and ``WignerDMatrices.D`` (pinned by ``wigner_ref.npz``); both are
  returned in float32/complex64 exactly as the reference would hold them.
* ``fle_ref.npz``      -- ``FLEBasis3D.lap_eig_ball`` (src/matcha/core/FLEBasis3D.py:700-799) at
  16^3/L=8, 32^3/L=16, 64^3/L=32 and 128^3/L=64, reading Bessel-zero tables written here
  (the reference's .mat files are not in its tree), and ``create_denseB`` (:570-698) applied
  as a = B^H f to seeded volumes (see ``gen_fle``).
* ``sigma_ref.npz``    -- ``CrossCorrelationMatcher._precompute_indices`` + ``compute_sigma``
  (src/matcha/core/CrossCorrelationMatcher.py:133-212) on the coefficients of ``fle_ref.npz``.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import refharness  # noqa: E402  (sets the Numba simulator flag before numba loads)
from oracle import wigner as W  # noqa: E402


def synthetic_sigma(rng, B, Lmax, noise=0.3, lmax_extra=0):
    """sigma_b = sum_l w_l conj(D^l(R_b)) + noise: f(R) peaks at R = R_b."""
    L = Lmax + lmax_extra
    n = W.dsize(L)
    a = rng.uniform(0, 2 * np.pi, B)
    b = np.arccos(rng.uniform(-1, 1, B))
    g = rng.uniform(0, 2 * np.pi, B)
    D = W.wigner_D(a, b, g, L)
    ls, _, _ = W.lmm(L)
    w = np.exp(-(ls / (0.6 * Lmax)) ** 2) * (2 * ls + 1)
    sig = np.conj(D) * w + noise * (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))) * w / (2 * ls + 1)
    return sig.astype(np.complex64), np.stack([a, b, g], -1)


def gen_wigner():
    import torch

    w = refharness.make_reference_wigner(ell_max=6, batchsize=1, num_candidates=2)
    al = torch.tensor([[0.9, 2.2]], dtype=torch.float32)
    be = torch.tensor([[1.2, 0.4]], dtype=torch.float32)
    ga = torch.tensor([[2.1, -0.7]], dtype=torch.float32)
    D5 = w.D(alpha=al, beta=be, gamma=ga, truncate=5).numpy()
    D6 = w.D(alpha=al, beta=be, gamma=ga, truncate=6).numpy()
    np.savez_compressed(os.path.join(HERE, "wigner_ref.npz"), alpha=al.numpy(), beta=be.numpy(),
                        gamma=ga.numpy(), D_trunc5=D5, D_trunc6=D6, ell_max=6)
    print("wigner_ref.npz", D5.shape, D6.shape)


def _install_spherical_stub():
    sph = sys.modules["spherical"]

    class Wigner:
        def __init__(self, ell_max):
            self.ell_max = int(ell_max)
            self.Dsize = W.dsize(self.ell_max)

        def d(self, expib):
            return W.small_d_all(self.ell_max, np.angle(expib)).astype(np.complex128)

        def Dindex(self, l, mp, m):
            return W.dindex(l, mp, m)

    sph.Wigner = Wigner


def _reference_matcha(B, C, Lmax, Li, num_steps, K=2):
    import torch

    refharness._install_stubs()
    _install_spherical_stub()
    wmod = refharness.load_wigner_module()
    Mmod = refharness.load_module("matcha.core.Matcha")
    cwd = os.getcwd()
    tmp = os.path.join("/tmp", "matcha_ref_cache")
    os.makedirs(tmp, exist_ok=True)
    os.chdir(tmp)
    try:
        cfg = refharness._ConfigDict(Li=list(Li), candidates=C, num_steps=num_steps,
                                     oversampling_factor_K=K)
        m = Mmod.Matcha(batchsize=B, device=torch.device("cpu"), L_max=Lmax, matcha_config=cfg)
    finally:
        os.chdir(cwd)

    def D_oracle(q=None, alpha=None, beta=None, gamma=None, truncate=None):
        t = Lmax if truncate is None else int(truncate)
        D = W.wigner_D(alpha.double().numpy(), beta.double().numpy(), gamma.double().numpy(), t)
        if t == Lmax:
            ls, mps, ms = W.lmm(t)
            D[..., (ls == t) & ((mps == -t) | (ms == -t))] = 0.0
        return torch.from_numpy(D.astype(np.complex64))

    m.WignerDMatrices.D = D_oracle
    return m, wmod


def gen_grad():
    import torch

    refharness._install_stubs()
    _install_spherical_stub()
    wmod = refharness.load_wigner_module()
    Gmod = refharness.load_module("matcha.core.WignerDGradients")
    rng = np.random.default_rng(7)
    L = 6
    cwd = os.getcwd()
    os.chdir("/tmp")
    try:
        w = refharness.make_reference_wigner(ell_max=L, batchsize=2, num_candidates=3)
        G = Gmod.WignerDGradients(wigner=w, device=torch.device("cpu"))
    finally:
        os.chdir(cwd)
    n = W.dsize(L)
    sig = (rng.standard_normal((2, n)) + 1j * rng.standard_normal((2, n))).astype(np.complex64)
    a = rng.uniform(0, 2 * np.pi, (2, 3))
    b = rng.uniform(0.1, 3.0, (2, 3))
    g = rng.uniform(0, 2 * np.pi, (2, 3))
    D = W.wigner_D(a, b, g, L).astype(np.complex64)
    Dp = np.concatenate([D, np.zeros((2, 3, 1), np.complex64)], -1)
    sp = np.concatenate([sig, np.zeros((2, 1), np.complex64)], -1)
    G.set_so3_coeffs(torch.from_numpy(sp))
    grad, hess = G.get_derivatives(torch.from_numpy(Dp), torch.from_numpy(a.astype(np.float32)))
    np.savez_compressed(os.path.join(HERE, "grad_ref.npz"), sigma=sig, alpha=a, beta=b, gamma=g,
                        grad=grad.numpy(), hess=hess.numpy(), ell_max=L)
    print("grad_ref.npz", grad.shape, hess.shape)


def gen_search():
    import torch

    cases = []
    for tag, (B, C, Lmax, Li, steps, seed) in {
        "small": (3, 10, 8, [4, 6], 1, 11),
        "mid": (4, 10, 16, [4, 8, 12], 2, 12),
    }.items():
        m, _ = _reference_matcha(B, C, Lmax, Li, steps)
        rng = np.random.default_rng(seed)
        sig, truth = synthetic_sigma(rng, B, Lmax)
        st = torch.from_numpy(sig)
        grid = m.SOFFT.eval(st.clone()).numpy().copy()
        a, b, g, s = m.search_orientations(st.clone())
        cases.append((tag, dict(sigma=sig, truth=truth, grid=grid, alpha=a.numpy(), beta=b.numpy(),
                                gamma=g.numpy(), score=s.numpy(), B=B, C=C, Lmax=Lmax,
                                Li=np.array(Li), num_steps=steps, K=2)))
        print(tag, a.numpy(), b.numpy(), g.numpy(), s.numpy())
    out = {}
    for tag, d in cases:
        for k, v in d.items():
            out[f"{tag}_{k}"] = v
    np.savez_compressed(os.path.join(HERE, "search_ref.npz"), **out)
    print("search_ref.npz")


def gen_shift():
    """ShiftMatcher reference path on the CPU: load_reference_full + estimate_shift_like_relion."""
    import torch

    refharness._install_stubs()
    S = refharness.load_module("matcha.core.ShiftMatcher")
    U = refharness.load_module("matcha.utils.setup_utils")
    sys.path.insert(0, ROOT)
    from tests.helpers import blob_template, haar_quaternions, rotate_volumes_reference
    from oracle import shift as OS

    N, uf, r = 32, 8, 3
    rng = np.random.default_rng(31)
    tmpl = blob_template(rng, N, 40, 9, (1.5, 3.0), mask_radius=13)
    q = haar_quaternions(rng, 3)
    vols = rotate_volumes_reference(np.repeat(tmpl[None], 3, 0), q)
    # integer and fractional true shifts via a Fourier phase ramp, plus noise
    true = np.array([[0.0, 0.0, 0.0], [1.0, -2.0, 0.5], [-1.25, 0.75, 2.0]])
    k = np.fft.fftfreq(N)
    kz, ky, kx = np.meshgrid(k, k, k, indexing="ij")
    for i in range(3):
        ph = np.exp(-2j * np.pi * (kz * true[i, 0] + ky * true[i, 1] + kx * true[i, 2]))
        vols[i] = np.fft.ifftn(np.fft.fftn(vols[i]) * ph).real
    vols = (vols + 0.3 * rng.standard_normal(vols.shape)).astype(np.float32)
    prior = np.array([[0.0, 0.0, 0.0], [0.5, -1.0, 0.25], [0.0, 0.0, 0.0]], dtype=np.float32)
    angles = OS.euler_zyz_deg_from_quat_conj(q)
    ref = S.load_reference_full(tmpl, volume_size=N, voxel_size=1.0)
    mask_full = torch.from_numpy(U._get_mask_full((N, N, N // 2 + 1))).unsqueeze(0)
    mo, mc, rc = U._compute_masks((N, N, N), N / 2.0, 5.0)
    cfg = refharness._ConfigDict(N=N, shift_upsample_factor=uf, shift_search_radius=r, do_ctf_correction=False,
                                 device=torch.device("cpu"),
                                 execution=refharness._ConfigDict(shape=torch.tensor((N, N, N)),
                                                                  dtype=torch.complex64))
    shift, score = S.estimate_shift_like_relion(
        torch.from_numpy(ref).unsqueeze(0).to(torch.complex64).expand(3, -1, -1, -1), torch.from_numpy(vols), None,
        torch.from_numpy(prior)[:, None, :], angles, mask_full, torch.from_numpy(mo), torch.from_numpy(mc),
        torch.from_numpy(rc).to(torch.float32), cfg)
    np.savez_compressed(os.path.join(HERE, "shift_ref.npz"), template=tmpl, subtomos=vols, quats=q, prior_zyx=prior,
                        angles_deg=angles, ref_fourier=ref.astype(np.complex64), shift_xyz=shift.numpy(),
                        score=score.numpy(), N=N, uf=uf, radius=r, true_zyx=true)
    print("shift_ref.npz", shift.numpy(), score.numpy())


def write_bessel_tables(directory, n_l, n_k):
    """The two tables the reference loads in lap_eig_ball (FLEBasis3D.py:726-730), absent from
    its tree: roots_table[l, k-1] = k-th positive zero of j_l and cs[l, k-1] =
    sqrt(2)/|j_{l+1}(root)|, for l < n_l, k <= n_k, written as .mat files."""
    from scipy.io import savemat
    from scipy.special import spherical_jn

    from matcha_b200.core.fle_tables import BesselZeros

    z = BesselZeros()
    roots = np.zeros((n_l, n_k))
    for l in range(n_l):
        roots[l] = z._compute(l, n_k)
    cs = np.sqrt(2.0) / np.abs(spherical_jn(np.arange(1, n_l + 1)[:, None], roots))
    rp, cp = os.path.join(directory, f"jl_zeros_l={n_l}_k={n_k}.mat"), os.path.join(directory, f"cs_l={n_l}_k={n_k}.mat")
    savemat(rp, {"roots_table": roots})
    savemat(cp, {"cs": cs})
    return rp, cp, roots


class _SplShim:
    """scipy.special with the ``sph_harm(m, l, azimuth, polar)`` call create_denseB makes
    (FLEBasis3D.py:595,603); scipy 1.18 removed it in favour of sph_harm_y(l, m, polar, azimuth)."""

    def __getattr__(self, name):
        import scipy.special as sps

        return getattr(sps, name)

    @staticmethod
    def sph_harm(m, l, p, t):
        from scipy.special import sph_harm_y

        return sph_harm_y(l, m, t, p)


def _reference_fle_object(N, bandlimit, rp, cp):
    """A reference FLEBasis3D whose constructor is skipped (its precomp needs cuFINUFFT and
    torch-harmonics): the attributes lap_eig_ball and create_denseB read are set, and
    lap_eig_ball itself is the reference's method."""
    refharness._install_stubs()
    F = refharness.load_module("matcha.core.FLEBasis3D")
    F.spl = _SplShim()
    obj = F.FLEBasis3D.__new__(F.FLEBasis3D)
    obj.jl_zeros_path, obj.cs_path = rp, cp
    obj.complexmode = True
    N2 = N + (N % 2)
    ls, ks, ms, mds, lmds, cs, ne = obj.lap_eig_ball(int(N2 ** 3 * np.pi / 6), bandlimit)
    obj.ls, obj.ks, obj.ms, obj.mds, obj.lmds, obj.cs, obj.ne = ls, ks, ms, mds, lmds, cs, ne
    obj.N = obj.N1 = N
    return obj


def _mpmath_root_check(roots, picks):
    """Independent check of the regenerated zeros: j_l(x) = sqrt(pi/2x) J_{l+1/2}(x), so the
    k-th zero of j_l is mpmath's k-th zero of J_{l+1/2}."""
    import mpmath

    return max(abs(float(mpmath.besseljzero(l + 0.5, k)) - roots[l, k - 1]) for l, k in picks)


def gen_fle():
    """fle_ref.npz: the reference's own lap_eig_ball (FLEBasis3D.py:700-799) for the shapes of
    the alignment (16^3/L=8, 32^3/L=16, 64^3/L=32, 128^3/L=64), and its create_denseB
    (FLEBasis3D.py:570-698) applied as the dense adjoint a = B^H f (h folded into B) to seeded
    volumes at 16^3 (R = 8) and 32^3 (R = 16), plus the 32^3 box at radius 15 (the alignment's
    default radius, min(N/2, int(0.95 N/2))): create_denseB on the 30^3 crop whose coordinates
    are -15..14 (the 32^3 box's voxels outside the crop have r >= 1, where every basis function
    is zero or j_l(lambda_lk) = 0)."""
    sys.path.insert(0, ROOT)
    from tests.helpers import blob_template

    tmp = os.path.join("/tmp", "matcha_ref_tables")
    os.makedirs(tmp, exist_ok=True)
    rp, cp, roots = write_bessel_tables(tmp, 260, 260)
    err = _mpmath_root_check(roots, [(0, 1), (0, 40), (7, 3), (31, 12), (42, 1), (100, 50), (200, 7), (259, 259)])
    print("regenerated zeros vs mpmath: max abs err", err)
    assert err < 1e-9
    out = {"root_check_err": err}
    for N, L in ((16, 8), (32, 16), (64, 32), (128, 64)):
        obj = _reference_fle_object(N, L, rp, cp)
        tag = f"t{N}"
        for k in ("ls", "ks", "ms", "mds", "lmds", "cs"):
            out[f"{tag}_{k}"] = np.asarray(getattr(obj, k))
        out[f"{tag}_ne"] = int(obj.ne)
        out[f"{tag}_L"] = L
        print(f"N={N} L={L}: ne={obj.ne} lmax={int(np.max(obj.ls))}")
    rng = np.random.default_rng(41)
    for N, L, radius in ((16, 8, 8), (32, 16, 16), (32, 16, 15)):
        obj = _reference_fle_object(N, L, rp, cp)
        vols = np.stack([blob_template(rng, N, 20, N // 4, (1.0, 2.5), mask_radius=N // 2 - 2),
                         rng.standard_normal((N, N, N))]).astype(np.float32)
        if radius == N // 2:
            B = obj.create_denseB()
            a = vols.reshape(2, -1).astype(np.float64) @ np.conj(B)
        else:
            lo = N // 2 - radius
            obj.N = obj.N1 = 2 * radius
            B = obj.create_denseB()
            crop = vols[:, lo:lo + 2 * radius, lo:lo + 2 * radius, lo:lo + 2 * radius]
            a = crop.reshape(2, -1).astype(np.float64) @ np.conj(B)
        tag = f"c{N}r{radius}"
        out[f"{tag}_volumes"] = vols
        out[f"{tag}_coeffs"] = a
        out[f"{tag}_L"] = L
        print(tag, a.shape, np.abs(a).max())
        del B
    np.savez_compressed(os.path.join(HERE, "fle_ref.npz"), **out)
    print("fle_ref.npz")


def gen_sigma():
    """sigma_ref.npz: the reference's CrossCorrelationMatcher._precompute_indices and
    compute_sigma (CrossCorrelationMatcher.py:133-212) on the 32^3 (radius 16) and 16^3
    coefficients of fle_ref.npz, volume 0 as the template, in complex128.  The index maps
    (idlm_list) are built from lap_eig_ball's output as precomp builds them
    (FLEBasis3D.py:337-357); spherical.Wigner(ell).Dindex is the reference's own WignerDindex
    (WignerDMatrices.py:969), the function it was adapted from."""
    import torch

    refharness._install_stubs()
    wmod = refharness.load_wigner_module()
    sph = sys.modules["spherical"]

    class _Wigner:
        def __init__(self, ell_max):
            self.ell_max = ell_max

        def Dindex(self, ell, mp, m):
            return wmod.WignerDindex(ell, mp, m)

    sph.Wigner = _Wigner
    C = refharness.load_module("matcha.core.CrossCorrelationMatcher")
    fx = np.load(os.path.join(HERE, "fle_ref.npz"))
    out = {}
    for N, radius in ((16, 8), (32, 16)):
        tag = f"c{N}r{radius}"
        ls, mds = fx[f"t{N}_ls"], fx[f"t{N}_mds"]
        ne = int(fx[f"t{N}_ne"])
        lmax = int(ls.max())
        idlm = [[[] for _ in range(2 * lmax + 1)] for _ in range(lmax + 1)]
        for i in range(ne):
            idlm[ls[i]][mds[i]].append(i)
        cc = C.CrossCorrelationMatcher.__new__(C.CrossCorrelationMatcher)
        cc.lmax = lmax
        cc.device = torch.device("cpu")
        cc.dtype = torch.complex128
        cc.fle = types.SimpleNamespace(idlm_list=idlm, ne=ne)
        cc.alpha1_indices, cc.alpha2_indices, cc.phase_factors, cc.wigner_indices = cc._precompute_indices()
        a = torch.from_numpy(fx[f"{tag}_coeffs"])
        cc.template_coefficients_alphas_torch = torch.nn.functional.pad(a[0], (0, 1))
        cc.bh_volumes_buffer = torch.zeros((a.shape[0], ne + 1), dtype=torch.complex128)
        cc.sigma = torch.zeros((a.shape[0], wmod.WignerDsize(0, lmax, lmax)), dtype=torch.complex128)
        cc.compute_sigma(a, 0, a.shape[0])
        out[f"{tag}_sigma"] = cc.sigma.numpy()
        out[f"{tag}_norms"] = torch.linalg.norm(a, dim=1).numpy()
        print(tag, "sigma", cc.sigma.shape)
    np.savez_compressed(os.path.join(HERE, "sigma_ref.npz"), **out)
    print("sigma_ref.npz")


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("fle", "all"):
        gen_fle()
    if what in ("sigma", "all"):
        gen_sigma()
    if what in ("wigner", "all"):
        gen_wigner()
    if what in ("grad", "all"):
        gen_grad()
    if what in ("search", "all"):
        gen_search()
    if what in ("shift", "all"):
        gen_shift()
