"""Generate the golden fixtures under tests/golden from the reference's own code.

Run in a container that has the reference tree (default /root/reference, override
with MATCHA_REFERENCE_ROOT):

    python tests/golden/make_golden.py [wigner|grad|search|all]

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


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    if what in ("wigner", "all"):
        gen_wigner()
    if what in ("grad", "all"):
        gen_grad()
    if what in ("search", "all"):
        gen_search()
    if what in ("shift", "all"):
        gen_shift()
