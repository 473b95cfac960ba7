"""The reference's fallback and failure behaviours on the GPU path, none of which faults a GPU.

* A singular Hessian: the reference skips the Newton step of that candidate
  (src/matcha/core/Matcha.py:316-343); so does the FP64 3x3 solve of the march kernel.
* ``step_type: gradient``: the ascent step -lr * gradient with base lr 5e-7
  (Matcha.py:14-15, :91, :344-345), against the oracle.
* A bounded device wait that runs out: the tensor-core expansion's stall hook makes its MMA
  thread wait for operands that never come; the kernel gives up after ~20 ms, records the
  error and returns, ``FLEBasis3D.status()`` raises status 4 (MTB_ERR_TIMEOUT), and the same
  handle then computes correct results again.
"""
import numpy as np
import pytest
import torch

from oracle import matcha as OM
from oracle import wigner as W
from tests.helpers import euler_dist_deg, synthetic_sigma

pytestmark = pytest.mark.gpu


def test_singular_hessian_takes_no_step(cuda_device):
    """sigma on the (l, 0, 0) entries only: f = sum_l Re(sigma_l00) P_l(cos beta) does not
    depend on alpha or gamma, so the Hessian's alpha and gamma rows are exactly zero at every
    candidate.  Every Newton step is skipped: the results are the grid candidates."""
    from matcha_b200.core.Matcha import Matcha

    B, Lmax, Li, K = 3, 8, [4, 6], 2
    rng = np.random.default_rng(5)
    sig = np.zeros((B, W.dsize(Lmax)), np.complex64)
    for l in range(Lmax + 1):
        sig[:, W.dindex(l, 0, 0)] = rng.standard_normal(B) * (2 * l + 1)
    m = Matcha(batchsize=B, device=cuda_device, L_max=Lmax,
               matcha_config=dict(Li=Li, candidates=10, num_steps=1, oversampling_factor_K=K))
    a, b, g, s = (t.cpu().numpy().astype(np.float64) for t in m.search_orientations(torch.from_numpy(sig).to(
        cuda_device)))
    n = 2 * min(Li) * K
    jb = b * (n - 1) / np.pi
    np.testing.assert_allclose(jb, np.rint(jb), atol=1e-4)   # beta on the grid: no step taken
    ja, jg = a * n / (2 * np.pi), g * n / (2 * np.pi)
    np.testing.assert_allclose(ja, np.rint(ja), atol=1e-4)
    np.testing.assert_allclose(jg, np.rint(jg), atol=1e-4)
    ao, bo, go, so = OM.search_orientations(sig, Li + [Lmax], Lmax, K=K, dtype=np.float64)
    np.testing.assert_allclose(b, bo, atol=1e-6)              # the same best grid beta
    np.testing.assert_allclose(s, so, rtol=1e-5)


def test_gradient_step_matches_oracle(cuda_device):
    from matcha_b200.core.Matcha import Matcha

    B, Lmax, Li = 6, 16, [4, 8, 12]
    rng = np.random.default_rng(9)
    sig, _ = synthetic_sigma(rng, B, Lmax)
    outs = {}
    for step_type in ("gradient", "newton"):
        m = Matcha(batchsize=B, device=cuda_device, L_max=Lmax,
                   matcha_config=dict(Li=Li, candidates=10, num_steps=2, oversampling_factor_K=2,
                                      step_type=step_type))
        outs[step_type] = [t.cpu().numpy().astype(np.float64) for t in
                           m.search_orientations(torch.from_numpy(sig).to(cuda_device))]
    ref = OM.search_orientations(sig, Li + [Lmax], Lmax, K=2, num_steps=2, dtype=np.float64,
                                 step_type="gradient")
    a, b, g, s = outs["gradient"]
    d = euler_dist_deg(a, b, g, *(np.asarray(x, np.float64) for x in ref[:3]))
    assert np.all(d < 0.05), d
    np.testing.assert_allclose(s, ref[3], rtol=1e-4)
    # the flag changes the search: the Newton steps move away from the gradient ones
    dn = euler_dist_deg(*outs["newton"][:3], a, b, g)
    assert dn.max() > 0.05


def test_bounded_wait_timeout_is_reported_and_recovered(cuda_device):
    from matcha_b200 import _native as nat
    from matcha_b200.core.FLEBasis3D import FLEBasis3D

    fle = FLEBasis3D(N=32, bandlimit=16, eps=1e-4, batchsize=4, radius=15, device=cuda_device,
                     dtype=torch.complex64, precision="bf16x3")
    vols = torch.randn(4, 32, 32, 32, device=cuda_device, generator=torch.Generator(cuda_device).manual_seed(3))
    good = fle.evaluate_t(vols).clone()
    fle.status()
    lib = nat.load()
    assert lib.mtb_fle_inject_stall(fle._h, 1) == nat.MTB_OK
    fle.evaluate_t(vols)
    with pytest.raises(RuntimeError, match="status 4"):
        fle.status()
    assert lib.mtb_fle_inject_stall(fle._h, 0) == nat.MTB_OK
    again = fle.evaluate_t(vols)
    fle.status()  # the flag was cleared when reported; the context is intact
    assert torch.equal(again, good)
    f32 = FLEBasis3D(N=32, bandlimit=16, eps=1e-4, batchsize=4, radius=15, device=cuda_device,
                     dtype=torch.complex64, precision="fp32")
    assert lib.mtb_fle_inject_stall(f32._h, 1) == nat.MTB_ERR_ARG
