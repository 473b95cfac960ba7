"""The differentiation workload at the benchmark shape: 256 subtomograms of 64^3 at L = 32.

One alternation finds each subtomogram's orientation and shift; then the summed aligned
correlation sum_b f_b(R_b exp(omega_b); sigma_b(a_template)) + sum_b c_b(s_b) is evaluated
at omega = 0, the found shifts and the template's own coefficients, and differentiated with
respect to all three.  Gradients are checked on a few subtomograms: the so(3) gradient
against central differences (1e-3 rad) of the oracle's FP64 score on the GPU's sigma, the
shift gradient against the oracle's analytic one and central differences (1e-3 voxel), and
the template gradient along random directions against the (linear) change of the sum.
"""
import os
import sys

import numpy as np
import pytest
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

pytestmark = pytest.mark.gpu


def test_summed_aligned_correlation_gradients_at_benchmark_shape(cuda_device):
    import bench
    from matcha_b200.autograd import (rotation_score, so3_exp, summed_aligned_correlation, template_sigma, zyz_angles,
                                      zyz_matrix)
    from matcha_b200.pipeline import AlignmentStep, StepConfig
    from oracle import matcha as OM
    from oracle import shift as OS

    B, N, L = 256, 64, 32
    rng = np.random.default_rng(3)
    template = bench.make_template(rng)
    vols, q, _ = bench.make_batch(template, np.random.default_rng(4), B, cuda_device)
    step = AlignmentStep(StepConfig(N=N, L=L, Li=[8, 16, 24], batch=B, shift_search_radius=5,
                                    shift_upsample_factor=8), cuda_device)
    step.set_template(template)
    tracker = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    tracker[:, 0] = 1
    z3 = torch.zeros((B, 3), device=cuda_device)
    out = step(vols, vols, tracker, z3)
    base = torch.stack([out["alpha"], out["beta"], out["gamma"]], -1).double()
    rot = step.rot[:B].clone()
    found = out["shift"].clone()

    omega = torch.zeros((B, 3), dtype=torch.float64, device=cuda_device, requires_grad=True)
    shift = found.clone().requires_grad_(True)
    a_t = step.correlator.template_coefficients_alphas_torch.detach().clone().requires_grad_(True)
    total = summed_aligned_correlation(step, vols, omega, base, a_t, shift, z3, rot)
    total.backward()
    for t in (omega.grad, shift.grad, a_t.grad):
        assert t is not None and bool(torch.isfinite(torch.view_as_real(t) if t.is_complex() else t).all())

    # --- so(3): central differences of the oracle's FP64 score on the GPU's sigma
    pick = [0, 1, 2, 3]
    sig = template_sigma(a_t.detach(), step.correlator, L)[pick].cpu().numpy().astype(np.complex128)
    bp = base[pick].cpu()

    def score(w):
        R = zyz_matrix(bp[:, 0], bp[:, 1], bp[:, 2]) @ so3_exp(torch.tensor(w))
        a, b, g = (t.numpy() for t in zyz_angles(R))
        D = OM.wigner_D_stage(a[:, None], b[:, None], g[:, None], L, L, False, np.float64)[:, 0]
        return np.sum(D * sig, -1).real

    h = 1e-3
    fd = np.zeros((len(pick), 3))
    for k in range(3):
        e = np.zeros((len(pick), 3))
        e[:, k] = h
        fd[:, k] = (score(e) - score(-e)) / (2 * h)
    got = omega.grad[pick].cpu().numpy()
    scale = np.abs(score(np.zeros((len(pick), 3)))).max()
    np.testing.assert_allclose(got, fd, atol=1e-5 * scale + 2e-3 * np.abs(fd).max())

    # --- shift: the oracle's analytic gradient and central differences at the found shifts
    ref = OS.load_reference_full(template, N, 1.0)
    trk = out["tracker"][pick].cpu().numpy()
    ang = OS.euler_zyz_deg_from_quat_conj(trk)
    v = vols[pick].cpu().numpy().astype(np.float64)
    s = found[pick].cpu().numpy().astype(np.float64)
    for j, i in enumerate(pick[:2]):
        c0, g0 = OS.shift_score_and_grad(ref, v[j], np.zeros(3), ang[j], s[j])
        np.testing.assert_allclose(shift.grad[i].cpu().numpy(), g0, atol=2e-3 * np.abs(g0).max() + 1e-5)
        e3 = np.eye(3) * 1e-3
        fdv = [(OS.shift_score_and_grad(ref, v[j], np.zeros(3), ang[j], s[j] + e3[k])[0]
                - OS.shift_score_and_grad(ref, v[j], np.zeros(3), ang[j], s[j] - e3[k])[0]) / 2e-3 for k in range(3)]
        np.testing.assert_allclose(g0, fdv, atol=1e-4 * np.abs(g0).max() + 1e-7)

    # --- template: the sum is linear in the template coefficients
    def F(t):
        with torch.no_grad():
            sg = template_sigma(t, step.correlator, L)
            return float(rotation_score(torch.zeros((B, 3), dtype=torch.float64, device=cuda_device), base, sg,
                                        step.matcher, L).sum())

    t0 = a_t.detach()
    for trial in range(2):
        d = torch.randn_like(t0) * t0.abs().mean()
        d[-1] = 0
        fdt = (F(t0 + d) - F(t0 - d)) / 2.0
        an = float((torch.conj(a_t.grad) * d).real.sum())
        assert abs(fdt - an) <= 2e-4 * (abs(fdt) + abs(F(t0))), (trial, fdt, an)
