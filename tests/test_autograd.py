"""Score derivatives at given rotations and the so(3) gradient of the alignment score: the CUDA
sweep against the oracle's Euler derivatives, the autograd gradient against central finite
differences of the oracle's score in FP64, and the rotation helpers on the CPU."""
import numpy as np
import pytest
import torch

from oracle import matcha as OM


def test_zyz_round_trip_and_kinematics():
    from matcha_b200.autograd import euler_to_body, right_jacobian, so3_exp, zyz_angles, zyz_matrix

    rng = np.random.default_rng(0)
    a, b, g = (torch.tensor(v, dtype=torch.float64) for v in
               (rng.uniform(-3, 3, 6), rng.uniform(0.2, 2.9, 6), rng.uniform(-3, 3, 6)))
    R = zyz_matrix(a, b, g)
    a2, b2, g2 = zyz_angles(R)
    torch.testing.assert_close(zyz_matrix(a2, b2, g2), R, atol=1e-12, rtol=0)
    # body rate of d/dt Rz(a) Ry(b) Rz(g) against R^T dR/dt by finite differences
    rate = torch.tensor(rng.standard_normal((6, 3)))
    h = 1e-6
    Rp = zyz_matrix(a + h * rate[:, 0], b + h * rate[:, 1], g + h * rate[:, 2])
    Rm = zyz_matrix(a - h * rate[:, 0], b - h * rate[:, 1], g - h * rate[:, 2])
    W = R.transpose(-1, -2) @ (Rp - Rm) / (2 * h)
    body = torch.stack([W[:, 2, 1], W[:, 0, 2], W[:, 1, 0]], -1)
    torch.testing.assert_close(body, (euler_to_body(b, g) @ rate[..., None])[..., 0], atol=1e-7, rtol=0)
    # right Jacobian: exp(w + dw) ~ exp(w) exp(Jr dw)
    w = torch.tensor(rng.standard_normal((6, 3)) * 0.7)
    dw = torch.tensor(rng.standard_normal((6, 3))) * 1e-6
    lhs = so3_exp(w).transpose(-1, -2) @ so3_exp(w + dw)
    rhs = so3_exp((right_jacobian(w) @ dw[..., None])[..., 0])
    torch.testing.assert_close(lhs, rhs, atol=1e-11, rtol=0)
    torch.testing.assert_close(so3_exp(torch.zeros(2, 3, dtype=torch.float64)),
                               torch.eye(3, dtype=torch.float64).expand(2, 3, 3))


def _oracle_score(sigma, a, b, g, L):
    D = OM.wigner_D_stage(a[:, None], b[:, None], g[:, None], L, L, False, np.float64)
    return np.sum(D[:, 0] * sigma, -1).real


def _matcher(dev, B, L):
    from matcha_b200.core.Matcha import Matcha

    return Matcha(batchsize=B, device=dev, L_max=L, matcha_config=dict(Li=[L], candidates=2, num_steps=1))


def _sigma(rng, B, L):
    from matcha_b200.core.wigner_index import dsize

    n = dsize(L)
    return (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))) / np.sqrt(n)


@pytest.mark.gpu
@pytest.mark.parametrize("L", [6, 12])
def test_score_derivatives_match_oracle(cuda_device, L):
    B = 4
    rng = np.random.default_rng(L)
    sig = _sigma(rng, B, L)
    a, b, g = rng.uniform(-3, 3, B), rng.uniform(0.1, 3.0, B), rng.uniform(-3, 3, B)
    m = _matcher(cuda_device, B, L)
    f, gr, H = m.score_derivatives(torch.from_numpy(sig.astype(np.complex64)).to(cuda_device),
                                   torch.tensor(a), torch.tensor(b), torch.tensor(g))
    a32, b32, g32 = (v.astype(np.float32).astype(np.float64) for v in (a, b, g))
    D = OM.wigner_D_stage(a32[:, None], b32[:, None], g32[:, None], L, L, False, np.float64)
    g_ref, H_ref = OM.derivatives(D, sig, a32[:, None], L)
    f_ref = np.sum(D[:, 0] * sig, -1).real
    scale = np.abs(H_ref).max()
    np.testing.assert_allclose(f.cpu().numpy(), f_ref, atol=2e-5 * scale)
    np.testing.assert_allclose(gr.cpu().numpy(), g_ref[:, 0], atol=2e-5 * scale)
    np.testing.assert_allclose(H.cpu().numpy(), H_ref[:, 0], atol=2e-5 * scale)


@pytest.mark.gpu
def test_rotation_gradient_matches_finite_differences(cuda_device):
    """d f / d omega of f(R_zyz(base) exp([omega]x)) against central differences (step 1e-3
    rad) of the oracle's score in FP64."""
    from matcha_b200.autograd import rotation_score, so3_exp, zyz_angles, zyz_matrix

    B, L = 5, 10
    rng = np.random.default_rng(3)
    sig = _sigma(rng, B, L)
    base = np.stack([rng.uniform(-3, 3, B), rng.uniform(0.3, 2.8, B), rng.uniform(-3, 3, B)], -1)
    omega0 = rng.standard_normal((B, 3)) * 0.3
    m = _matcher(cuda_device, B, L)
    sg = torch.from_numpy(sig.astype(np.complex64)).to(cuda_device)
    omega = torch.tensor(omega0, device=cuda_device, requires_grad=True)
    f = rotation_score(omega, torch.tensor(base, device=cuda_device), sg, m)
    f.sum().backward()
    got = omega.grad.cpu().numpy()

    def score(w):
        tb = torch.tensor(base)
        R = zyz_matrix(tb[:, 0], tb[:, 1], tb[:, 2]) @ so3_exp(torch.tensor(w))
        a, b, g = (t.numpy() for t in zyz_angles(R))
        return _oracle_score(sig, a, b, g, L)

    h = 1e-3
    fd = np.zeros((B, 3))
    for k in range(3):
        e = np.zeros(3)
        e[k] = h
        fd[:, k] = (score(omega0 + e) - score(omega0 - e)) / (2 * h)
    np.testing.assert_allclose(f.detach().cpu().numpy(), score(omega0), atol=1e-4 * np.abs(fd).max())
    np.testing.assert_allclose(got, fd, atol=2e-3 * np.abs(fd).max())


def _oracle_D(a, b, g, L):
    return OM.wigner_D_stage(np.asarray(a)[:, None], np.asarray(b)[:, None], np.asarray(g)[:, None], L, L, False,
                             np.float64)[:, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("beta0", [0.0, 1e-6, 0.02, np.pi - 1e-6, np.pi])
def test_rotation_gradient_at_and_near_gimbal_lock(cuda_device, beta0):
    """The body-frame gradient from the generators has no Euler singularity: at beta = 0, pi
    and next to them it matches central differences of the oracle's FP64 score."""
    from matcha_b200.autograd import rotation_score, so3_exp, zyz_angles, zyz_matrix

    B, L = 3, 8
    rng = np.random.default_rng(int(beta0 * 1000) + 5)
    sig = _sigma(rng, B, L)
    base = np.stack([rng.uniform(-3, 3, B), np.full(B, beta0), rng.uniform(-3, 3, B)], -1)
    m = _matcher(cuda_device, B, L)
    omega = torch.zeros((B, 3), dtype=torch.float64, device=cuda_device, requires_grad=True)
    f = rotation_score(omega, torch.tensor(base, device=cuda_device),
                       torch.from_numpy(sig.astype(np.complex64)).to(cuda_device), m)
    f.sum().backward()
    got = omega.grad.cpu().numpy()

    def score(w):
        tb = torch.tensor(base)
        R = zyz_matrix(tb[:, 0], tb[:, 1], tb[:, 2]) @ so3_exp(torch.tensor(w))
        a, b, g = (t.numpy() for t in zyz_angles(R))
        return np.sum(_oracle_D(a, b, g, L) * sig, -1).real

    h = 1e-4
    fd = np.zeros((B, 3))
    for k in range(3):
        e = np.zeros((B, 3))
        e[:, k] = h
        fd[:, k] = (score(e) - score(-e)) / (2 * h)
    assert np.all(np.isfinite(got))
    np.testing.assert_allclose(got, fd, atol=1e-3 * np.abs(fd).max())


@pytest.mark.gpu
def test_body_gradient_maps_to_reference_euler_gradient(cuda_device):
    """T(beta, gamma)^T applied to the body-frame gradient is the Euler gradient the
    reference's WignerDGradients.get_derivatives returns (tests/golden/grad_ref.npz)."""
    from matcha_b200 import _native as nat
    from matcha_b200.autograd import euler_to_body
    from tests.helpers import golden

    z = golden("grad_ref.npz")
    sig = np.repeat(z["sigma"], z["alpha"].shape[1], axis=0)  # one row per (b, candidate)
    a, b, g = (z[k].reshape(-1) for k in ("alpha", "beta", "gamma"))
    L = int(z["ell_max"])
    B = sig.shape[0]
    sg = torch.from_numpy(sig.astype(np.complex64)).to(cuda_device)
    ang = [torch.tensor(v, dtype=torch.float32, device=cuda_device) for v in (a, b, g)]
    body = torch.empty((B, 3), dtype=torch.float64, device=cuda_device)
    lib = nat.load()
    nat.check(lib.mtb_score_backward(nat.ptr(sg), sg.stride(0), B, L, *(nat.ptr(t) for t in ang), None, None, 0,
                                     nat.ptr(body), nat.stream_ptr(cuda_device)), "mtb_score_backward")
    a32, b32, g32 = (t.cpu().double() for t in ang)
    euler = (euler_to_body(b32, g32).transpose(-1, -2) @ body.cpu()[..., None])[..., 0].numpy()
    ref = z["grad"].reshape(B, 3)
    np.testing.assert_allclose(euler, ref, atol=2e-4 * np.abs(ref).max())


@pytest.mark.gpu
def test_sigma_gradient_is_conjugate_D(cuda_device):
    from matcha_b200.autograd import rotation_score

    B, L = 4, 10
    rng = np.random.default_rng(11)
    sig = torch.from_numpy(_sigma(rng, B, L).astype(np.complex64)).to(cuda_device).requires_grad_(True)
    base = np.stack([rng.uniform(-3, 3, B), rng.uniform(0.1, 3.0, B), rng.uniform(-3, 3, B)], -1)
    w = torch.tensor(rng.standard_normal(B), device=cuda_device)
    m = _matcher(cuda_device, B, L)
    f = rotation_score(torch.zeros((B, 3), dtype=torch.float64, device=cuda_device),
                       torch.tensor(base, device=cuda_device), sig, m)
    (w * f).sum().backward()
    a32, b32, g32 = (base[:, k].astype(np.float32).astype(np.float64) for k in range(3))
    ref = w.cpu().numpy()[:, None] * np.conj(_oracle_D(a32, b32, g32, L))
    np.testing.assert_allclose(sig.grad.cpu().numpy(), ref, atol=2e-6 * np.abs(ref).max())


@pytest.mark.gpu
def test_template_gradient_matches_finite_differences(cuda_device):
    """d/d a_template of sum_b w_b Re sum D(R_b) sigma_b(a_template): sigma is linear in the
    template, so central differences along random complex directions are exact up to
    rounding; evaluated with the oracle's sigma and D in FP64."""
    from matcha_b200.autograd import rotation_score, template_sigma
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher
    from oracle import fle as OF
    from tests.helpers import blob_template

    N, B, radius = 16, 3, 7
    rng = np.random.default_rng(21)
    tmpl = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7)
    vols = (np.repeat(tmpl[None], B, 0) + 0.3 * rng.standard_normal((B, N, N, N))).astype(np.float32)
    cc = CrossCorrelationMatcher(N=N, device=cuda_device, batchsize=B, bandlimit=8, radius=radius, precision="fp32")
    cc.set_template(tmpl)
    L = cc.lmax - 1  # the score reads degrees <= L; the degree above gets no gradient
    aV = cc.expand(torch.from_numpy(vols).to(cuda_device)).cpu().numpy().astype(np.complex128)
    aT = cc.template_coefficients_alphas_torch.detach().clone().requires_grad_(True)
    m = _matcher(cuda_device, B, L)
    base = np.stack([rng.uniform(-3, 3, B), rng.uniform(0.2, 2.9, B), rng.uniform(-3, 3, B)], -1)
    w = rng.standard_normal(B)
    sig = template_sigma(aT, cc, L)
    f = rotation_score(torch.zeros((B, 3), dtype=torch.float64, device=cuda_device),
                       torch.tensor(base, device=cuda_device), sig, m, L)
    (torch.tensor(w, device=cuda_device) * f).sum().backward()
    grad = aT.grad.cpu().numpy().astype(np.complex128)
    a32, b32, g32 = (base[:, k].astype(np.float32).astype(np.float64) for k in range(3))
    D = _oracle_D(a32, b32, g32, L)

    def F(t):
        s = OF.compute_sigma(cc.fle.tables, t[:-1], aV)[:, :D.shape[1]]
        return float(np.sum(w * np.sum(D * s, -1).real))

    t0 = aT.detach().cpu().numpy().astype(np.complex128)
    for trial in range(3):
        d = rng.standard_normal(t0.shape) + 1j * rng.standard_normal(t0.shape)
        d[-1] = 0
        fd = (F(t0 + d) - F(t0 - d)) / 2.0
        an = float(np.sum((np.conj(grad) * d).real))
        assert abs(fd - an) <= 1e-4 * (abs(fd) + np.abs(grad).sum() * 1e-3), (trial, fd, an)
    # degrees above L get no gradient
    from matcha_b200.core import fle_tables as T

    tb = T.lap_eig_ball(N, 8, radius)
    assert np.any(tb.ls > L)
    assert np.all(grad[:-1][tb.ls > L] == 0) and grad[-1] == 0


@pytest.mark.gpu
def test_shift_score_gradient(cuda_device):
    """The continuous correlation of the shift match: on the 1/uf grid it is the value the
    search maximises, and its gradient matches the oracle's analytic gradient and central
    differences."""
    from matcha_b200.core.ShiftMatcher import ShiftMatcher
    from oracle import shift as OS
    from tests.helpers import blob_template, haar_quaternions, rotate_volumes_reference

    class Cfg(dict):
        __getattr__ = dict.__getitem__

    N, uf, r, B = 32, 8, 3, 3
    rng = np.random.default_rng(33)
    tmpl = blob_template(rng, N, 40, 9, (1.5, 3.0), mask_radius=13)
    q = haar_quaternions(rng, B)
    vols = (rotate_volumes_reference(np.repeat(tmpl[None], B, 0), q) + 0.3 * rng.standard_normal((B, N, N, N))
            ).astype(np.float32)
    prior = rng.uniform(-1, 1, (B, 3)).astype(np.float32)
    for precision in ("fp32", "bf16x3"):
        sm = ShiftMatcher(Cfg(N=N, voxel_size=1.0, num_subtomograms_per_batch=B, shift_upsample_factor=uf,
                              shift_search_radius=r, do_ctf_correction=False, box_size=N), cuda_device,
                          torch.complex64, precision=precision)
        sm.set_reference(tmpl)
        dv = torch.from_numpy(vols).to(cuda_device)
        dp = torch.from_numpy(prior).to(cuda_device)
        trk = torch.from_numpy(q).to(cuda_device)
        shift, score = sm.search_shifts(subtomos=dv, ctfs=None, shift_zyx=dp, rotation_tracker=trk)
        rot = torch.empty((B, 9), device=cuda_device)
        from matcha_b200 import _native as nat

        nat.check(sm._lib.mtb_tracker_rotation(nat.ptr(trk), B, nat.ptr(rot), nat.stream_ptr(cuda_device)), "rot")
        c_grid, _ = sm.score_and_gradient(dv, dp, rot, shift)
        np.testing.assert_allclose(c_grid.cpu().numpy(), score.cpu().numpy(), rtol=2e-4 if precision == "bf16x3" else 2e-5)
    s = shift.cpu().numpy() + rng.uniform(-0.05, 0.05, (B, 3)).astype(np.float32)
    c, gr = sm.score_and_gradient(dv, dp, rot, torch.from_numpy(s).to(cuda_device))
    ref = OS.load_reference_full(tmpl, N, 1.0)
    ang = OS.euler_zyz_deg_from_quat_conj(q)
    h = 1e-3
    for i in range(B):
        co, go = OS.shift_score_and_grad(ref, vols[i].astype(np.float64), prior[i].astype(np.float64), ang[i], s[i])
        np.testing.assert_allclose(c[i].item(), co, rtol=1e-4)
        np.testing.assert_allclose(gr[i].cpu().numpy(), go, atol=1e-3 * np.abs(go).max() + 1e-6)
        fd = []
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            fd.append((OS.shift_score_and_grad(ref, vols[i].astype(np.float64), prior[i].astype(np.float64), ang[i],
                                               s[i] + e)[0]
                       - OS.shift_score_and_grad(ref, vols[i].astype(np.float64), prior[i].astype(np.float64),
                                                 ang[i], s[i] - e)[0]) / (2 * h))
        np.testing.assert_allclose(go, np.array(fd), atol=1e-4 * np.abs(go).max() + 1e-7)
