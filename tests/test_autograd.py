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
