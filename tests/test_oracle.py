"""The oracle against the reference's own outputs (golden fixtures) and against mathematics."""
import numpy as np
import pytest

from oracle import matcha as M
from oracle import wigner as W
from tests.helpers import euler_dist_deg, golden


def test_small_d_explicit_matches_recurrence():
    for l in range(0, 9):
        for beta in (0.0, 0.3, 1.2, 2.9, np.pi, -0.7, 4.0):
            a = W.small_d_block_explicit(l, beta)
            b = W.small_d_all(l, beta)[W.dsize(l - 1):].reshape(2 * l + 1, 2 * l + 1)
            np.testing.assert_allclose(a, b, atol=1e-12)


def test_small_d_symmetries_and_unitarity():
    L = 12
    d = W.small_d_all(L, 1.1)
    for l in range(L + 1):
        blk = d[W.dsize(l - 1):W.dsize(l)].reshape(2 * l + 1, 2 * l + 1)
        np.testing.assert_allclose(blk @ blk.T, np.eye(2 * l + 1), atol=1e-10)
        m = np.arange(-l, l + 1)
        sign = (-1.0) ** (m[:, None] - m[None, :])
        np.testing.assert_allclose(blk.T, sign * blk, atol=1e-12)       # d_{m m'} = (-1)^{m'-m} d_{m' m}
        np.testing.assert_allclose(blk[::-1, ::-1], sign * blk, atol=1e-12)  # d_{-m',-m} = (-1)^{m'-m} d_{m'm}


def test_wigner_matches_reference_kernels():
    z = golden("wigner_ref.npz")
    L = int(z["ell_max"])
    D = W.wigner_D(z["alpha"].astype(np.float64), z["beta"].astype(np.float64), z["gamma"].astype(np.float64), L)
    np.testing.assert_allclose(z["D_trunc5"], D[..., :W.dsize(L - 1)], atol=2e-6)
    # truncate == ell_max: the reference's top block loses its m'=-L row and m=-L column
    Dc = M.wigner_D_stage(z["alpha"], z["beta"], z["gamma"], L, L, True, np.float64)
    np.testing.assert_allclose(z["D_trunc6"], Dc, atol=2e-6)
    ls, mps, ms = W.lmm(L)
    bad = (ls == L) & ((mps == -L) | (ms == -L))
    assert np.abs(D[..., bad]).max() > 1e-3  # the defect is visible, not vacuous


def test_derivatives_match_reference_gradients():
    z = golden("grad_ref.npz")
    L = int(z["ell_max"])
    D = W.wigner_D(z["alpha"], z["beta"], z["gamma"], L).astype(np.complex64).astype(np.complex128)
    g, H = M.derivatives(D, z["sigma"].astype(np.complex128), z["alpha"].astype(np.float32).astype(np.float64), L)
    np.testing.assert_allclose(g, z["grad"], rtol=0, atol=2e-6 * np.abs(z["grad"]).max())
    np.testing.assert_allclose(H, z["hess"], rtol=0, atol=2e-6 * np.abs(z["hess"]).max())
    g2, H2 = M.derivatives_bank(D, z["sigma"].astype(np.complex128), z["alpha"].astype(np.float32).astype(np.float64), L)
    np.testing.assert_allclose(g, g2, atol=1e-9)
    np.testing.assert_allclose(H, H2, atol=1e-9)


def test_derivatives_finite_differences():
    rng = np.random.default_rng(3)
    L = 6
    n = W.dsize(L)
    sig = rng.standard_normal((1, n)) + 1j * rng.standard_normal((1, n))
    x = np.array([0.9, 1.2, 2.1])
    f = lambda v: np.sum(W.wigner_D(np.array([[v[0]]]), np.array([[v[1]]]), np.array([[v[2]]]), L) * sig[:, None]).real
    D = W.wigner_D(np.array([[x[0]]]), np.array([[x[1]]]), np.array([[x[2]]]), L)
    g, H = M.derivatives(D, sig, np.array([[x[0]]]), L)
    h = 1e-5
    fd = [(f(x + h * e) - f(x - h * e)) / (2 * h) for e in np.eye(3)]
    np.testing.assert_allclose(g[0, 0], fd, rtol=1e-7, atol=1e-6)
    h = 1e-4
    Hfd = np.array([[(f(x + h * ei + h * ej) - f(x + h * ei - h * ej) - f(x - h * ei + h * ej) + f(x - h * ei - h * ej))
                     / (4 * h * h) for ej in np.eye(3)] for ei in np.eye(3)])
    np.testing.assert_allclose(H[0, 0], Hfd, atol=1e-4 * np.abs(Hfd).max())


@pytest.mark.parametrize("tag", ["small", "mid"])
def test_search_matches_reference(tag):
    s = golden("search_ref.npz")
    sig = s[tag + "_sigma"]
    Lmax = int(s[tag + "_Lmax"])
    Li = [int(x) for x in s[tag + "_Li"]]
    C = int(s[tag + "_C"])
    steps = int(s[tag + "_num_steps"])
    f = M.sofft_eval(sig, min(M.march_schedule(Li, Lmax)), 2, dtype=np.float32)
    np.testing.assert_allclose(f, s[tag + "_grid"], atol=1e-5 * np.abs(f).max())
    a, b, g, sc = M.search_orientations(sig, Li, Lmax, candidates=C, num_steps=steps, compat_top_block=True,
                                        dtype=np.float64)
    d = euler_dist_deg(a, b, g, s[tag + "_alpha"], s[tag + "_beta"], s[tag + "_gamma"])
    assert d.max() < 0.05, d
    np.testing.assert_allclose(sc, s[tag + "_score"], rtol=1e-5)
    # and the search finds the planted rotation
    t = s[tag + "_truth"]
    dt = euler_dist_deg(a, b, g, t[:, 0], t[:, 1], t[:, 2])
    assert np.median(dt) < 2.0, dt
