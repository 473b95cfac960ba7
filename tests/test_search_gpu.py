"""Orientation search on the GPU against the oracle and the reference fixtures."""
import numpy as np
import pytest
import torch

from oracle import matcha as M
from tests.helpers import euler_dist_deg, golden, synthetic_sigma

pytestmark = pytest.mark.gpu


def _matcha(B, Lmax, Li, C=10, steps=1, compat=False, device="cuda:0"):
    from matcha_b200.core.Matcha import Matcha

    return Matcha(batchsize=B, device=torch.device(device), L_max=Lmax,
                  matcha_config=dict(Li=list(Li), candidates=C, num_steps=steps, oversampling_factor_K=2),
                  compat_top_block=compat)


@pytest.mark.parametrize("L0,K", [(4, 2), (8, 2), (8, 1), (12, 2), (16, 2)])
def test_grid_matches_oracle(cuda_device, L0, K):
    from matcha_b200.core.SOFFT import SOFFT

    rng = np.random.default_rng(L0 * 10 + K)
    sig, _ = synthetic_sigma(rng, 3, L0)
    s = SOFFT(L=L0, device=cuda_device, batchsize=3, oversampling_factor=K)
    f = s.eval(torch.from_numpy(sig).to(cuda_device)).cpu().numpy()
    ref = M.sofft_eval(sig.astype(np.complex128), L0, K)
    np.testing.assert_allclose(f, ref, atol=2e-5 * np.abs(ref).max())


@pytest.mark.parametrize("L0,Lmax", [(8, 16), (12, 24), (16, 32)])
def test_grid_topk_indices_bit_exact_on_clear_peaks(cuda_device, L0, Lmax):
    """L0 = 8, 12, 16 (n = 32, 48, 64): the compile-time instantiations of the grid kernel."""
    rng = np.random.default_rng(5 + L0)
    B, C = 6, 10
    n = 4 * L0
    sig, _ = synthetic_sigma(rng, B, Lmax)
    m = _matcha(B, Lmax, [L0, Lmax], C=C)
    a, b, g = m._grid_search_so3fft(torch.from_numpy(sig).to(cuda_device))
    f = M.sofft_eval(sig.astype(np.complex128), L0, 2)
    ids, vals = M.topk_grid(f, C + 1)
    ra, rb, rg = M.ids_to_angles(ids[:, :C], n, dtype=np.float32)
    margin = (vals[:, :-1] - vals[:, 1:]) / np.abs(vals[:, :1])
    for bi in range(B):
        for c in range(C):
            # a rank is only well defined when it is separated from the next value
            if margin[bi, c] > 1e-5 and (c == 0 or margin[bi, c - 1] > 1e-5):
                # angles are float32(index) * float32(step), as torch computes them
                got = np.rint([b[bi, c].item() / (np.pi / (n - 1)), a[bi, c].item() / (2 * np.pi / n),
                               g[bi, c].item() / (2 * np.pi / n)]).astype(int)
                assert tuple(got) == tuple(ids[bi, c]), (bi, c, got, ids[bi, c])
                np.testing.assert_allclose([a[bi, c].item(), b[bi, c].item(), g[bi, c].item()],
                                           [ra[bi, c], rb[bi, c], rg[bi, c]], atol=1e-6)


@pytest.mark.parametrize("compat", [False, True])
def test_search_matches_oracle(cuda_device, compat):
    rng = np.random.default_rng(21 + compat)
    B, Lmax, Li = 8, 16, [4, 8, 12]
    sig, truth = synthetic_sigma(rng, B, Lmax)
    m = _matcha(B, Lmax, Li, steps=2, compat=compat)
    a, b, g, s = (x.cpu().numpy() for x in m.search_orientations(torch.from_numpy(sig).to(cuda_device)))
    ra, rb, rg, rs = M.search_orientations(sig, Li, Lmax, candidates=10, num_steps=2, compat_top_block=compat)
    d = euler_dist_deg(a, b, g, ra, rb, rg)
    assert np.all(d < 0.05), d
    np.testing.assert_allclose(s, rs, rtol=0, atol=2e-5 * np.abs(rs).max())


def test_march_matches_oracle_at_L32(cuda_device):
    rng = np.random.default_rng(99)
    B, Lmax, Li, C = 4, 32, [8, 16, 24], 10
    sig, truth = synthetic_sigma(rng, B, Lmax)
    m = _matcha(B, Lmax, Li, C=C, steps=1)
    st = torch.from_numpy(sig).to(cuda_device)
    a0, b0, g0 = m._grid_search_so3fft(st)
    a, b, g, s = (x.cpu().numpy() for x in m.march(a0, b0, g0, st))
    ra, rb, rg = a0.cpu().numpy(), b0.cpu().numpy(), g0.cpu().numpy()
    for Li_ in M.march_schedule(Li, Lmax):
        ra, rb, rg, rs = M.optimize(ra, rb, rg, sig, Li_, Lmax, 1, False, np.float64)
    d = euler_dist_deg(a, b, g, ra, rb, rg)
    assert np.all(d < 0.05), d
    np.testing.assert_allclose(s, rs, rtol=0, atol=3e-5 * np.abs(rs).max())


@pytest.mark.parametrize("tag", ["small", "mid"])
def test_search_matches_reference_fixture(cuda_device, tag):
    z = golden("search_ref.npz")
    sig = z[tag + "_sigma"]
    m = _matcha(int(z[tag + "_B"]), int(z[tag + "_Lmax"]), [int(x) for x in z[tag + "_Li"]],
                C=int(z[tag + "_C"]), steps=int(z[tag + "_num_steps"]), compat=True)
    a, b, g, s = (x.cpu().numpy() for x in m.search_orientations(torch.from_numpy(sig).to(cuda_device)))
    d = euler_dist_deg(a, b, g, z[tag + "_alpha"], z[tag + "_beta"], z[tag + "_gamma"])
    assert np.all(d < 0.05), d
    np.testing.assert_allclose(s, z[tag + "_score"], rtol=2e-5)
    grid = m.SOFFT.eval(torch.from_numpy(sig).to(cuda_device)).cpu().numpy()
    np.testing.assert_allclose(grid, z[tag + "_grid"], atol=2e-5 * np.abs(grid).max())


def test_errors_match_reference_contract(cuda_device):
    from matcha_b200.core.Matcha import Matcha

    with pytest.raises(ValueError, match="Li"):
        Matcha(batchsize=2, device=cuda_device, L_max=8, matcha_config=dict(candidates=3))
    m = _matcha(2, 8, [4])
    with pytest.raises(ValueError):
        m.search_orientations(torch.zeros((3, 1000), dtype=torch.complex64, device=cuda_device))
