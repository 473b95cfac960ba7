"""Ball expansion and sigma on the GPU against the oracle; end-to-end rotation recovery."""
import numpy as np
import pytest
import torch

from matcha_b200.core import fle_tables as T
from oracle import fle as F
from tests.helpers import (alignment_error_deg, blob_template, haar_quaternions, rotate_volumes_reference)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N1,bl,radius", [(32, 16, 14), (32, 16, 16), (31, 12, 13)])
def test_evaluate_t_matches_dense_definition(cuda_device, N1, bl, radius):
    from matcha_b200.core.FLEBasis3D import FLEBasis3D

    fle = FLEBasis3D(N=N1, bandlimit=bl, eps=1e-4, batchsize=3, radius=radius, device=cuda_device,
                     dtype=torch.complex64)
    rng = np.random.default_rng(N1 + radius)
    vols = rng.standard_normal((3, N1, N1, N1)).astype(np.float32)
    a = fle.evaluate_t(torch.from_numpy(vols).to(cuda_device)).cpu().numpy()
    ref = F.evaluate_t(fle.tables, vols, float(radius))
    err = np.linalg.norm(a - ref) / np.linalg.norm(ref)
    assert err < 1e-5, err
    assert np.abs(a - ref).max() < 1e-5 * np.abs(ref).max()


def test_sigma_and_norms_match_oracle(cuda_device):
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher

    N1, radius = 32, 14
    rng = np.random.default_rng(4)
    tmpl = blob_template(rng, N1, 40, 12, (1.5, 3.0), mask_radius=14)
    vols = rotate_volumes_reference(np.repeat(tmpl[None], 4, 0), haar_quaternions(rng, 4))
    cc = CrossCorrelationMatcher(N=N1, device=cuda_device, batchsize=5, bandlimit=16, radius=radius)
    cc.set_template(tmpl)
    sig, norms = cc.get_sigma(torch.from_numpy(vols).to(cuda_device))
    sig, norms = sig.cpu().numpy(), norms.cpu().numpy()
    at = F.evaluate_t(cc.fle.tables, tmpl[None], float(radius))[0]
    av = F.evaluate_t(cc.fle.tables, vols, float(radius))
    ref = F.compute_sigma(cc.fle.tables, at, av)
    assert sig.shape == (5, ref.shape[1])
    err = np.linalg.norm(sig[:4] - ref) / np.linalg.norm(ref)
    assert err < 2e-5, err
    assert np.all(sig[4] == 0)  # rows past the batch stay zero (reference zeroes sigma per call)
    np.testing.assert_allclose(norms[:4], np.linalg.norm(av, axis=1), rtol=1e-5)
    np.testing.assert_allclose(cc.bh_norm_template.item(), np.linalg.norm(at), rtol=1e-5)


def test_sigma_upto_is_the_leading_degrees_of_sigma(cuda_device):
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher
    from matcha_b200.core.wigner_index import compute_size

    N1, radius = 32, 14
    rng = np.random.default_rng(5)
    tmpl = blob_template(rng, N1, 40, 12, (1.5, 3.0), mask_radius=14)
    vols = torch.from_numpy(rotate_volumes_reference(np.repeat(tmpl[None], 3, 0), haar_quaternions(rng, 3)))
    cc = CrossCorrelationMatcher(N=N1, device=cuda_device, batchsize=4, bandlimit=16, radius=radius)
    cc.set_template(tmpl)
    full, n_full = cc.get_sigma(vols.to(cuda_device))
    full, n_full = full[:3].cpu().numpy(), n_full[:3].cpu().numpy()
    for lmax in (0, 7, cc.lmax):
        part, n_part = cc.get_sigma_upto(vols.to(cuda_device), lmax)
        assert part.shape == (3, compute_size(lmax + 1))
        np.testing.assert_array_equal(part.cpu().numpy(), full[:, :compute_size(lmax + 1)])
        np.testing.assert_array_equal(n_part.cpu().numpy(), n_full)
    with pytest.raises(ValueError):
        cc.get_sigma_upto(vols.to(cuda_device), cc.lmax + 1)


def test_rotation_recovery_end_to_end(cuda_device):
    """Template rotated by known rotations, expanded, correlated and searched: the
    recovered Euler angles, composed with the tracker as the reference's benchmark
    does, must give back the identity."""
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher
    from matcha_b200.core.Matcha import Matcha

    N1, radius, Lmax = 32, 14, 16
    rng = np.random.default_rng(2024)
    tmpl = blob_template(rng, N1, 40, 12, (1.5, 3.0), mask_radius=14)
    q = haar_quaternions(rng, 8)
    vols = rotate_volumes_reference(np.repeat(tmpl[None], 8, 0), q)
    cc = CrossCorrelationMatcher(N=N1, device=cuda_device, batchsize=8, bandlimit=Lmax, radius=radius)
    cc.set_template(tmpl)
    sig, _ = cc.get_sigma(torch.from_numpy(vols).to(cuda_device))
    m = Matcha(batchsize=8, device=cuda_device, L_max=Lmax,
               matcha_config=dict(Li=[4, 8, 12], candidates=10, num_steps=1, oversampling_factor_K=2))
    a, b, g, s = (x.cpu().numpy() for x in m.search_orientations(sig))
    err = alignment_error_deg(a, b, g, q)
    assert np.median(err) < 3.0, err


@pytest.mark.parametrize("N1,bl,radius", [(32, 16, 14), (31, 12, 13)])
def test_tensor_core_split_matches_dense_definition(cuda_device, N1, bl, radius):
    """BF16 hi+lo split GEMM on tcgen05: within 1e-4 relative of the exact adjoint."""
    from matcha_b200.core.FLEBasis3D import FLEBasis3D

    fle = FLEBasis3D(N=N1, bandlimit=bl, eps=1e-4, batchsize=130, radius=radius, device=cuda_device,
                     dtype=torch.complex64, precision="bf16x3")
    rng = np.random.default_rng(3 * N1 + radius)
    vols = rng.standard_normal((130, N1, N1, N1)).astype(np.float32)  # two M tiles, the second ragged
    a = fle.evaluate_t(torch.from_numpy(vols).to(cuda_device))
    fle.status()
    a = a.cpu().numpy()
    idx = [0, 1, 127, 128, 129]
    ref = F.evaluate_t(fle.tables, vols[idx], float(radius))
    err = np.linalg.norm(a[idx] - ref) / np.linalg.norm(ref)
    assert err < 1e-4, err
    # and agrees with the FP32 CUDA-core path on every volume
    f32 = FLEBasis3D(N=N1, bandlimit=bl, eps=1e-4, batchsize=130, radius=radius, device=cuda_device,
                     dtype=torch.complex64, precision="fp32")
    b = f32.evaluate_t(torch.from_numpy(vols).to(cuda_device)).cpu().numpy()
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4


def test_tensor_core_split_at_benchmark_shape(cuda_device):
    from matcha_b200.core.FLEBasis3D import FLEBasis3D

    kw = dict(N=64, bandlimit=32, eps=1e-4, batchsize=200, radius=30, device=cuda_device, dtype=torch.complex64)
    tc = FLEBasis3D(precision="bf16x3", **kw)
    fp = FLEBasis3D(precision="fp32", **kw)
    v = torch.randn(200, 64, 64, 64, device=cuda_device)
    a, b = tc.evaluate_t(v), fp.evaluate_t(v)
    tc.status()
    rel = (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()
    assert rel < 1e-4, rel


@pytest.mark.parametrize("split_degree", [20, 40])
def test_degree_schedule_at_benchmark_shape(cuda_device, split_degree):
    """split_degree: the GEMM tiles whose columns are all of degree <= split_degree run in plain
    BF16 (one MMA per K step), the others keep the hi+lo split.  Columns are sorted by degree
    inside each parity class, so the tiles above the threshold hold the high degrees; their
    coefficients keep the split's accuracy, the plain ones BF16's (about 2e-3 relative on noise
    volumes, where nothing cancels the rounding)."""
    from matcha_b200.core.FLEBasis3D import FLEBasis3D

    kw = dict(N=64, bandlimit=32, eps=1e-4, batchsize=200, radius=30, device=cuda_device, dtype=torch.complex64)
    mixed = FLEBasis3D(precision="bf16x3", split_degree=split_degree, **kw)
    full = FLEBasis3D(precision="bf16x3", **kw)
    fp = FLEBasis3D(precision="fp32", **kw)
    n_split, n_tiles = mixed.split_tiles()
    assert full.split_tiles() == (n_tiles, n_tiles) and fp.split_tiles() == (0, 0)
    assert 0 < n_split < n_tiles, (n_split, n_tiles)
    v = torch.randn(200, 64, 64, 64, device=cuda_device)
    a, b = mixed.evaluate_t(v), fp.evaluate_t(v)
    mixed.status()
    ls = torch.from_numpy(np.asarray(mixed.ls)).to(cuda_device)
    # a tile takes the split when any of its columns is above the threshold, so every column of
    # degree > split_degree is in a split tile
    hi = ls > split_degree
    rel_hi = (torch.linalg.norm((a - b)[:, hi]) / torch.linalg.norm(b[:, hi])).item()
    rel_all = (torch.linalg.norm(a - b) / torch.linalg.norm(b)).item()
    assert rel_hi < 1e-4, rel_hi
    assert rel_all < 5e-3, rel_all


@pytest.mark.parametrize("precision,tol", [("fp32", 1e-5), ("bf16x3", 1e-4)])
@pytest.mark.parametrize("tag,N1,bl,radius", [("c16r8", 16, 8, 8), ("c32r16", 32, 16, 16), ("c32r15", 32, 16, 15)])
def test_evaluate_t_matches_reference_dense_basis(cuda_device, tag, N1, bl, radius, precision, tol):
    """Coefficients of the volumes in tests/golden/fle_ref.npz against the reference's own
    create_denseB adjoint (FLEBasis3D.py:570-698), at the FP32 and BF16 hi+lo tolerances."""
    from matcha_b200.core.FLEBasis3D import FLEBasis3D
    from tests.helpers import golden

    fx = golden("fle_ref.npz")
    vols, ref = fx[f"{tag}_volumes"], fx[f"{tag}_coeffs"]
    fle = FLEBasis3D(N=N1, bandlimit=bl, eps=1e-4, batchsize=vols.shape[0], radius=radius, device=cuda_device,
                     dtype=torch.complex64, precision=precision)
    assert fle.ne == ref.shape[1]
    a = fle.evaluate_t(torch.from_numpy(vols).to(cuda_device))
    fle.status()
    a = a.cpu().numpy()
    for i in range(vols.shape[0]):
        err = np.linalg.norm(a[i] - ref[i]) / np.linalg.norm(ref[i])
        assert err < tol, (i, err)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
@pytest.mark.parametrize("tag,N1,bl,radius", [("c16r8", 16, 8, 8), ("c32r16", 32, 16, 16)])
def test_sigma_matches_reference_compute_sigma(cuda_device, tag, N1, bl, radius, precision):
    """sigma and the norms of tests/golden/sigma_ref.npz (the reference's compute_sigma,
    CrossCorrelationMatcher.py:133-212, volume 0 as the template)."""
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher
    from tests.helpers import golden

    fx, sx = golden("fle_ref.npz"), golden("sigma_ref.npz")
    vols = fx[f"{tag}_volumes"]
    cc = CrossCorrelationMatcher(N=N1, device=cuda_device, batchsize=2, bandlimit=bl, radius=radius,
                                 precision=precision)
    cc.set_template(vols[0])
    sig, norms = cc.get_sigma(torch.from_numpy(vols).to(cuda_device))
    ref = sx[f"{tag}_sigma"]
    sig = sig.cpu().numpy()
    assert sig.shape == ref.shape
    tol = 2e-5 if precision == "fp32" else 2e-4
    for i in range(2):
        assert np.linalg.norm(sig[i] - ref[i]) / np.linalg.norm(ref[i]) < tol
    np.testing.assert_allclose(norms.cpu().numpy(), sx[f"{tag}_norms"], rtol=1e-5 if precision == "fp32" else 1e-4)
    np.testing.assert_allclose(cc.bh_norm_template.item(), sx[f"{tag}_norms"][0], rtol=1e-5 if precision == "fp32" else 1e-4)
