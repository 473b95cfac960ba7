"""Shift match on the GPU against the oracle and the reference fixture."""
import numpy as np
import pytest
import torch

from oracle import shift as OS
from tests.helpers import blob_template, golden, haar_quaternions, rotate_volumes_reference

pytestmark = pytest.mark.gpu


class Cfg(dict):
    __getattr__ = dict.__getitem__


def _matcher(N, B, uf, r, device, box=None, precision="fp32"):
    from matcha_b200.core.ShiftMatcher import ShiftMatcher

    cfg = Cfg(N=N, voxel_size=1.0, num_subtomograms_per_batch=B, shift_upsample_factor=uf, shift_search_radius=r,
              do_ctf_correction=False, box_size=box if box is not None else N)
    return ShiftMatcher(cfg, device, torch.complex64, precision=precision)


def test_shift_matches_reference_fixture(cuda_device):
    z = golden("shift_ref.npz")
    N, uf, r = int(z["N"]), int(z["uf"]), int(z["radius"])
    sm = _matcher(N, 3, uf, r, cuda_device)
    sm.set_reference(z["template"])
    ref_host = sm.reference_data_fourier[0].cpu().numpy()
    np.testing.assert_allclose(ref_host, z["ref_fourier"], atol=1e-6 * np.abs(z["ref_fourier"]).max())
    # trackers whose conjugate has the fixture's Euler angles
    q = z["quats"]
    shift, score = sm.search_shifts(subtomos=torch.from_numpy(z["subtomos"]).to(cuda_device), ctfs=None,
                                    shift_zyx=torch.from_numpy(z["prior_zyx"]).to(cuda_device), rotation_tracker=q)
    np.testing.assert_allclose(shift.cpu().numpy(), z["shift_xyz"], atol=1e-6)
    np.testing.assert_allclose(score.cpu().numpy(), z["score"], rtol=2e-5)


@pytest.mark.parametrize("N,uf,r,precision", [(32, 8, 3, "fp32"), (64, 8, 5, "fp32"), (32, 4, 2, "fp32"),
                                              (64, 8, 5, "bf16x3"), (32, 8, 3, "bf16x3"),
                                              (16, 4, 1, "bf16x3"), (32, 4, 2, "bf16x3"),
                                              (32, 8, 5, "bf16x3"), (16, 8, 5, "bf16x3"),
                                              (128, 8, 8, "auto"), (48, 8, 6, "fp32"), (96, 8, 6, "auto"),
                                              (80, 4, 3, "fp32"),
                                              # the unfused tensor-core passes: boxes outside the fused
                                              # kernels, and U > 128 (two column parts of the N-tile)
                                              (128, 8, 8, "bf16x3"), (96, 8, 6, "bf16x3"), (48, 8, 6, "bf16x3"),
                                              (80, 4, 3, "bf16x3"), (64, 8, 8, "bf16x3"), (32, 8, 9, "bf16x3"),
                                              (128, 8, 8, "fp32")])
def test_shift_matches_oracle(cuda_device, N, uf, r, precision):
    rng = np.random.default_rng(N + uf + r)
    tmpl = blob_template(rng, N, 60, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    B = 3
    q = haar_quaternions(rng, B)
    vols = rotate_volumes_reference(np.repeat(tmpl[None], B, 0), q)
    vols = (vols + 0.5 * rng.standard_normal(vols.shape)).astype(np.float32)
    prior = rng.uniform(-1.5, 1.5, (B, 3)).astype(np.float32)
    sm = _matcher(N, B, uf, r, cuda_device, precision=precision)
    sm.set_reference(tmpl)
    shift, score = sm.search_shifts(subtomos=torch.from_numpy(vols).to(cuda_device), ctfs=None,
                                    shift_zyx=torch.from_numpy(prior).to(cuda_device), rotation_tracker=q)
    sm.status()
    shift, score = shift.cpu().numpy(), score.cpu().numpy()
    tol = 3e-5 if precision == "fp32" else 1e-4
    ref = OS.load_reference_full(tmpl, N, 1.0)
    ang = OS.euler_zyz_deg_from_quat_conj(q)
    for b in range(B):
        (s_ref, sc_ref), parts = OS.estimate_shift_like_relion(ref, vols[b], prior[b], ang[b], uf, r,
                                                               return_parts=True)
        grid = parts["grid"].ravel()
        top2 = np.sort(grid)[-2:]
        if (top2[1] - top2[0]) > tol * abs(top2[1]):  # unique peak at this precision
            np.testing.assert_allclose(shift[b], s_ref, atol=1e-6)
        np.testing.assert_allclose(score[b], sc_ref, rtol=tol)


@pytest.mark.parametrize("N,uf,r,B", [(128, 4, 1, 1), (96, 8, 6, 1), (32, 8, 15, 2), (48, 2, 0, 5), (64, 4, 15, 2)])
def test_shift_tensor_path_edges_match_oracle(cuda_device, N, uf, r, B):
    """Edges of the tensor-core geometry: a single subtomogram (one partial row tile per pass),
    U = 248 at box 32 (N-tile and pass-3 tile at their 256-column limit, the two TMEM
    accumulators filling its 512 columns), U = 2 at box 48, and U = 124 at box 64 (2U fits the
    fused kernel's N-tile but its shared memory does not: the unfused passes run)."""
    rng = np.random.default_rng(N * 7 + r)
    tmpl = blob_template(rng, N, 60, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    q = haar_quaternions(rng, B)
    vols = rotate_volumes_reference(np.repeat(tmpl[None], B, 0), q)
    vols = (vols + 0.5 * rng.standard_normal(vols.shape)).astype(np.float32)
    prior = rng.uniform(-1.0, 1.0, (B, 3)).astype(np.float32)
    sm = _matcher(N, B, uf, r, cuda_device, precision="bf16x3")
    sm.set_reference(tmpl)
    shift, score = sm.search_shifts(subtomos=torch.from_numpy(vols).to(cuda_device), ctfs=None,
                                    shift_zyx=torch.from_numpy(prior).to(cuda_device), rotation_tracker=q)
    sm.status()
    assert sm.effective_precision == "bf16x3"
    shift, score = shift.cpu().numpy(), score.cpu().numpy()
    ref = OS.load_reference_full(tmpl, N, 1.0)
    ang = OS.euler_zyz_deg_from_quat_conj(q)
    for b in range(B):
        (s_ref, sc_ref), parts = OS.estimate_shift_like_relion(ref, vols[b], prior[b], ang[b], uf, r,
                                                               return_parts=True)
        grid = parts["grid"].ravel()
        top2 = np.sort(grid)[-2:]
        if (top2[1] - top2[0]) > 1e-4 * abs(top2[1]):
            np.testing.assert_allclose(shift[b], s_ref, atol=1e-6)
        np.testing.assert_allclose(score[b], sc_ref, rtol=1e-4)


def test_shift_requires_reference(cuda_device):
    sm = _matcher(16, 1, 4, 1, cuda_device)
    with pytest.raises(RuntimeError):
        sm.search_shifts(subtomos=torch.zeros((1, 16, 16, 16), device=cuda_device), ctfs=None,
                         shift_zyx=torch.zeros((1, 3), device=cuda_device), rotation_tracker=np.array([[1.0, 0, 0, 0]]))


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_shift_profile_records_kernel_groups(cuda_device, precision):
    N, B = 32, 2
    rng = np.random.default_rng(3)
    tmpl = blob_template(rng, N, 30, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    vols = torch.from_numpy(np.repeat(tmpl[None], B, 0)).to(cuda_device)
    sm = _matcher(N, B, 8, 3, cuda_device, precision=precision)
    sm.set_reference(tmpl)
    q = np.tile([1.0, 0, 0, 0], (B, 1))
    z = torch.zeros((B, 3), device=cuda_device)
    first = sm.search_shifts(subtomos=vols, ctfs=None, shift_zyx=z, rotation_tracker=q)
    sm.profile(3)
    for _ in range(2):
        again = sm.search_shifts(subtomos=vols, ctfs=None, shift_zyx=z, rotation_tracker=q)
    ms, calls = sm.profile_read()
    assert calls == 2
    assert set(ms) == set(sm.PROFILE_STAGES)
    assert all(v >= 0 for v in ms.values()) and ms["patch_xy_fft"] > 0 and ms["updft_pass23"] > 0
    if precision == "bf16x3":  # the FP32 path has no Nyquist kernel: its entry is two adjacent events
        assert ms["nyquist"] > 0
    sm.profile(0)
    assert sm.profile_read() == ({k: 0.0 for k in sm.PROFILE_STAGES}, 0)
    np.testing.assert_array_equal(again[0].cpu().numpy(), first[0].cpu().numpy())


def test_shift_tensor_path_many_tiles_per_cta(cuda_device):
    """B = 40 at 64^3, uf 8, r 5: 840 pass-2/3 tiles, several per persistent CTA, against the
    FP32 path (itself checked against the oracle above)."""
    N, B = 64, 40
    rng = np.random.default_rng(11)
    tmpl = blob_template(rng, N, 60, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    vols = torch.from_numpy(np.repeat(tmpl[None], B, 0) + 0.5 * rng.standard_normal((B, N, N, N)).astype(np.float32))
    vols = vols.to(cuda_device)
    q = haar_quaternions(rng, B)
    z = torch.from_numpy(rng.uniform(-1.5, 1.5, (B, 3)).astype(np.float32)).to(cuda_device)
    out = {}
    for precision in ("fp32", "bf16x3"):
        sm = _matcher(N, B, 8, 5, cuda_device, precision=precision)
        sm.set_reference(tmpl)
        shift, score = sm.search_shifts(subtomos=vols, ctfs=None, shift_zyx=z, rotation_tracker=q)
        sm.status()
        out[precision] = (shift.cpu().numpy(), score.cpu().numpy())
    np.testing.assert_allclose(out["bf16x3"][1], out["fp32"][1], rtol=1e-4)
    same = np.all(np.abs(out["bf16x3"][0] - out["fp32"][0]) <= 1e-6, axis=1)
    assert same.mean() >= 0.9, same


@pytest.mark.parametrize("N,uf,r,B", [(128, 8, 8, 12), (96, 8, 6, 40)])
def test_shift_unfused_tensor_path_many_tiles(cuda_device, N, uf, r, B):
    """The unfused tensor-core passes over many row tiles per persistent CTA (at 128^3, r 8: two
    column parts per tile and 145 pass-3 tiles per subtomogram) against the FP32 path, itself
    checked against the oracle above."""
    rng = np.random.default_rng(N + B)
    tmpl = blob_template(rng, N, 80, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    vols = torch.from_numpy(np.repeat(tmpl[None], B, 0) + 0.5 * rng.standard_normal((B, N, N, N)).astype(np.float32))
    vols = vols.to(cuda_device)
    q = haar_quaternions(rng, B)
    z = torch.from_numpy(rng.uniform(-1.5, 1.5, (B, 3)).astype(np.float32)).to(cuda_device)
    out = {}
    for precision in ("fp32", "bf16x3"):
        sm = _matcher(N, B, uf, r, cuda_device, precision=precision)
        sm.set_reference(tmpl)
        shift, score = sm.search_shifts(subtomos=vols, ctfs=None, shift_zyx=z, rotation_tracker=q)
        sm.status()
        assert sm.effective_precision == precision
        out[precision] = (shift.cpu().numpy(), score.cpu().numpy())
        del sm
    np.testing.assert_allclose(out["bf16x3"][1], out["fp32"][1], rtol=1e-4)
    same = np.all(np.abs(out["bf16x3"][0] - out["fp32"][0]) <= 1e-6, axis=1)
    assert same.mean() >= 0.9, same


def test_shift_nan_subtomogram_follows_argmax_order(cuda_device):
    """A NaN voxel makes the subtomogram's whole correlation grid NaN; argmax then takes the
    first grid point, as torch.argmax and numpy.argmax do, on both paths.  The other
    subtomograms of the batch are unaffected."""
    N, B = 32, 3
    rng = np.random.default_rng(5)
    tmpl = blob_template(rng, N, 60, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    vols = np.repeat(tmpl[None], B, 0) + 0.3 * rng.standard_normal((B, N, N, N)).astype(np.float32)
    clean = torch.from_numpy(vols.copy()).to(cuda_device)
    vols[1, 7, 9, 11] = np.nan
    dirty = torch.from_numpy(vols).to(cuda_device)
    q = haar_quaternions(rng, B)
    z = torch.zeros((B, 3), device=cuda_device)
    out = {}
    for precision in ("fp32", "bf16x3"):
        sm = _matcher(N, B, 8, 3, cuda_device, precision=precision)
        sm.set_reference(tmpl)
        s_d, c_d = sm.search_shifts(subtomos=dirty, ctfs=None, shift_zyx=z, rotation_tracker=q)
        s_c, c_c = sm.search_shifts(subtomos=clean, ctfs=None, shift_zyx=z, rotation_tracker=q)
        sm.status()
        s_d, c_d, s_c, c_c = (t.cpu().numpy() for t in (s_d, c_d, s_c, c_c))
        assert np.isnan(c_d[1]) and np.all(np.isfinite(c_d[[0, 2]]))
        assert s_d[1, 0] == s_d[1, 1] == s_d[1, 2] < 0  # flat index 0: u0 = u1 = u2 = 0
        np.testing.assert_array_equal(s_d[[0, 2]], s_c[[0, 2]])
        np.testing.assert_allclose(c_d[[0, 2]], c_c[[0, 2]], rtol=1e-6)  # norms sum in any order
        out[precision] = s_d[1]
    np.testing.assert_array_equal(out["bf16x3"], out["fp32"])


@pytest.mark.parametrize("N,voxel", [(32, 1.0), (15, 1.0), (48, 1.7), (16, 0.6)])
def test_shift_reference_on_device_matches_oracle(cuda_device, N, voxel):
    """set_reference computes load_reference_full on the device (FP64 DFTs): odd and even boxes,
    low-pass radii from the voxel size; the result is complex64."""
    rng = np.random.default_rng(N)
    tmpl = blob_template(rng, N, 30, N * 0.3, (1.0, 2.5), mask_radius=N * 0.4).astype(np.float64)
    tmpl += 1e-3 * rng.standard_normal(tmpl.shape)  # FP64 detail below float32 resolution
    sm = _matcher(N, 1, 4, 1, cuda_device)
    sm.config["voxel_size"] = voxel
    sm.set_reference(tmpl)
    ref = OS.load_reference_full(tmpl, N, voxel)
    got = sm.reference_data_fourier[0].cpu().numpy()
    assert got.dtype == np.complex64
    np.testing.assert_allclose(got, ref, atol=2e-7 * np.abs(ref).max(), rtol=0)


def test_precision_selection(cuda_device):
    """bf16x3 on a box the tensor-core kernels do not cover is an error, not a silent FP32 run;
    "auto" says what it resolved to; without the argument the config decides (b200.precision,
    else precision_mode "fast" -> "auto", "accurate" -> "fp32")."""
    from matcha_b200.core.ShiftMatcher import ShiftMatcher

    with pytest.raises(ValueError):
        sm = _matcher(8, 1, 4, 1, cuda_device, precision="bf16x3")
        sm._handle(1)
    for N, want in ((8, "fp32"), (64, "bf16x3"), (128, "bf16x3"), (96, "bf16x3")):
        sm = _matcher(N, 1, 8 if N > 8 else 4, {8: 1, 64: 5, 128: 8, 96: 6}[N], cuda_device, precision="auto")
        sm._handle(1)
        assert sm.effective_precision == want
    base = dict(N=64, voxel_size=1.0, num_subtomograms_per_batch=2, shift_upsample_factor=8, shift_search_radius=5,
                do_ctf_correction=False, box_size=64)
    for extra, want in (({"precision_mode": "fast"}, "auto"), ({"precision_mode": "accurate"}, "fp32"), ({}, "fp32"),
                        ({"precision_mode": "fast", "b200": {"precision": "fp32"}}, "fp32"),
                        ({"b200": {"precision": "bf16x3"}}, "bf16x3")):
        sm = ShiftMatcher(Cfg(**base, **extra), cuda_device, torch.complex64)
        assert sm.precision == want, (extra, sm.precision)
