"""Subtomogram preparation of every alternation (shifted patch, normalisation in the spherical
mask, rotation into the tracker's orientation): the oracle against torch's grid_sample as the
reference calls it, and the CUDA entry point against the oracle."""
import numpy as np
import pytest
import torch

from oracle import prepare as OP
from tests.helpers import haar_quaternions, rotate_volumes_reference


def _extract_reference(vols, shift_xyz):
    """extract_subtomogram_patch_batch (src/matcha/utils/io_utils.py:113-178), torch CPU, the
    grid arithmetic as written there (float32), normalize=False."""
    import torch.nn.functional as F

    v = torch.from_numpy(np.asarray(vols, dtype=np.float32)).unsqueeze(1)
    B, _, D, H, W = v.shape
    z = torch.arange(D)
    y = torch.arange(H)
    x = torch.arange(W)
    X, Y, Z = torch.meshgrid(z, y, x, indexing="ij")
    base = torch.stack((Z, Y, X), dim=-1)
    size = torch.tensor([D, H, W]) - 1
    out = []
    for b in range(B):
        grid = base + torch.from_numpy(np.asarray(shift_xyz[b], dtype=np.float32)).view(1, 1, 1, 3)
        ng = (2 * grid / size.flip(-1).view(1, 1, 1, 3) - 1).unsqueeze(0)
        out.append(F.grid_sample(v[b:b + 1], ng, mode="bilinear", align_corners=True)[0, 0])
    return torch.stack(out).numpy()


def test_oracle_extract_matches_grid_sample():
    rng = np.random.default_rng(1)
    vols = rng.standard_normal((3, 16, 16, 16)).astype(np.float32)
    shifts = rng.uniform(-2.5, 2.5, (3, 3)).astype(np.float32)
    ref = _extract_reference(vols, shifts)
    for b in range(3):
        got = OP.extract_patch(vols[b].astype(np.float64), shifts[b].astype(np.float64))
        np.testing.assert_allclose(got, ref[b], atol=2e-5)


def test_oracle_rotation_matches_grid_sample():
    rng = np.random.default_rng(2)
    vols = rng.standard_normal((3, 16, 16, 16)).astype(np.float32)
    q = haar_quaternions(rng, 3)
    ref = rotate_volumes_reference(vols, q)
    for b in range(3):
        np.testing.assert_allclose(OP.rotate_volume(vols[b].astype(np.float64), q[b]), ref[b], atol=2e-5)


def test_oracle_identity_is_the_masked_normalised_volume():
    rng = np.random.default_rng(3)
    vol = rng.standard_normal((1, 16, 16, 16))
    mask = OP.spherical_mask(16, 7.0)
    out = OP.prepare(vol, np.zeros((1, 3)), np.array([[1.0, 0, 0, 0]]), 7.0)[0]
    np.testing.assert_allclose(out, OP.normalise_masked(vol[0], mask), atol=1e-12)
    inside = out[mask > 0]
    assert abs(inside.mean()) < 1e-12 and abs(inside.std() - 1) < 1e-12


def _prepare_gpu(vols, shifts, q, radius, device):
    from matcha_b200 import _native as nat

    lib = nat.load()
    B, N = vols.shape[0], vols.shape[1]
    v = torch.from_numpy(np.ascontiguousarray(vols, dtype=np.float32)).to(device)
    s = torch.from_numpy(np.ascontiguousarray(shifts, dtype=np.float32)).to(device)
    t = torch.from_numpy(np.ascontiguousarray(q, dtype=np.float64)).to(device)
    work = torch.empty(v.shape + (2,), dtype=torch.float32, device=device)
    stats = torch.empty((B, 2), dtype=torch.float64, device=device)
    out = torch.empty_like(v)
    with torch.cuda.device(device):
        nat.check(lib.mtb_prepare_subtomos(nat.ptr(v), B, N, nat.ptr(s), nat.ptr(t), float(radius), nat.ptr(work),
                                           nat.ptr(stats), nat.ptr(out), nat.stream_ptr(device)),
                  "mtb_prepare_subtomos")
    torch.cuda.synchronize(device)
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("N,B,radius", [(16, 3, 7.0), (15, 3, 7.0), (16, 3, 9.5), (32, 4, 15.0), (64, 2, 30.0),
                                         (64, 2, 32.0), (80, 2, 36.0), (112, 2, 50.0)])
def test_prepare_matches_oracle(cuda_device, N, B, radius):
    """Even and odd boxes, masks inside the box and reaching past it (radius 9.5 of 16); 112 is
    past the box size whose plane fits the staged patch kernel's shared memory."""
    rng = np.random.default_rng(N + B + int(radius))
    vols = (rng.standard_normal((B, N, N, N)) + 3.0).astype(np.float32)  # a mean to remove
    shifts = rng.uniform(-3, 3, (B, 3)).astype(np.float32)
    shifts[0] = np.round(shifts[0])  # an integer shift: the patch is a plain translation
    shifts[1] = [0.45 * N, -0.6 * N, 0.3]  # most of the patch outside the volume
    q = haar_quaternions(rng, B)
    q[0] = [1.0, 0.0, 0.0, 0.0]  # the identity tracker of the first alternation
    q[-1] *= 1.03  # a tracker off unit norm after many updates: its rotation is that of q / |q|
    got = _prepare_gpu(vols, shifts, q, radius, cuda_device)
    ref = OP.prepare(vols, shifts, q, radius)
    # FP32 coordinates and weights against FP64: values are O(1) after the normalisation
    np.testing.assert_allclose(got, ref, atol=2e-4)


@pytest.mark.gpu
def test_prepare_rejects_bad_arguments(cuda_device):
    from matcha_b200 import _native as nat

    lib = nat.load()
    v = torch.zeros((1, 8, 8, 8), device=cuda_device)
    s = torch.zeros((1, 3), device=cuda_device)
    t = torch.tensor([[1.0, 0, 0, 0]], dtype=torch.float64, device=cuda_device)
    st = torch.zeros((1, 2), dtype=torch.float64, device=cuda_device)
    with torch.cuda.device(cuda_device):
        rc = lib.mtb_prepare_subtomos(nat.ptr(v), 1, 8, nat.ptr(s), nat.ptr(t), 0.0, nat.ptr(v), nat.ptr(st),
                                      nat.ptr(v), nat.stream_ptr(cuda_device))
    assert rc == nat.MTB_ERR_ARG


@pytest.mark.gpu
def test_alternations_prepare_then_align(cuda_device):
    """Two alternations of rotated template copies from the identity tracker: the first
    alternation's input is the prepared batch, and the second, prepared with the tracker the
    first found, leaves a residual rotation near the identity and no shift."""
    from scipy.spatial.transform import Rotation

    from matcha_b200.pipeline import AlignmentStep, StepConfig
    from tests.helpers import blob_template

    B, N, radius = 4, 16, 7
    rng = np.random.default_rng(21)
    tmpl = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    q = haar_quaternions(rng, B)
    vols = np.stack([OP.rotate_volume(tmpl.astype(np.float64), q[b]) for b in range(B)]).astype(np.float32)
    step = AlignmentStep(StepConfig(N=N, L=12, Li=[4, 8], batch=B, radius=radius, shift_search_radius=1,
                                    shift_upsample_factor=4), cuda_device)
    step.set_template(tmpl)
    dv = torch.from_numpy(vols).to(cuda_device)
    tracker = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    tracker[:, 0] = 1
    zeros = torch.zeros((B, 3), device=cuda_device)
    local = zeros.clone()

    prepared = step.prepare(dv, zeros, tracker.clone()).cpu().numpy()
    np.testing.assert_allclose(prepared, OP.prepare(vols, np.zeros((B, 3)), tracker.cpu().numpy(), radius),
                               atol=2e-4)

    res = step.run_alternations(dv, tracker, local, zeros, zeros, num_alternations=2)
    torch.cuda.synchronize()
    assert len(res) == 2
    for r in res:
        assert torch.isfinite(r["normalized_rotation_score"]).all()
    a, b, g = (res[1][k].reshape(-1).cpu().numpy() for k in ("alpha", "beta", "gamma"))
    resid = Rotation.from_euler("ZYZ", np.stack([a, b, g], -1)).magnitude()
    assert np.all(resid < np.deg2rad(12)), np.rad2deg(resid)
    assert float(local.abs().max()) < 1.0
