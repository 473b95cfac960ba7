"""Per-batch result bookkeeping: rows of store_alignment_parameters (io_utils.py:181-225)
from one packed device array, and the device-side rotation of a tracker for the shift match."""
import numpy as np
import pandas as pd
import pytest
import torch

from oracle import prepare as OP
from oracle import shift as OS
from tests.helpers import blob_template, haar_quaternions, rotate_volumes_reference

COLUMNS = ["path", "rotation_score", "shift_score", "rotation", "translation", "file_name", "grid_shift",
           "prior_shift", "alternation_index", "rlnTomoParticleName", "half"]


@pytest.mark.parametrize("path,token", [
    ("Subtomograms/TS_01/12_data.mrc", "TS_01/12"),
    ("Subtomograms/TS_01/TS_01_subtomo000012_data.mrc", "TS_01/TS_01_000012"),
    ("000004@Extract/job012/TS_03/4_weights.mrc", "TS_03/4"),
    ("C:\\runs\\TS_02\\7_ctf.mrc", "TS_02/7"),
    ("single.mrc", "single"),
])
def test_particle_token_follows_the_reference(path, token):
    """Expected tokens worked through io_utils.py:14-25 by hand."""
    from matcha_b200.results import particle_token

    assert particle_token(path) == token


def test_rows_from_a_packed_batch():
    from matcha_b200.results import append_rows

    packed = np.arange(4 * 11, dtype=np.float64).reshape(4, 11) / 8.0
    names = ["a/TS_1/1_data.mrc", "a/TS_1/2_data.mrc", "a/TS_1/3_data.mrc"]  # a padded batch of 4
    df = append_rows(pd.DataFrame(columns=COLUMNS), packed, names, "half1", alternation_index=2)
    assert len(df) == 3 and list(df.columns) == COLUMNS
    r = df.iloc[1]
    assert r["path"] == names[1] and r["file_name"] == "2_data.mrc" and r["rlnTomoParticleName"] == "TS_1/2"
    assert r["rotation_score"] == packed[1, 0] and r["shift_score"] == packed[1, 10]
    np.testing.assert_array_equal(r["rotation"], packed[1, 1:4])
    assert r["translation"].dtype == np.float32 and r["prior_shift"].dtype == np.float32
    np.testing.assert_array_equal(r["translation"], packed[1, 4:7].astype(np.float32))
    assert r["alternation_index"] == 2 and r["half"] == "half1"


@pytest.mark.gpu
def test_pack_results_matches_host_values(cuda_device, tmp_path):
    from matcha_b200.results import store_alignment_parameters

    B = 5
    rng = np.random.default_rng(5)
    q = haar_quaternions(rng, B) * np.array([[1.0], [2.0], [0.5], [1.0], [1.0]])  # norms the Euler angles ignore
    rs = rng.standard_normal(B).astype(np.float32)
    ss = rng.standard_normal(B).astype(np.float32)
    ls = rng.standard_normal((B, 1, 3)).astype(np.float32)
    ps = rng.standard_normal((B, 1, 3)).astype(np.float32)
    dev = lambda a: torch.from_numpy(a).to(cuda_device)
    cfg = {"num_subtomograms_per_batch": B, "execution": {"output_file_name": str(tmp_path / "res")}}
    names = [f"TS_9/{i}_data.mrc" for i in range(B)]
    df = store_alignment_parameters(cfg, pd.DataFrame(columns=COLUMNS), names, dev(rs), dev(ss), dev(ls), dev(q),
                                    dev(ps), "half2", alternation_index=1)
    assert (tmp_path / "res.pkl").exists()
    euler = np.deg2rad(OP.euler_zyz_deg(q))
    for i in range(B):
        r = df.iloc[i]
        assert r["rotation_score"] == float(rs[i]) and r["shift_score"] == float(ss[i])
        np.testing.assert_allclose(r["rotation"], euler[i], atol=1e-12)
        np.testing.assert_array_equal(r["translation"], ls[i, 0])
        np.testing.assert_array_equal(r["prior_shift"], ps[i, 0])


@pytest.mark.gpu
def test_tracker_rotation_on_device(cuda_device):
    from scipy.spatial.transform import Rotation

    from matcha_b200 import _native as nat

    B = 7
    q = haar_quaternions(np.random.default_rng(6), B) * 1.3
    t = torch.from_numpy(q).to(cuda_device)
    rot = torch.empty((B, 9), device=cuda_device)
    with torch.cuda.device(cuda_device):
        nat.check(nat.load().mtb_tracker_rotation(nat.ptr(t), B, nat.ptr(rot), nat.stream_ptr(cuda_device)),
                  "mtb_tracker_rotation")
    ref = Rotation.from_euler("ZYZ", OS.euler_zyz_deg_from_quat_conj(q), degrees=True).as_matrix().reshape(B, 9)
    np.testing.assert_allclose(rot.cpu().numpy(), ref, atol=1e-6)


@pytest.mark.gpu
def test_search_shifts_takes_a_device_tracker(cuda_device):
    from matcha_b200.core.ShiftMatcher import ShiftMatcher

    class Cfg(dict):
        __getattr__ = dict.__getitem__

    N, B = 32, 3
    rng = np.random.default_rng(8)
    tmpl = blob_template(rng, N, 60, N * 0.3, (1.5, 3.0), mask_radius=N * 0.4)
    q = haar_quaternions(rng, B)
    vols = rotate_volumes_reference(np.repeat(tmpl[None], B, 0), q).astype(np.float32)
    cfg = Cfg(N=N, voxel_size=1.0, num_subtomograms_per_batch=B, shift_upsample_factor=8, shift_search_radius=3,
              do_ctf_correction=False, box_size=N)
    sm = ShiftMatcher(cfg, cuda_device, torch.complex64)
    sm.set_reference(tmpl)
    v = torch.from_numpy(vols).to(cuda_device)
    prior = torch.zeros((B, 3), device=cuda_device)
    s_host, sc_host = sm.search_shifts(subtomos=v, ctfs=None, shift_zyx=prior, rotation_tracker=q)
    s_dev, sc_dev = sm.search_shifts(subtomos=v, ctfs=None, shift_zyx=prior,
                                     rotation_tracker=torch.from_numpy(q).to(cuda_device))
    np.testing.assert_allclose(s_dev.cpu().numpy(), s_host.cpu().numpy(), atol=1e-6)
    np.testing.assert_allclose(sc_dev.cpu().numpy(), sc_host.cpu().numpy(), rtol=1e-5)
