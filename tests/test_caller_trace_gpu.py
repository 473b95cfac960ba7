"""The reference's own alignment driver, replayed on the drop-in classes.

``tests/golden/caller_trace.npz`` (``tests/golden/make_caller_trace.py``) holds every call
that the reference's ``AlignmentRuntimeBuilder.prepare_config`` and ``BatchProcessor``
(``_ensure_template``, ``_run_alternations``; src/matcha/align_subtomograms.py:69-136,
182-200, 316-361) made on the three hot-path classes, for 4 subtomograms of 32^3 and two
alternations with ``precision_mode: fast`` - recorded on the CPU with the reference's own
``Matcha`` and ``ShiftMatcher`` answering and the oracle's exact expansion standing in for its
``CrossCorrelationMatcher``.  Here the same calls, with the same arguments and in the same
order, go to matcha_b200's classes on the GPU, and each answer is compared with the
reference's:

* every constructor and method call is accepted with the recorded keyword arguments;
* every result has the type, shape and dtype the driver consumed;
* sigma within 2e-4 and the norms within 1e-4 relative (the BF16 hi+lo expansion that
  ``precision_mode: fast`` selects);
* orientations within 0.05 degrees of the reference's, or of the FP64 oracle's on the same
  sigma where the reference's FP32 march took another accept/reject decision (recorded
  beside it); rotation scores within 1e-3 relative;
* shifts identical on the 1/uf grid and their scores within 1e-4, except where the oracle's
  own correlation grid has a near-tie at the pick.
"""
import json

import numpy as np
import pytest
import torch

from tests.helpers import euler_dist_deg, golden

pytestmark = pytest.mark.gpu

ROT_TOL_DEG = 0.05
TIE_REL = 1e-5


class _Cfg(dict):
    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as exc:
            raise AttributeError(k) from exc


def _value(z, d, device):
    """The recorded argument ``d`` as the driver passed it (tensors on ``device``)."""
    if isinstance(d, dict) and "array" in d and "shape" in d:
        a = z[d["array"]]
        if "torch" in d:
            t = torch.from_numpy(np.ascontiguousarray(a)).to(device)
            return t.to(getattr(torch, d["torch"]))
        return np.asarray(a, dtype=d["numpy"])
    if isinstance(d, dict) and set(d) == {"dtype"}:
        return getattr(torch, d["dtype"])
    if isinstance(d, dict) and set(d) == {"device"}:
        return device
    if isinstance(d, list):
        return [_value(z, x, device) for x in d]
    if isinstance(d, dict):
        return {k: _value(z, v, device) for k, v in d.items()}
    return d


def _check_like(got, rec):
    """Same kind, shape and dtype as the recorded result."""
    assert isinstance(got, torch.Tensor), type(got)
    assert list(got.shape) == rec["shape"], (list(got.shape), rec["shape"])
    assert str(got.dtype).replace("torch.", "") == rec["torch"], (got.dtype, rec["torch"])


def test_reference_driver_calls_replay_on_the_drop_in_classes(cuda_device):
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher
    from matcha_b200.core.Matcha import Matcha
    from matcha_b200.core.ShiftMatcher import ShiftMatcher
    from oracle import shift as OS

    z = golden("caller_trace.npz")
    events = json.loads(str(z["events"]))
    obj = {}
    seen = []
    for ev in events:
        call, args, res = ev["call"], ev["args"], ev["result"]
        seen.append(call)
        kw = _value(z, args, cuda_device)
        if call == "CrossCorrelationMatcher":
            obj["ccm"] = CrossCorrelationMatcher(**kw)
        elif call == "Matcha":
            obj["matcha"] = Matcha(**kw)
        elif call == "ShiftMatcher":
            kw["config"] = _Cfg(kw["config"])
            obj["shift"] = ShiftMatcher(**kw)
        elif call == "CrossCorrelationMatcher.set_template":
            kw["template_data"] = np.asarray(kw["template_data"])
            obj["ccm"].set_template(**kw)
            ref = float(np.asarray(z[res["bh_norm_template"]["array"]]).reshape(-1)[0])
            assert abs(float(obj["ccm"].bh_norm_template) - ref) <= 1e-4 * ref
        elif call == "ShiftMatcher.set_reference":
            obj["shift"].set_reference(template_data=np.asarray(kw["template_data"]))
            template = np.asarray(kw["template_data"])
        elif call == "ShiftMatcher.get_base_shifts":
            got = obj["shift"].get_base_shifts(**kw)
            _check_like(got, res)
            np.testing.assert_array_equal(got.cpu().numpy(), z[res["array"]])
        elif call == "CrossCorrelationMatcher.get_sigma":
            sig, norms = obj["ccm"].get_sigma(kw["volumes"])
            _check_like(sig, res[0])
            _check_like(norms, res[1])
            rs, rn = z[res[0]["array"]], z[res[1]["array"]]
            s = sig.cpu().numpy()
            for i in range(s.shape[0]):
                assert np.linalg.norm(s[i] - rs[i]) / np.linalg.norm(rs[i]) < 2e-4, i
            np.testing.assert_allclose(norms.cpu().numpy(), rn, rtol=1e-4)
        elif call == "Matcha.search_orientations":
            out = obj["matcha"].search_orientations(sigma=kw["sigma"])
            assert len(out) == 4
            for g, r in zip(out, res["result"]):
                _check_like(g, r)
            got = [x.cpu().numpy().astype(np.float64) for x in out]
            ref = [z[r["array"]].astype(np.float64) for r in res["result"]]
            ex = [z[r["array"]] for r in res["fp64"]]
            d_ref = euler_dist_deg(*got[:3], *ref[:3])
            d_ex = euler_dist_deg(*got[:3], *ex[:3])
            assert np.all((d_ref < ROT_TOL_DEG) | (d_ex < ROT_TOL_DEG)), (d_ref, d_ex)
            close = d_ref < ROT_TOL_DEG
            np.testing.assert_allclose(got[3][close], ref[3][close], rtol=1e-3)
        elif call == "ShiftMatcher.search_shifts":
            trk = np.asarray(kw["rotation_tracker"])
            shift, score = obj["shift"].search_shifts(subtomos=kw["subtomos"], ctfs=kw["ctfs"],
                                                      shift_zyx=kw["shift_zyx"], rotation_tracker=trk)
            _check_like(shift, res[0])
            _check_like(score, res[1])
            rsh, rsc = z[res[0]["array"]], z[res[1]["array"]]
            g_sh, g_sc = shift.cpu().numpy(), score.cpu().numpy()
            cfg = obj["shift"].config
            uf, r = int(cfg["shift_upsample_factor"]), int(cfg["shift_search_radius"])
            ref_f = OS.load_reference_full(template, int(cfg["N"]), 1.0)
            ang = OS.euler_zyz_deg_from_quat_conj(trk)
            vols = kw["subtomos"].cpu().numpy().astype(np.float64)
            prior = kw["shift_zyx"].cpu().numpy().reshape(-1, 3).astype(np.float64)
            for i in range(g_sh.shape[0]):
                if np.abs(g_sh[i] - rsh[i]).max() <= 1e-6:
                    np.testing.assert_allclose(g_sc[i], rsc[i], rtol=1e-4)
                    continue
                (_, _), parts = OS.estimate_shift_like_relion(ref_f, vols[i], prior[i], ang[i], uf, r,
                                                              return_parts=True)
                grid = parts["grid"]
                U = grid.shape[0]
                idx = np.rint(g_sh[i][::-1] * uf + np.floor(U / 2.0)).astype(int)
                assert np.all((idx >= 0) & (idx < U)), (i, g_sh[i], rsh[i])
                assert grid.max() - grid[tuple(idx)] <= TIE_REL * abs(grid.max()), (i, g_sh[i], rsh[i])
        else:
            raise AssertionError(f"unexpected call {call}")
    # the driver built the three matchers, prepared the template and ran two alternations
    assert seen.count("CrossCorrelationMatcher.get_sigma") == 2
    assert seen.count("Matcha.search_orientations") == 2
    assert seen.count("ShiftMatcher.search_shifts") == 2
