"""Fixture generator: the calls the reference's own alignment driver makes on the hot path.

    MATCHA_REFERENCE_ROOT=/path/to/Matcha python tests/golden/make_caller_trace.py

Runs the reference's ``AlignmentRuntimeBuilder.prepare_config`` and its ``BatchProcessor``
(``_ensure_template``, ``_run_alternations``; src/matcha/align_subtomograms.py:69-136,
182-200, 316-361) on the CPU for 4 subtomograms of 32^3 and two alternations, with recorders
in place of the three hot-path classes:

* ``Matcha`` and ``ShiftMatcher`` are the reference's own classes (src/matcha/core/Matcha.py,
  ShiftMatcher.py) running on the CPU - the Wigner-D matrices from the oracle, as in
  ``make_golden.gen_search``, its gradients under Numba's CUDA simulator;
* ``CrossCorrelationMatcher`` computes its results with the oracle's exact expansion and
  sigma (the reference's transform needs cuFINUFFT, which is not installed; the oracle is
  pinned to the reference's dense basis by ``fle_ref.npz``).

Every constructor and method call, its arguments (tensors as arrays) and the result it
returned is written to ``caller_trace.npz``; for each orientation search the FP64 oracle's
answer on the same sigma is stored beside the reference's.  ``tests/test_caller_trace_gpu.py``
replays the calls, in order, on matcha_b200's classes.  Uses the driver shims of
``refharness.py`` (quaternionic, mrcfile) and writes nothing but the fixture and a pickle
under /tmp.
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, ROOT)

import refharness  # noqa: E402  (sets the Numba simulator flag before numba loads)

EVENTS = []
ARRAYS = {}


def _store(a, key):
    """Keep array ``a`` under ``key``, or point to an identical array stored earlier; a complex
    array whose imaginary part is zero is kept as its real part (``real_only``)."""
    a = np.ascontiguousarray(a)
    real_only = bool(np.iscomplexobj(a) and not np.any(a.imag))
    body = a.real.copy() if real_only else a
    for k, b in ARRAYS.items():
        if b.shape == body.shape and b.dtype == body.dtype and np.array_equal(b, body):
            return k, real_only
    ARRAYS[key] = body
    return key, real_only


def _plain(v, key):
    """JSON-able description of an argument or result; arrays go to ARRAYS."""
    import torch

    if isinstance(v, torch.Tensor):
        k, ro = _store(v.detach().cpu().numpy(), key)
        return {"array": k, "real_only": ro, "torch": str(v.dtype).replace("torch.", ""), "shape": list(v.shape)}
    if isinstance(v, np.ndarray):
        quat = type(v).__name__ == "QArray"
        k, ro = _store(np.asarray(v).view(np.ndarray), key)
        return {"array": k, "real_only": ro, "numpy": str(np.asarray(v).dtype), "shape": list(v.shape),
                "quaternionic": quat}
    if isinstance(v, torch.dtype):
        return {"dtype": str(v).replace("torch.", "")}
    if isinstance(v, torch.device):
        return {"device": str(v)}
    if isinstance(v, (tuple, list)):
        return [_plain(x, f"{key}_{i}") for i, x in enumerate(v)]
    if isinstance(v, dict):
        return {str(k): _plain(x, f"{key}_{k}") for k, x in v.items()
                if k != "execution" and not str(k).startswith("_")}
    if isinstance(v, (bool, int, float, str)) or v is None:
        return v
    if isinstance(v, np.generic):
        return v.item()
    return {"repr": repr(v)[:80]}


def record(call, args, result):
    i = len(EVENTS)
    EVENTS.append({"call": call, "args": _plain(args, f"e{i}_arg"), "result": _plain(result, f"e{i}_res")})
    return i


def _reference_classes():
    """The reference's Matcha and ShiftMatcher classes (loaded before the recorders replace
    their modules) and the oracle D hook of make_golden."""
    import make_golden as MG

    refharness.install_driver_shims()
    MG._install_spherical_stub()
    refharness.load_wigner_module()
    Mmod = refharness.load_module("matcha.core.Matcha")
    Smod = refharness.load_module("matcha.core.ShiftMatcher")
    return Mmod.Matcha, Smod.ShiftMatcher


def main():
    import torch

    RefMatcha, RefShift = _reference_classes()
    from matcha_b200.core import fle_tables as T
    from oracle import fle as OF
    from oracle import matcha as OM
    from oracle import pipeline as OP
    from oracle import wigner as W
    from tests.helpers import blob_template, make_subtomograms

    class RecordingCorrelator:
        """CrossCorrelationMatcher: the oracle's exact expansion and sigma."""

        def __init__(self, N, device, expansion_epsilon=1e-4, batchsize=1, reduce_memory=True, bandlimit=None,
                     micro_batch_split=2, dtype=torch.float32, radius=None, jl_zeros_path=None, cs_path=None,
                     precision_mode="accurate"):
            record("CrossCorrelationMatcher", dict(N=N, device=device, expansion_epsilon=expansion_epsilon,
                                                   batchsize=batchsize, reduce_memory=reduce_memory,
                                                   bandlimit=bandlimit, micro_batch_split=micro_batch_split,
                                                   dtype=dtype, radius=radius, jl_zeros_path=jl_zeros_path,
                                                   cs_path=cs_path, precision_mode=precision_mode), None)
            self.tables = T.lap_eig_ball(int(N), bandlimit, float(radius))
            self.ff = OP.FoldedFLE(self.tables, int(N), float(radius))
            self.lmax = self.tables.lmax
            self.batchsize = batchsize
            self.bh_norm_template = None

        def set_template(self, template_data, mask=None):
            self.a_t = self.ff.evaluate_t(np.asarray(template_data, dtype=np.float64)[None])[0]
            self.bh_norm_template = torch.tensor(float(np.linalg.norm(self.a_t)), dtype=torch.float32)
            record("CrossCorrelationMatcher.set_template", dict(template_data=template_data, mask=mask),
                   dict(bh_norm_template=self.bh_norm_template))

        def get_sigma(self, volumes):
            v = volumes.real if volumes.is_complex() else volumes
            a = self.ff.evaluate_t(v.double().numpy())
            sig = OF.compute_sigma(self.tables, self.a_t, a)
            out = (torch.from_numpy(sig.astype(np.complex64)), torch.from_numpy(np.linalg.norm(a, axis=1).astype(np.float32)))
            record("CrossCorrelationMatcher.get_sigma", dict(volumes=volumes), list(out))
            return out

    class RecordingMatcha(RefMatcha):
        def __init__(self, batchsize, device, L_max, matcha_config):
            record("Matcha", dict(batchsize=batchsize, device=device, L_max=L_max, matcha_config=dict(matcha_config)),
                   None)
            cwd = os.getcwd()
            tmp = os.path.join("/tmp", "matcha_ref_cache")
            os.makedirs(tmp, exist_ok=True)
            os.chdir(tmp)
            try:
                super().__init__(batchsize=batchsize, device=device, L_max=L_max, matcha_config=matcha_config)
            finally:
                os.chdir(cwd)
            Lmax = L_max

            def D_oracle(q=None, alpha=None, beta=None, gamma=None, truncate=None):
                t = Lmax if truncate is None else int(truncate)
                D = W.wigner_D(alpha.double().numpy(), beta.double().numpy(), gamma.double().numpy(), t)
                if t == Lmax:
                    ls, mps, ms = W.lmm(t)
                    D[..., (ls == t) & ((mps == -t) | (ms == -t))] = 0.0
                return torch.from_numpy(D.astype(np.complex64))

            self.WignerDMatrices.D = D_oracle
            self._cfg = dict(matcha_config)
            self._Lmax = L_max

        def search_orientations(self, sigma, *args, **kw):
            out = super().search_orientations(sigma.clone(), *args, **kw)
            c = self._cfg
            ex = OM.search_orientations(sigma.numpy().astype(np.complex128), list(c["Li"]), self._Lmax,
                                        K=c.get("oversampling_factor_K", 2), candidates=c["candidates"],
                                        num_steps=c["num_steps"], dtype=np.float64)
            record("Matcha.search_orientations", dict(sigma=sigma),
                   dict(result=list(out), fp64=[np.asarray(x, dtype=np.float64) for x in ex]))
            return out

    class RecordingShift(RefShift):
        def __init__(self, config, device, dtype, micro_batch_size=None):
            record("ShiftMatcher", dict(config=dict(config), device=device, dtype=dtype), None)
            super().__init__(config=config, device=device, dtype=dtype, micro_batch_size=micro_batch_size)

        def set_reference(self, template_data):
            super().set_reference(template_data)
            record("ShiftMatcher.set_reference", dict(template_data=template_data), None)

        def get_base_shifts(self, num_subtomograms_per_batch, num_base_shifts, dtype_real):
            out = super().get_base_shifts(num_subtomograms_per_batch=num_subtomograms_per_batch,
                                          num_base_shifts=num_base_shifts, dtype_real=dtype_real)
            record("ShiftMatcher.get_base_shifts", dict(num_subtomograms_per_batch=num_subtomograms_per_batch,
                                                        num_base_shifts=num_base_shifts, dtype_real=dtype_real), out)
            return out

        def search_shifts(self, *, subtomos, ctfs, shift_zyx, rotation_tracker, micro_batch_size=None):
            out = super().search_shifts(subtomos=subtomos, ctfs=ctfs, shift_zyx=shift_zyx,
                                        rotation_tracker=rotation_tracker, micro_batch_size=micro_batch_size)
            record("ShiftMatcher.search_shifts", dict(subtomos=subtomos, ctfs=ctfs, shift_zyx=shift_zyx,
                                                      rotation_tracker=rotation_tracker), list(out))
            return out

    for name, cls in (("CrossCorrelationMatcher", RecordingCorrelator), ("Matcha", RecordingMatcha),
                      ("ShiftMatcher", RecordingShift)):
        mod = types.ModuleType(f"matcha.core.{name}")
        setattr(mod, name, cls)
        sys.modules[f"matcha.core.{name}"] = mod
    torch.cuda.set_device = lambda *a, **k: None  # the driver selects a GPU; everything here is on the CPU
    A = refharness.load_module("matcha.align_subtomograms")
    A.AlignmentRuntimeBuilder._resolve_device = staticmethod(lambda gpu_id: torch.device("cpu"))
    from matcha.utils.setup_utils import get_rotation_tracker

    N, B = 32, 4
    out_dir = os.path.join("/tmp", "matcha_caller_trace")
    os.makedirs(out_dir, exist_ok=True)
    cfg = refharness._ConfigDict(
        N=N, gpu_id=0, random_seed=42, precision="float32", radius=N // 2, path_template_mask="",
        expansion_epsilon=1e-4, precision_mode="fast", reduce_memory=True, micro_batch_split=2,
        num_subtomograms_per_batch=B,
        matcha_config=dict(Li=[4, 8, 12, 16], candidates=10, num_steps=2, oversampling_factor_K=2),
        matcha_config_expert=dict(reinits=1, step_type="newton", stop_early=False, do_random_sampling=False,
                                  reinits_iterations=0),
        jl_zeros_path="jl_zeros_l=3000_k=2500.mat", cs_path="cs_l=3000_k=2500.mat", num_alternations=2,
        shift_search_radius=3, shift_upsample_factor=8, do_ctf_correction=False, box_size=N, voxel_size=1.0,
        path_output=os.path.join(out_dir, "result"), use_prior_rotation=False)
    runtime = A.AlignmentRuntimeBuilder.prepare_config(cfg)

    class _Stream:
        def wait_event(self, ev):
            pass

    bp = A.BatchProcessor(runtime, df=None, compute_stream=_Stream(), num_subtomograms_per_batch=B,
                          num_base_shifts=1)
    rng = np.random.default_rng(2024)
    tmpl = blob_template(rng, N, 40, 12, (1.5, 3.0), mask_radius=14)
    refharness.MRC_FILES["template_half1.mrc"] = tmpl
    vols, q_true, shifts = make_subtomograms(tmpl, rng, B, 2.0)
    bp._ensure_template("template_half1.mrc")
    bp._set_output_target("half1")
    names = [f"particle_{i:03d}.mrc" for i in range(B)]
    base = bp.shift_matcher.get_base_shifts(num_subtomograms_per_batch=B, num_base_shifts=1, dtype_real=torch.float32)
    tracker = get_rotation_tracker(tomogram_file_names=names, df=None, config=runtime)
    local = torch.zeros((B, 1, 3), dtype=torch.float32)
    prior = torch.zeros((B, 1, 3), dtype=torch.float32)
    subtomograms = torch.from_numpy(vols)
    bp._run_alternations(subtomograms=subtomograms, subtomos=subtomograms.clone(), ctfs=None, ev_ctf=None,
                         tomogram_file_names=names, half="half1", base_shifts=base, local_shifts=local,
                         rotation_tracker=tracker, prior_shifts=prior)
    ARRAYS["true_quaternions"] = q_true
    ARRAYS["true_shifts"] = shifts
    calls = [e["call"] for e in EVENTS]
    print("\n".join(calls))
    np.savez_compressed(os.path.join(HERE, "caller_trace.npz"), events=np.array(json.dumps(EVENTS)), **ARRAYS)
    print("caller_trace.npz:", len(EVENTS), "events")


if __name__ == "__main__":
    main()
