"""One alternation of the alignment hot path for a batch, entirely on the device.

Mirrors ``BatchProcessor._search_rotation`` + ``_search_shift``
(src/matcha/align_subtomograms.py:254-285): correlation coefficients of the batch
(``CrossCorrelationMatcher.get_sigma``), orientation search (``Matcha.search_orientations``),
rotation-tracker update (``update_rotation_estimate``, src/matcha/utils/rotation_ops.py:23-34)
and the shift match (``ShiftMatcher.search_shifts``).  The tracker update and the
rotation the shift match needs are computed on the device (``mtb_update_rotation``), so a
step issues no host synchronisation and can be captured in a CUDA graph.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as nat
from .core.CrossCorrelationMatcher import CrossCorrelationMatcher
from .core.Matcha import Matcha
from .core.ShiftMatcher import ShiftMatcher


@dataclass
class StepConfig:
    N: int = 64
    L: int = 32                      # L_max of the march; FLE bandlimit = L (align_subtomograms.py:125-134)
    Li: list = field(default_factory=lambda: [8, 16, 24])
    batch: int = 1000
    radius: int | None = None        # ball radius; default min(N//2, int(0.95 N/2)) (align_subtomograms.py:94)
    candidates: int = 10
    num_steps: int = 1
    K: int = 2
    shift_upsample_factor: int = 8
    shift_search_radius: int = 5
    box_size: float | None = None
    voxel_size: float = 1.0
    shift_tile_rows: int = 0         # FP32 upsampled DFT tile (0: default), set by matcha_b200.autotune
    precision: str = "auto"          # dense contractions (ball expansion, upsampled DFT): "bf16x3" on
                                     # tcgen05 with a hi+lo split (an error where the shift kernels do
                                     # not cover the box), "fp32" on CUDA cores, or "auto": the
                                     # expansion on tcgen05 and the upsampled DFT there where its
                                     # kernels cover the box (ShiftMatcher.effective_precision)
    expansion_split_degree: int | None = None  # tensor-core expansion: plain BF16 for the columns
                                     # of degree <= this, the hi+lo split above (None: split
                                     # everywhere)


class _Cfg(dict):
    def __getattr__(self, k):
        try:
            return self[k]
        except KeyError as exc:
            raise AttributeError(k) from exc


class AlignmentStep:
    """get_sigma -> search_orientations -> tracker update -> search_shifts for one batch."""

    def __init__(self, cfg: StepConfig, device="cuda:0"):
        self.cfg = cfg
        self.device = torch.device(device)
        radius = cfg.radius if cfg.radius is not None else min(cfg.N // 2, int(cfg.N // 2 * 0.95))
        if cfg.precision not in ("bf16x3", "fp32", "auto"):
            raise ValueError("precision must be 'bf16x3', 'fp32' or 'auto'")
        self.correlator = CrossCorrelationMatcher(N=cfg.N, device=self.device, batchsize=cfg.batch,
                                                  bandlimit=cfg.L, radius=radius, precision_mode="fast",
                                                  precision="fp32" if cfg.precision == "fp32" else "bf16x3",
                                                  split_degree=None if cfg.precision == "fp32"
                                                  else cfg.expansion_split_degree)
        self.matcher = Matcha(batchsize=cfg.batch, device=self.device, L_max=cfg.L,
                              matcha_config=dict(Li=list(cfg.Li) + [cfg.L], candidates=cfg.candidates,
                                                 num_steps=cfg.num_steps, oversampling_factor_K=cfg.K))
        self.shifter = ShiftMatcher(_Cfg(N=cfg.N, voxel_size=cfg.voxel_size, num_subtomograms_per_batch=cfg.batch,
                                         shift_upsample_factor=cfg.shift_upsample_factor,
                                         shift_search_radius=cfg.shift_search_radius, do_ctf_correction=False,
                                         box_size=cfg.box_size if cfg.box_size is not None else cfg.N),
                                    self.device, torch.complex64, precision=cfg.precision,
                                    tile_rows=cfg.shift_tile_rows)
        B = cfg.batch
        self.rot = torch.empty((B, 9), device=self.device, dtype=torch.float32)
        self.shift = torch.empty((B, 3), device=self.device, dtype=torch.float32)
        self.shift_score = torch.empty((B,), device=self.device, dtype=torch.float32)

    def set_template(self, template: np.ndarray):
        self.correlator.set_template(template)
        self.shifter.set_reference(template)
        # upload the shift reference now so that steps issue no host work
        self.shifter._handle(self.cfg.batch)
        ref = self.shifter.reference_data_fourier.to(torch.complex64).contiguous()
        with torch.cuda.device(self.device):
            nat.check(self.shifter._lib.mtb_shift_set_reference(self.shifter._h, nat.ptr(ref),
                                                                nat.stream_ptr(self.device)), "mtb_shift_set_reference")
        self.shifter._ref_dev = ref
        self.shifter._uploaded_version = self.shifter._ref_version

    @torch.no_grad()
    def __call__(self, volumes: torch.Tensor, subtomos: torch.Tensor, tracker: torch.Tensor,
                 shift_zyx: torch.Tensor):
        """volumes: (B, N, N, N) input of the expansion; subtomos: (B, N, N, N) for the shift
        match; tracker: (B, 4) float64 (w, x, y, z), updated in place; shift_zyx (B, 3)."""
        B = volumes.shape[0]
        sigma, norms = self.correlator.get_sigma_upto(volumes, self.cfg.L)
        a, b, g, score = self.matcher.search_orientations(sigma)
        dev = self.device
        with torch.cuda.device(dev):
            nat.check(self.matcher._lib.mtb_update_rotation(nat.ptr(a), nat.ptr(b), nat.ptr(g), nat.ptr(tracker), B,
                                                            nat.ptr(tracker), nat.ptr(self.rot), nat.stream_ptr(dev)),
                      "mtb_update_rotation")
            nat.check(self.shifter._lib.mtb_shift_search(self.shifter._h, nat.ptr(subtomos), nat.ptr(shift_zyx),
                                                         nat.ptr(self.rot), None, B, nat.ptr(self.shift),
                                                         nat.ptr(self.shift_score), nat.stream_ptr(dev)),
                      "mtb_shift_search")
        return dict(alpha=a, beta=b, gamma=g, rotation_score=score, bh_norms=norms[:B], tracker=tracker,
                    shift=self.shift[:B], shift_score=self.shift_score[:B])

    @torch.no_grad()
    def prepare(self, subtomograms: torch.Tensor, current_shift: torch.Tensor, tracker: torch.Tensor):
        """``BatchProcessor._extract_rotated_batch`` (src/matcha/align_subtomograms.py:240-252):
        the patch of each (N, N, N) subtomogram at ``current_shift`` (B, 3), normalised in the
        spherical mask of radius ``radius`` and masked, rotated by its tracker (B, 4) float64.
        The first component of ``current_shift`` moves along the last (x) axis, as the
        reference's grid_sample reads it.  Returns a (B, N, N, N) buffer of this object,
        rewritten by the next call (``mtb_prepare_subtomos``, two launches)."""
        B, N = subtomograms.shape[0], self.cfg.N
        if B > self.cfg.batch:
            raise ValueError(f"batch {B} exceeds the configured batch {self.cfg.batch}")
        if subtomograms.shape[1:] != (N, N, N) or subtomograms.dtype != torch.float32:
            raise ValueError("subtomograms must be (B, N, N, N) float32")
        if getattr(self, "_prep", None) is None:
            Bc, dev = self.cfg.batch, self.device
            self._prep = dict(work=torch.empty((Bc, N, N, N, 2), device=dev, dtype=torch.float32),
                              out=torch.empty((Bc, N, N, N), device=dev, dtype=torch.float32),
                              stats=torch.empty((Bc, 2), device=dev, dtype=torch.float64))
        vols = subtomograms.contiguous()
        shift = current_shift.reshape(B, 3).to(torch.float32).contiguous()
        trk = tracker.contiguous()
        p = self._prep
        with torch.cuda.device(self.device):
            nat.check(nat.load().mtb_prepare_subtomos(nat.ptr(vols), B, N, nat.ptr(shift), nat.ptr(trk),
                                                      float(self.correlator.radius), nat.ptr(p["work"]),
                                                      nat.ptr(p["stats"]), nat.ptr(p["out"]),
                                                      nat.stream_ptr(self.device)), "mtb_prepare_subtomos")
        return p["out"][:B]

    @torch.no_grad()
    def run_alternations(self, subtomograms: torch.Tensor, tracker: torch.Tensor, local_shifts: torch.Tensor,
                         prior_shifts: torch.Tensor, base_shifts: torch.Tensor, num_alternations: int):
        """``BatchProcessor._run_alternations`` (src/matcha/align_subtomograms.py:316-361) for
        one batch on the device: each alternation prepares the subtomograms at the current
        shift and orientation, searches the rotation, matches the shift and adds it to
        ``local_shifts`` (B, 3), updated in place like ``tracker``.  Returns one dict of
        outputs per alternation (copies), with ``rotation_score`` also divided by the norms
        as the stored score is (align_subtomograms.py:300-302)."""
        results = []
        for _ in range(num_alternations):
            current = prior_shifts + base_shifts + local_shifts
            data = self.prepare(subtomograms, current, tracker)
            o = self(data, subtomograms, tracker, current)
            local_shifts += o["shift"]
            r = {k: v.clone() for k, v in o.items()}
            r["normalized_rotation_score"] = r["rotation_score"].reshape(-1) / (
                r["bh_norms"].reshape(-1) * self.correlator.bh_norm_template).clamp_min(1e-12)
            r["local_shifts"] = local_shifts.clone()
            results.append(r)
        return results

    @torch.no_grad()
    def capture(self, B: int, alternations: int = 0):
        """A CUDA graph of one batch of B subtomograms, replayed with ``CapturedStep.replay()``.

        alternations == 0: one alternation as ``__call__`` on prepared volumes (inputs
        ``volumes``, ``tracker``, ``shift``); alternations >= 1: ``run_alternations`` from the
        raw subtomograms (inputs ``volumes``, ``tracker``, ``local_shifts``, ``prior_shifts``,
        ``base_shifts``), each alternation preparing the batch first.  Inputs are static device
        tensors of the returned object: copy a batch into them, replay, read its outputs (also
        static, rewritten by each replay).  The step issues no host synchronisation, so every
        launch of the library and every torch operation of the loop is in the graph; the
        library's handles and the step's buffers are created by two eager runs first.

        The graph's outputs and intermediates are the step's own buffers (``shift``,
        ``shift_score``, the matcher's and correlator's result buffers, the preparation
        workspace): an eager call of this ``AlignmentStep``, or the replay of a second graph
        captured from it, rewrites them.  Keep one captured graph per step and read a replay's
        outputs before the next call.  ``set_template`` may be called between replays: the
        template's coefficients, norm and shift reference are updated in place, at the
        addresses the graph reads."""
        if not 0 < B <= self.cfg.batch:
            raise ValueError(f"batch must be in [1, {self.cfg.batch}]")
        return CapturedStep(self, B, alternations)

    _KEYS = ("alpha", "beta", "gamma", "rotation_score", "bh_norms", "shift", "shift_score")

    @torch.no_grad()
    def align_host(self, volumes_host: torch.Tensor, tracker: torch.Tensor, shift_zyx: torch.Tensor,
                   chunks: int = 4):
        """One alternation for a batch held in host memory (pinned for overlap).

        The batch is cut into ``chunks`` pieces: the host-to-device copy of piece k + 1 runs
        on a side stream while piece k is aligned on the current stream, so the transfer of
        the volumes (4 N^3 bytes each) and the alignment overlap.  Two device staging buffers
        alternate between calls, so the next call's first copies also overlap the end of this
        call's alignment.  tracker (B, 4) float64 and shift_zyx (B, 3) are device tensors;
        tracker is updated in place.  Returns the outputs of ``__call__`` for the whole batch,
        in tensors of their own (rewritten by the next call), and ``copies_done``, the CUDA
        event after which ``volumes_host`` is no longer read."""
        B = volumes_host.shape[0]
        if B > self.cfg.batch:
            raise ValueError(f"batch {B} exceeds the configured batch {self.cfg.batch}")
        dev = self.device
        N = self.cfg.N
        if getattr(self, "_stage", None) is None:
            self._stage = [torch.empty((self.cfg.batch, N, N, N), device=dev, dtype=torch.float32)
                           for _ in range(2)]
            self._stage_free = [None, None]  # compute-stream events after each buffer's last reader
            self._stage_next = 0
            self._copy_stream = torch.cuda.Stream(device=dev)
            self._out = {k: torch.empty((self.cfg.batch,) + ((3,) if k == "shift" else ()), device=dev,
                                        dtype=torch.float32) for k in self._KEYS}
        which = self._stage_next
        stage, cs = self._stage[which], self._copy_stream
        compute = torch.cuda.current_stream(dev)
        if self._stage_free[which] is not None:
            cs.wait_event(self._stage_free[which])  # the alignment that read this buffer is done
        bounds = [B * k // chunks for k in range(chunks + 1)]
        ready = []
        with torch.cuda.stream(cs):
            for k in range(chunks):
                lo, hi = bounds[k], bounds[k + 1]
                if hi > lo:
                    stage[lo:hi].copy_(volumes_host[lo:hi], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(cs)
                ready.append(ev)
        for k in range(chunks):
            lo, hi = bounds[k], bounds[k + 1]
            compute.wait_event(ready[k])
            if hi == lo:
                continue
            vols = stage[lo:hi]
            o = self(vols, vols, tracker[lo:hi], shift_zyx[lo:hi])
            for key in self._KEYS:
                self._out[key][lo:hi].copy_(o[key])
        free = torch.cuda.Event()
        free.record(compute)
        self._stage_free[which] = free
        self._stage_next = which ^ 1
        out = {k: self._out[k][:B] for k in self._KEYS}
        out["tracker"] = tracker
        out["copies_done"] = ready[-1]  # after it the host batch may be overwritten
        return out


class CapturedStep:
    """See ``AlignmentStep.capture``."""

    def __init__(self, step: AlignmentStep, B: int, alternations: int):
        N, dev = step.cfg.N, step.device
        self.step, self.B, self.alternations = step, B, alternations
        self.volumes = torch.zeros((B, N, N, N), device=dev, dtype=torch.float32)
        self.tracker = torch.zeros((B, 4), device=dev, dtype=torch.float64)
        self.tracker[:, 0] = 1
        self._tracker0 = self.tracker.clone()
        z = lambda: torch.zeros((B, 3), device=dev, dtype=torch.float32)
        if alternations == 0:
            self.shift = z()
        else:
            self.local_shifts, self.prior_shifts, self.base_shifts = z(), z(), z()
            self._local0 = z()
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.device(dev), torch.cuda.stream(side):
            for _ in range(2):
                self._restore()
                self._run()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self._restore()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.device(dev), torch.cuda.graph(self.graph):
            self.outputs = self._run()
        torch.cuda.synchronize(dev)

    def _restore(self):
        self.tracker.copy_(self._tracker0)
        if self.alternations:
            self.local_shifts.copy_(self._local0)

    def _run(self):
        s = self.step
        if self.alternations == 0:
            return s(self.volumes, self.volumes, self.tracker, self.shift)
        return s.run_alternations(self.volumes, self.tracker, self.local_shifts, self.prior_shifts,
                                  self.base_shifts, self.alternations)

    def replay(self):
        """Run the captured batch on the current inputs; returns the static outputs (a dict, or
        a list of dicts, one per alternation).  tracker (and local_shifts) are updated in place
        as the eager calls update them."""
        self.graph.replay()
        return self.outputs