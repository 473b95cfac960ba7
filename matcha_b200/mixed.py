"""Alignment of a batch whose subtomograms have different box sizes (and bandlimits).

The reference aligns one box size per run: its batches come from one STAR file and one
template (src/matcha/align_subtomograms.py:316-361).  An uneven workload - boxes 48, 64 and 96
with bandlimits 24, 32 and 48, each from its own template - is here one ``MixedAlignment``:
one ``AlignmentStep`` per box size, its kernel tiles chosen by ``matcha_b200.autotune``, all
run on one stream.  ``capture`` records the steps of every box size back to back into one
CUDA graph, so a whole mixed batch is one replay with no host work between the box sizes.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np
import torch

from . import autotune
from .pipeline import AlignmentStep, StepConfig


@dataclass
class BoxSpec:
    """One box size of the mixed batch: its step configuration (N, L, Li, shift settings;
    ``batch`` is the capacity) and its template (N, N, N) float32.  ``timings`` is filled
    by the tuner ({tile rows: ms per step})."""
    cfg: StepConfig
    template: np.ndarray
    timings: dict = field(default_factory=dict)


class MixedAlignment:
    def __init__(self, boxes: list, device="cuda:0", tune: bool = True):
        self.device = torch.device(device)
        self.boxes = {}
        for spec in boxes:
            N = spec.cfg.N
            if N in self.boxes:
                raise ValueError(f"box size {N} given twice")
            cfg, timings = spec.cfg, {}
            if tune:
                cfg, timings = autotune.tune_step(cfg, self.device, batch=min(cfg.batch, 128))
            step = AlignmentStep(cfg, self.device)
            step.set_template(spec.template)
            self.boxes[N] = (replace(spec, cfg=cfg, timings=timings), step)

    @torch.no_grad()
    def __call__(self, batches: dict):
        """batches: {N: (volumes (B_N, N, N, N) float32, tracker (B_N, 4) float64,
        shift_zyx (B_N, 3) float32)} on the device, trackers updated in place.  One
        alternation per box size on the current stream; returns {N: outputs of that step}."""
        out = {}
        for N, (vols, tracker, shift) in batches.items():
            out[N] = self.boxes[N][1](vols, vols, tracker, shift)
        return out

    @torch.no_grad()
    def capture(self, counts: dict):
        """One CUDA graph of one alternation for counts {N: B_N} subtomograms of each box size
        (``MixedCapturedStep``)."""
        return MixedCapturedStep(self, counts)


class MixedCapturedStep:
    """Static inputs ``volumes[N]``, ``tracker[N]``, ``shift[N]`` per box size; ``replay()``
    runs every box size's alternation in one graph launch and returns the static outputs
    (the steps' own buffers, rewritten by the next replay or eager call)."""

    def __init__(self, mixed: MixedAlignment, counts: dict):
        dev = mixed.device
        self.mixed = mixed
        self.volumes, self.tracker, self.shift = {}, {}, {}
        for N, B in counts.items():
            step = mixed.boxes[N][1]
            if not 0 < B <= step.cfg.batch:
                raise ValueError(f"box {N}: batch must be in [1, {step.cfg.batch}]")
            self.volumes[N] = torch.zeros((B, N, N, N), device=dev, dtype=torch.float32)
            self.tracker[N] = torch.zeros((B, 4), device=dev, dtype=torch.float64)
            self.tracker[N][:, 0] = 1
            self.shift[N] = torch.zeros((B, 3), device=dev, dtype=torch.float32)
        self._tracker0 = {N: t.clone() for N, t in self.tracker.items()}
        side = torch.cuda.Stream(device=dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.device(dev), torch.cuda.stream(side):
            for _ in range(2):
                self.restore()
                self._run()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        self.restore()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.device(dev), torch.cuda.graph(self.graph):
            self.outputs = self._run()
        torch.cuda.synchronize(dev)

    def restore(self):
        """Reset the trackers to the identity (each replay updates them in place)."""
        for N, t in self.tracker.items():
            t.copy_(self._tracker0[N])

    def _run(self):
        return self.mixed({N: (self.volumes[N], self.tracker[N], self.shift[N]) for N in self.volumes})

    def replay(self):
        self.graph.replay()
        return self.outputs
