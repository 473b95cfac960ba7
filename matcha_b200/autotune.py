"""Batch capacity and kernel tile choice per box size, measured on the device.

The reference sizes its batches by probing: a child process allocates its pipeline at growing
batch sizes until CUDA runs out of memory (``_probe_batch_size_impl``,
src/matcha/utils/run_utils.py:184-355, :817-868), so that a failure cannot poison the parent.
Here nothing runs out of memory on purpose:

* ``plan_capacity`` builds an ``AlignmentStep`` at two small capacities, runs one alternation
  on each and reads the device memory each one holds (``torch.cuda.mem_get_info``, which sees
  the library's own allocations as well as torch's); the step's memory is affine in its
  capacity, so the largest capacity under a budget follows from the two points.
* ``tune_step`` times the candidate tile shapes of the kernels that have one (the rows per CTA
  of the FP32 upsampled DFT's passes 2+3, which boxes without tensor-core shift kernels use) on
  a synthetic batch with CUDA events and keeps the fastest; the choice changes no result.

``matcha_b200.mixed.MixedAlignment`` uses ``tune_step`` for each box size of an uneven batch.
"""
from __future__ import annotations

from dataclasses import dataclass, replace

import numpy as np
import torch

from .pipeline import AlignmentStep, StepConfig


@dataclass
class CapacityPlan:
    bytes_fixed: int          # memory of a step independent of its capacity (tables, basis)
    bytes_per_subtomo: int    # memory per subtomogram of capacity, the batch's volumes included
    capacity: int             # the largest capacity within the budget


def _synthetic(cfg: StepConfig, B: int, device, seed=0):
    rng = np.random.default_rng(seed)
    N = cfg.N
    g = np.arange(N) - N // 2
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    tmpl = np.zeros((N, N, N))
    for _ in range(24):
        c = rng.uniform(-0.25 * N, 0.25 * N, 3)
        tmpl += np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * (0.04 * N) ** 2))
    tmpl = tmpl.astype(np.float32)
    gen = torch.Generator(device=device).manual_seed(seed)
    vols = torch.from_numpy(tmpl).to(device)[None] + 0.5 * torch.randn((B, N, N, N), device=device, generator=gen)
    return tmpl, vols


def _run_once(step: AlignmentStep, vols):
    B = vols.shape[0]
    tracker = torch.zeros((B, 4), dtype=torch.float64, device=vols.device)
    tracker[:, 0] = 1
    return step(vols, vols, tracker, torch.zeros((B, 3), device=vols.device))


def step_bytes(cfg: StepConfig, capacity: int, device) -> int:
    """Device memory a step of ``cfg`` at ``capacity`` holds after one alternation and one
    preparation (its input batch excluded)."""
    device = torch.device(device)
    tmpl, vols = _synthetic(cfg, capacity, device)
    torch.cuda.synchronize(device)
    torch.cuda.empty_cache()
    free0 = torch.cuda.mem_get_info(device)[0]
    step = AlignmentStep(replace(cfg, batch=capacity), device)
    step.set_template(tmpl)
    _run_once(step, vols)
    step.prepare(vols, torch.zeros((capacity, 3), device=device),
                 torch.tensor([[1.0, 0, 0, 0]] * capacity, dtype=torch.float64, device=device))
    torch.cuda.synchronize(device)
    free1 = torch.cuda.mem_get_info(device)[0]
    del step
    torch.cuda.synchronize(device)
    torch.cuda.empty_cache()
    return free0 - free1


def plan_capacity(cfg: StepConfig, device, budget_bytes: int = None, probe=(128, 384),
                  margin: float = 1.1) -> CapacityPlan:
    """The largest batch capacity of a step of ``cfg`` whose memory, with its batch of input
    volumes, fits ``budget_bytes`` (default: 85 % of the device memory free now).  The probe
    capacities are multiples of 128, the row tile the expansion pads its batch to, so the two
    measurements see the same padding; ``margin`` covers the allocator's rounding."""
    device = torch.device(device)
    if budget_bytes is None:
        budget_bytes = int(0.85 * torch.cuda.mem_get_info(device)[0])
    c1, c2 = probe
    m1, m2 = step_bytes(cfg, c1, device), step_bytes(cfg, c2, device)
    per_step = max(0, int(np.ceil(margin * (m2 - m1) / (c2 - c1))))
    fixed = max(0, m1 - per_step * c1)
    per = per_step + 4 * cfg.N ** 3  # + the batch's input volumes
    cap = int(max(0, budget_bytes - fixed) // per)
    return CapacityPlan(bytes_fixed=int(fixed), bytes_per_subtomo=int(per), capacity=cap)


def tune_step(cfg: StepConfig, device, batch: int = 128, candidates=(1, 2, 4, 8), reps: int = 3):
    """Time the FP32 upsampled DFT's tile candidates for a step of ``cfg`` (when its shift
    match runs the FP32 kernels) and return (cfg with the fastest tile, {tile: ms per step});
    a step whose shift match runs on the tensor cores has nothing to tune ({})."""
    device = torch.device(device)
    timings = {}
    tmpl, vols = _synthetic(cfg, batch, device, seed=1)
    for rows in candidates:
        step = AlignmentStep(replace(cfg, batch=batch, shift_tile_rows=rows), device)
        step.set_template(tmpl)
        if step.shifter.effective_precision != "fp32":
            return replace(cfg, shift_tile_rows=0), {}
        _run_once(step, vols)
        st = torch.cuda.current_stream(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(st)
        for _ in range(reps):
            _run_once(step, vols)
        e1.record(st)
        torch.cuda.synchronize(device)
        timings[rows] = e0.elapsed_time(e1) / reps
        del step
    best = min(timings, key=timings.get)
    return replace(cfg, shift_tile_rows=best), timings
