#!/usr/bin/env python
"""Throughput of one alignment alternation: subtomograms/s at 64^3, L=32 on B200.

Workload (the plain-method benchmark shape): a 64^3 float32 template made of 400
Gaussian blobs (sigma U[1, 2.5] voxels) in two lobes of radius 26 and 18 voxels,
soft-masked; 1000 subtomograms, each the template rotated by a Haar-uniform rotation
(trilinear resampling in the reference's convention), shifted by a uniform offset in
[-5, 5]^3 voxels (Fourier phase ramp) and given white Gaussian noise at 0 dB SNR inside
the mask.  One step is one alternation over the whole batch: ball expansion and
correlation coefficients (L = 32), SO(3) grid search and Newton march over
L = 8, 16, 24, 32 with 10 candidates and one Newton step, rotation-tracker update and
the FFT shift match (search radius 5, upsample factor 8).  Synthetic data; inputs are
generated on the device before the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank aligns its own batch (no collective on the data path); the
step time is the maximum over ranks.  ``--impl reference`` times the CPU restatement of
the reference's algorithm (the oracle) on the host cores, on a bounded sample per step.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BOX, L_MAX, LI = 64, 32, [8, 16, 24]
SHIFT_RADIUS, UPSAMPLE = 5, 8
METRIC = "subtomograms/s at 64^3 L=32 (one alternation: FLE+sigma, SO(3) grid, Newton march, shift)"
KERNELS_PER_STEP = 16  # FLE fold_split, gemm_tc, expand; sigma; SO(3) grid; fold_sigma, newton_march,
# reduce_candidates; tracker_update; shift patch_fft_xy64, fft_z64, updft1_tc x2 (the Nyquist plane),
# updft1_tc, updft23_tc, finalize_tc


def parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=1000)
    p.add_argument("--cpu-sample", type=int, default=8,
                   help="subtomograms per CPU-baseline step (also the accuracy comparison with the oracle)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp32", action="store_true", help="skip the plain-FP32 comparison run")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--mixed", action="store_true",
                   help="uneven boxes instead of the metric's shape: 4096 subtomograms drawn from boxes 48, 64, 96 "
                        "(L 24, 32, 48; own templates of 150, 400, 900 blobs), shifts in +-6, SNR U[-10, 5] dB, one "
                        "captured graph per alternation (a reported extra, not the metric)")
    p.add_argument("--split-degree", type=int, default=None,
                   help="--highband: also run the expansion in plain BF16 up to this degree with the hi+lo split "
                        "above (default 40, the shape's own schedule) and report it beside the split everywhere")
    p.add_argument("--highband", action="store_true",
                   help="the high-bandlimit shape instead of the metric's: 128^3, L=64, march 16/32/48/64, "
                        "shift r=8, -5 dB (a reported extra, not the metric; --batch defaults to 512; --cpu-sample "
                        "subtomograms, default 8, checked against the FP64 oracle)")
    return p.parse_args()


# ---------------------------------------------------------------- synthetic data (numpy, host)
def make_template(rng, N=N_BOX, n_blobs=400, window=None):
    """Gaussian blobs in two lobes (radii 26 and 18 voxels; scaled with the box below 64^3)
    under a soft spherical mask; window (voxels) evaluates each blob only within that distance
    of its centre per axis (for large boxes)."""
    g = np.arange(N) - N // 2
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    vol = np.zeros((N, N, N))
    sc = N / 64.0 if N < 64 else 1.0
    lobes = [(26.0 * sc, np.array([-3.0, 1.0, 0.0]) * sc), (18.0 * sc, np.array([6.0, -4.0, 3.0]) * sc)]
    for i in range(n_blobs):
        r_l, off = lobes[i % 2]
        d = rng.standard_normal(3)
        c = off + d / np.linalg.norm(d) * r_l * rng.uniform() ** (1 / 3)
        s = rng.uniform(1.0, 2.5)
        a = rng.uniform(0.5, 1.0)
        if window is None:
            vol += a * np.exp(-((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2) / (2 * s * s))
        else:
            lo = np.clip(np.floor(c + N // 2 - window).astype(int), 0, N)
            hi = np.clip(np.ceil(c + N // 2 + window).astype(int) + 1, 0, N)
            sl = tuple(slice(lo[k], hi[k]) for k in range(3))
            vol[sl] += a * np.exp(-((z[sl] - c[0]) ** 2 + (y[sl] - c[1]) ** 2 + (x[sl] - c[2]) ** 2) / (2 * s * s))
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    vol *= np.clip((0.45 * N + 2 - r) / 4, 0, 1)
    return vol.astype(np.float32)


def make_batch(template, rng, B, device, snr_db=0.0, max_shift=5.0, count=None):
    """Rotated (reference rotate_volumes convention), shifted, noisy subtomograms on ``device``.

    Every random parameter of all B subtomograms is drawn first (Haar quaternions, uniform
    shifts in voxels (z, y, x), one noise seed per subtomogram), then the first ``count``
    (default B) volumes are synthesised, so the CPU arm can rebuild exactly the first few
    subtomograms of the GPU arm's batch.  Noise: white Gaussian at ``snr_db`` against the
    signal power inside the sphere of radius 0.45 N (src/matcha/example.py:93-124)."""
    import torch
    import torch.nn.functional as TF
    from scipy.spatial.transform import Rotation as R

    N = template.shape[0]
    q = rng.standard_normal((B, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    shifts = rng.uniform(-max_shift, max_shift, (B, 3)).astype(np.float32)
    seeds = rng.integers(0, 1 << 62, B)
    n = B if count is None else min(int(count), B)
    mats = torch.tensor(R.from_quat(np.roll(q[:n], -1, axis=1)).as_matrix(), dtype=torch.float32, device=device)
    t = torch.from_numpy(template).to(device)
    tp = TF.pad(t[None, None], (0, 1, 0, 1, 0, 1))
    lin = torch.linspace(-1, 1, N + 1, device=device)
    wg, hg, dg = torch.meshgrid(lin, lin, lin, indexing="ij")
    coords = torch.stack([dg.flatten(), hg.flatten(), wg.flatten()], 0)
    k = torch.fft.fftfreq(N, device=device)
    kz, ky, kx = torch.meshgrid(k, k, k, indexing="ij")
    g = torch.arange(N, device=device) - N // 2
    zz, yy, xx = torch.meshgrid(g, g, g, indexing="ij")
    mask = (torch.sqrt((xx ** 2 + yy ** 2 + zz ** 2).float()) < 0.45 * N)
    out = torch.empty((n, N, N, N), device=device, dtype=torch.float32)
    sh = torch.from_numpy(shifts[:n]).to(device)
    for s in range(0, n, 50):
        e = min(n, s + 50)
        rc = (mats[s:e] @ coords).permute(0, 2, 1).reshape(e - s, N + 1, N + 1, N + 1, 3)
        v = TF.grid_sample(tp.expand(e - s, -1, -1, -1, -1), rc, mode="bilinear", align_corners=True)
        v = v[:, 0, :N, :N, :N]
        ph = torch.exp(-2j * np.pi * (kz[None] * sh[s:e, 0, None, None, None] + ky[None] * sh[s:e, 1, None, None, None]
                                      + kx[None] * sh[s:e, 2, None, None, None]))
        v = torch.fft.ifftn(torch.fft.fftn(v, dim=(1, 2, 3)) * ph, dim=(1, 2, 3)).real
        power = (v[:, mask] ** 2).mean(dim=1)
        noise = np.stack([np.random.default_rng(int(seeds[i])).standard_normal((N, N, N), dtype=np.float32)
                          for i in range(s, e)])
        snr = torch.as_tensor(np.broadcast_to(np.asarray(snr_db, dtype=np.float64), (n,))[s:e].copy(), device=device)
        out[s:e] = v + torch.from_numpy(noise).to(device) * torch.sqrt(power * 10.0 ** (-snr / 10.0)).to(
            torch.float32)[:, None, None, None]
    return out, q, shifts


def rotation_error_deg(alpha, beta, gamma, q_true):
    """Tracker angle after update_rotation_estimate from the true rotation (example.py:208-220)."""
    from scipy.spatial.transform import Rotation as R

    est = R.from_euler("ZYZ", np.stack([alpha, beta, gamma], -1)).as_quat()
    qw = np.roll(est, 1, axis=1)
    qw[:, [1, 3]] = qw[:, [3, 1]]
    sw = R.from_quat(np.roll(qw, -1, axis=1))
    tr = R.from_quat(np.roll(q_true, -1, axis=1))
    return np.rad2deg((tr * sw.inv()).magnitude())


def tracker_error_deg(tracker, q_true):
    """Angle between the true rotation and a tracker (w, x, y, z) after any number of
    alternations: rotation_error_deg's tr * sw^-1 with sw^-1 the tracker's rotation (from the
    identity one update gives tracker = conj(sw))."""
    from scipy.spatial.transform import Rotation as R

    t = R.from_quat(np.roll(np.asarray(tracker, dtype=np.float64), -1, axis=1))
    tr = R.from_quat(np.roll(q_true, -1, axis=1))
    return np.rad2deg((tr * t).magnitude())


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"mtb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def wait_first(self, busy, limit_s=5.0):
        """Keep the GPU busy (busy() runs one untimed step) until the sampler has written
        its first row, so that every row of the timed region is taken under load."""
        import torch

        t0 = time.time()
        while self.proc is not None and time.time() - t0 < limit_s:
            busy()
            torch.cuda.synchronize()
            if os.path.exists(self.path) and os.path.getsize(self.path) > 0:
                break

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- CPU restatement (oracle)
_ORACLE_SETUP = {}  # per template: the oracle's folded basis, template coefficients, shift reference


def cpu_align(sample, template, vols, dtype=np.float32):
    """The oracle's alternation (FP64 expansion; orientation search in ``dtype``: float32 is the
    reference's arithmetic, float64 the exact answer) on the first ``sample`` volumes; returns
    (seconds per subtomogram of the alignment itself, outputs)."""
    from matcha_b200.core import fle_tables as T
    from oracle import pipeline as OP
    from oracle import shift as OS

    key = id(template)
    if key not in _ORACLE_SETUP:
        radius = min(N_BOX // 2, int(N_BOX // 2 * 0.95))
        tb = T.lap_eig_ball(N_BOX, L_MAX, radius)
        ff = OP.FoldedFLE(tb, N_BOX, float(radius))
        _ORACLE_SETUP[key] = (ff, ff.evaluate_t(template[None])[0], OS.load_reference_full(template, N_BOX, 1.0))
    ff, a_t, ref = _ORACLE_SETUP[key]
    v = np.asarray(vols[:sample], dtype=np.float64)
    tracker = np.tile([1.0, 0, 0, 0], (sample, 1))
    t0 = time.perf_counter()
    out = OP.align_batch(ff, a_t, ref, v, v, tracker, np.zeros((sample, 3)), L_MAX, LI, uf=UPSAMPLE,
                         shift_radius=SHIFT_RADIUS, dtype=dtype)
    dt = time.perf_counter() - t0
    return dt / sample, out


def euler_dev_deg(a1, b1, g1, a2, b2, g2):
    from scipy.spatial.transform import Rotation as R

    r1 = R.from_euler("ZYZ", np.stack([a1, b1, g1], -1).astype(np.float64))
    r2 = R.from_euler("ZYZ", np.stack([a2, b2, g2], -1).astype(np.float64))
    return np.rad2deg((r1.inv() * r2).magnitude())


def accuracy_vs_oracle(gpu, o32, o64, q_true, n):
    """Per-subtomogram rotation deviation of a GPU run from the oracle on the same n inputs."""
    ang = lambda d: [np.asarray(d[k][:n], dtype=np.float64) for k in ("alpha", "beta", "gamma")]
    d32 = euler_dev_deg(*ang(gpu), *ang(o32))
    d64 = euler_dev_deg(*ang(gpu), *ang(o64))
    err = rotation_error_deg(*ang(gpu), q_true[:n])
    return {"median_rot_err_deg": float(np.median(err)),
            "median_dev_vs_ref_deg": float(np.median(d32)), "max_dev_vs_ref_deg": float(d32.max()),
            "frac_within_0p05deg": float(np.mean(d32 < 0.05)),
            "median_dev_vs_fp64_deg": float(np.median(d64)), "max_dev_vs_fp64_deg": float(d64.max()),
            "frac_within_0p05deg_of_fp64": float(np.mean(d64 < 0.05)),
            "shift_equal_frac": float(np.mean(np.all(np.abs(np.asarray(gpu["shift"][:n]) - o64["shift"]) < 1e-6,
                                                     axis=1)))}


# ---------------------------------------------------------------- roofline of every kernel of the step
def kernel_work(B):
    """Algorithmic work of each kernel of one alternation at 64^3, L = 32 (ne = 8252 coefficients,
    8252 real basis columns, 15 216 octant representatives of the radius-30 ball, U = 88): FLOP
    counted once per multiply-add pair of the exact product (a hi+lo split issues 3x as many),
    bytes the compulsory HBM traffic of inputs and outputs.  Returns {kernel: (bound, amount)}
    per launch of B subtomograms, amount in bytes for "hbm" and FLOP for "tensor"/"fp32"."""
    N, H, U = N_BOX, N_BOX // 2 + 1, int(np.ceil(UPSAMPLE * (2 * SHIFT_RADIUS + 1)))
    n_rep, n_cols, ne = 15216, 8252, 8252
    vol = 4 * N ** 3                     # one float32 subtomogram
    spec = 8 * N * N * H                 # (N, N, N/2+1) complex64 plane transforms
    a1 = 2 * 2 * (N // 2) * N * 2 * N    # pass-1 operand: rows (m2 < N/2, m1), K (m0, re/im), bf16 hi and lo
    a1n = 2 * 2 * N * 2 * N              # the Nyquist plane's pass-1 operand
    a2 = 2 * 2 * U * (N // 2) * 2 * N    # pass-2 operand: rows (u0, m2 < N/2), K (m1, re/im), hi and lo
    dsize = lambda L: (L + 1) * (2 * L + 1) * (2 * L + 3) // 3
    work = {
        "fold_split_kernel": ("hbm", vol + 2 * 2 * 8 * n_rep),
        "gemm_tc_kernel": ("tensor", 2.0 * n_rep * n_cols),
        "expand_kernel": ("hbm", 4 * n_cols + 8 * ne),
        "sigma_kernel": ("hbm", 8 * ne + 8 * dsize(L_MAX)),
        "so3_grid_topk_kernel": ("hbm", 8 * dsize(8)),
        "fold_sigma_kernel": ("hbm", 8 * dsize(L_MAX) + 16 * sum((l + 1) ** 2 for l in range(L_MAX + 1))),
        "tracker_update_kernel": ("hbm", 3 * 4 + 2 * 32 + 36),
        "patch_fft_xy64_kernel": ("hbm", vol + spec),
        "fft_z64_kernel": ("hbm", spec + a1 + a1n),
        "updft1_tc_kernel": ("tensor", 2.0 * (N // 2 * N) * (2 * N) * (2 * U)),
        # the Nyquist plane m2 = N/2 as its own two small GEMMs: rows (b, m1), then rows (b, u0)
        "updft1_tc_kernel (Nyquist plane, pass 1)": ("tensor", 2.0 * N * (2 * N) * (2 * U)),
        "updft1_tc_kernel (Nyquist plane, pass 2)": ("tensor", 2.0 * U * (2 * N) * (2 * U)),
        "updft23_tc_kernel": ("tensor", 2.0 * (U * N // 2) * (2 * U) * (2 * N) + 2.0 * U * U * U * (N + 2)),
        "finalize_tc_kernel": ("hbm", 16),
    }
    # newton_march_kernel has no entry: its folded wedge chains do far less arithmetic than the
    # reference's 15-column bank contraction, and ncu shows it bound by issue and L2 latency
    # (profiles/search_L32_b296.md), not by a pipe's throughput
    return {k: (b, a * B) for k, (b, a) in work.items()}, {"a2_bytes": a2}


def fp32_peak_tflops(dev):
    """FP32 CUDA-core throughput: cuBLAS SGEMM 8192^3 with TF32 off, best of 5 (CUDA events)."""
    import torch

    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        a = torch.randn(8192, 8192, device=dev)
        b = torch.randn(8192, 8192, device=dev)
        c = a @ b
        best = None
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            c = a @ b
            e1.record()
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1)
            best = t if best is None else min(best, t)
        del a, b, c
        return 2.0 * 8192 ** 3 / (best * 1e-3) / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def kernel_table(prof, steps, B, peaks, fp32_peak):
    """Per kernel: ms per step, share of the step's kernel time, and roofline against the
    measured peaks (HBM copy bandwidth, sustained bf16 tensor throughput, cuBLAS SGEMM)."""
    work, _ = kernel_work(B)
    total = sum(v["ms"] for v in prof.values())
    table = {}
    for name, v in prof.items():
        ms = v["ms"] / steps
        row = {"ms_per_step": ms, "launches_per_step": v["launches"] / steps, "share": v["ms"] / total if total else None}
        base = name if name in work else name.split(" (")[0]
        if base in work and v["launches"] / steps == 1:
            bound, amount = work[base]
            if bound == "hbm":
                ach, peak, unit = amount / (ms * 1e-3) / 1e9, float(peaks.get("hbm_gbs", 6535.4)), "GB/s"
            elif bound == "tensor":
                ach, peak, unit = amount / (ms * 1e-3) / 1e12, float(peaks.get("bf16_tflops_sustained", 1401.9)), "TFLOP/s"
            else:
                ach, peak, unit = amount / (ms * 1e-3) / 1e12, fp32_peak, "TFLOP/s"
            row.update(bound=bound, achieved=ach, peak=peak, unit=unit, frac=ach / peak if peak else None)
            if DRAM_BYTES_PER_SUBTOMO.get(name):
                row["traffic"] = DRAM_BYTES_PER_SUBTOMO[name] * B
        table[name] = row
    return table, total / steps


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per subtomogram of the shift kernels,
# from one ncu capture at 200 subtomograms (profiles/shift_64_uf8_b200.md), scaled to a launch by
# the subtomograms it processes (their traffic grows in proportion to the batch)
DRAM_BYTES_PER_SUBTOMO = {"patch_fft_xy64_kernel": 1_910_000, "fft_z64_kernel": 2_085_000,
                          "updft1_tc_kernel": 2_205_000, "updft23_tc_kernel": 1_525_000}


# ---------------------------------------------------------------- ranks
def dist_env():
    """(world size, rank, local rank) from the launcher's environment (one process per GPU)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest of the ranks' values: a replica job's step time is its slowest rank's (an
    all_reduce of the timing only; the ranks exchange no data).  The identity on one rank."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(world: int, batch: int, ms: float) -> float:
    """Subtomograms per second of the whole job: every rank aligns its own batch of ``batch``
    in the max-over-ranks step time ``ms`` (weak scaling)."""
    return world * batch / (ms * 1e-3)


# ---------------------------------------------------------------- our implementation
def run_ours(args):
    import torch
    import torch.distributed as dist

    world, rank, local = dist_env()
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    from matcha_b200 import _native as nat
    from matcha_b200.pipeline import AlignmentStep, StepConfig

    rng = np.random.default_rng(args.seed)
    template = make_template(rng)
    B = args.batch
    vols, q_true, shifts = make_batch(template, np.random.default_rng(args.seed + 1 + rank), B, dev)
    step = AlignmentStep(StepConfig(N=N_BOX, L=L_MAX, Li=LI, batch=B, shift_search_radius=SHIFT_RADIUS,
                                    shift_upsample_factor=UPSAMPLE, precision="bf16x3"), dev)
    step.set_template(template)
    ident = torch.zeros((B, 4), device=dev, dtype=torch.float64)
    ident[:, 0] = 1
    tracker = ident.clone()
    zeros3 = torch.zeros((B, 3), device=dev, dtype=torch.float32)

    def one():
        tracker.copy_(ident)
        return step(vols, vols, tracker, zeros3)

    for _ in range(args.warmup):
        out = one()
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    # timed region: every launch of the library bracketed by CUDA events on its stream
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        clk.wait_first(one)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        nat.profile_start(args.steps * (KERNELS_PER_STEP + 4))
        torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches
        start.record(st)
        for _ in range(args.steps):
            out = one()
        end.record(st)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
        nat.profile_stop()
    ms = start.elapsed_time(end) / args.steps
    prof, dropped = nat.profile_read()
    launches = sum(v["launches"] for v in prof.values())
    ms = max_over_ranks(ms, world, dev)
    if world > 1:
        dist.barrier()
    # end-to-end through the public API with host buffers
    # (AlignmentStep.align_host: the volumes' host-to-device copy overlaps the alignment in
    # four pieces; the results come back to pinned host memory every step)
    host = vols.cpu().pin_memory()
    res_host = torch.empty((B, 8), dtype=torch.float32).pin_memory()
    res_dev = torch.empty((B, 8), device=dev, dtype=torch.float32)
    e2e_start, e2e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def e2e_step():
        tracker.copy_(ident)
        o = step.align_host(host, tracker, zeros3, chunks=4)
        res_dev[:, 0], res_dev[:, 1], res_dev[:, 2], res_dev[:, 3] = o["alpha"], o["beta"], o["gamma"], o["rotation_score"]
        res_dev[:, 4:7] = o["shift"]
        res_dev[:, 7] = o["shift_score"]
        res_host.copy_(res_dev, non_blocking=True)

    e2e_step()  # untimed: allocates the staging buffer
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, 5))
    e2e_start.record(st)
    for _ in range(e2e_steps):
        e2e_step()
    e2e_end.record(st)
    torch.cuda.synchronize()
    e2e_ms = e2e_start.elapsed_time(e2e_end) / e2e_steps
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    # accuracy of the chosen path on the full batch (one more step; the end-to-end runs' pieces
    # overwrote the step's output buffers), kept for the comparison with the oracle below
    out = one()
    chosen = {k: out[k].cpu().numpy() for k in ("alpha", "beta", "gamma", "shift")}
    # the same step with the plain FP32 kernels (the expansion GEMM and the upsampled DFT on
    # CUDA cores instead of the BF16 hi+lo tensor-core split): the comparison the metric names
    plain = None
    plain_out = None
    if not args.no_fp32:
        step32 = AlignmentStep(StepConfig(N=N_BOX, L=L_MAX, Li=LI, batch=B, shift_search_radius=SHIFT_RADIUS,
                                          shift_upsample_factor=UPSAMPLE, precision="fp32"), dev)
        step32.set_template(template)
        for _ in range(2):
            tracker.copy_(ident)
            step32(vols, vols, tracker, zeros3)
        n32 = max(3, args.steps // 4)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        nat.profile_start(n32 * (KERNELS_PER_STEP + 4))
        e32s, e32e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e32s.record(st)
        for _ in range(n32):
            tracker.copy_(ident)
            o32 = step32(vols, vols, tracker, zeros3)
        e32e.record(st)
        torch.cuda.synchronize()
        nat.profile_stop()
        prof32, _ = nat.profile_read()
        ms32 = e32s.elapsed_time(e32e) / n32
        plain_out = {k: o32[k].cpu().numpy() for k in ("alpha", "beta", "gamma", "shift")}
        ms32 = max_over_ranks(ms32, world, dev)
        plain = {"value": whole_job_value(world, B, ms32), "ms_per_step": ms32, "steps": n32,
                 "chosen_speedup": ms32 / ms, "kernels_ms_per_step": {k: v["ms"] / n32 for k, v in prof32.items()}}
        del step32
    # three alternations per batch, as an alignment run makes them: each prepares the batch at
    # the current shift and orientation (patch, masked normalisation, rotation), then sigma,
    # search, tracker update and shift match (AlignmentStep.run_alternations)
    local3 = torch.zeros((B, 3), device=dev, dtype=torch.float32)

    def three():
        tracker.copy_(ident)
        local3.zero_()
        return step.run_alternations(vols, tracker, local3, zeros3, zeros3, 3)

    three()
    torch.cuda.synchronize()
    n3 = max(2, args.steps // 4)
    if world > 1:
        dist.barrier()
    e3s, e3e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e3s.record(st)
    for _ in range(n3):
        three()
    e3e.record(st)
    torch.cuda.synchronize()
    ms3 = e3s.elapsed_time(e3e) / n3
    ep0, ep1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ep0.record(st)
    for _ in range(5):
        step.prepare(vols, zeros3, tracker)
    ep1.record(st)
    torch.cuda.synchronize()
    ms_prep = max_over_ranks(ep0.elapsed_time(ep1) / 5, world, dev)
    ms3 = max_over_ranks(ms3, world, dev)
    # rotation error of the tracker after the third alternation (the last run's)
    trk = tracker.cpu().numpy()
    err3 = tracker_error_deg(trk, q_true)
    alternations = {"value": whole_job_value(world, B, ms3), "unit": "subtomograms/s", "alternations": 3,
                    "ms_per_batch": ms3, "runs": n3, "prepare_ms_per_alternation": ms_prep,
                    "median_rot_err_deg": float(np.median(err3)), "p90_rot_err_deg": float(np.percentile(err3, 90))}
    err = rotation_error_deg(chosen["alpha"], chosen["beta"], chosen["gamma"], q_true)
    fp32_peak = fp32_peak_tflops(dev)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peaks = {}
    # (the FP32 CUDA-core peak is measured on this GPU: cuBLAS SGEMM, above)
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    table, kernel_ms = kernel_table(prof, args.steps, B, peaks, fp32_peak)
    if plain is not None:
        plain["kernels"], _ = kernel_table({k: {"ms": v * n32, "launches": prof32[k]["launches"]}
                                            for k, v in plain["kernels_ms_per_step"].items()}, n32, B, peaks, fp32_peak)
        del plain["kernels_ms_per_step"]
    # the roofline of the largest kernel that has a throughput bound (every kernel above it
    # in time is named in `kernels` with its own bound)
    top = max((k for k in table if "bound" in table[k]), key=lambda k: table[k]["ms_per_step"])
    row = table[top]
    dram = DRAM_BYTES_PER_SUBTOMO.get(top)
    clocks = clk.summary()
    line = {
        "metric": METRIC,
        "value": whole_job_value(world, B, ms),
        "unit": "subtomograms/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+bf16x3",
        "precision": "expansion and upsampled-DFT GEMMs as BF16 hi+lo splits (3 MMAs, FP32 accumulation) on "
                     "tcgen05; FP32 elsewhere; FP64 Newton 3x3 solve",
        "data": "synthetic",
        "config": {"workload": f"{B} subtomograms 64^3, L=32, march 8/16/24/32, C=10, 1 Newton step, "
                               f"shift r=5 uf=8, 0 dB", "batch_per_gpu": B, "box": N_BOX, "L": L_MAX,
                   "parallelism": f"replicas x{world}", "l2": "inputs 1.05 GB per step > 126 MB L2"},
        "median_rot_err_deg": float(np.median(err)),
        "p90_rot_err_deg": float(np.percentile(err, 90)),
        "roofline": {"kernel": top, "bound": {"hbm": "hbm", "tensor": "tensor", "fp32": "fp32"}[row["bound"]],
                     "achieved": row["achieved"], "peak": row["peak"], "unit": row["unit"], "frac": row["frac"],
                     "peak_source": "MEASURED_PEAKS.json (hbm_gbs copy bandwidth / bf16_tflops_sustained); "
                                    "fp32: cuBLAS SGEMM measured in this run",
                     "kernel_ms": row["ms_per_step"],
                     "traffic": (dram * B) if dram else None, "traffic_unit": "bytes per launch"},
        "kernels": table,
        "kernel_ms_per_step": kernel_ms,
        "fp32_sgemm_tflops": fp32_peak,
        "plain_fp32": plain,
        "three_alternations": alternations,
        "one_alternation_with_preparation": {"ms_per_step": ms + ms_prep,
                                             "value": whole_job_value(world, B, ms + ms_prep)},
        "e2e": {"value": whole_job_value(world, B, e2e_ms), "unit": "subtomograms/s",
                "h2d_bytes_per_step": int(B * N_BOX ** 3 * 4), "d2h_bytes_per_step": int(B * 8 * 4)},
        "gpu_launches": int(launches),
        "profile_dropped_launches": dropped,
        "clocks": clocks,
    }
    if not args.no_cpu_baseline and world == 1:
        try:
            n = args.cpu_sample
            sample_vols = vols[:n].cpu().numpy()
            sec, o32 = cpu_align(n, template, sample_vols, np.float32)
            _, o64 = cpu_align(n, template, sample_vols, np.float64)
            line["cpu_baseline"] = {"value": 1.0 / sec, "unit": "subtomograms/s", "cores": os.cpu_count(),
                                    "kind": "port", "sample": f"{n} subtomograms of the batch through the oracle "
                                                              f"(FP64 expansion, FP32 search, shift match)"}
            acc = {"sample": n, "ref_median_rot_err_deg": float(np.median(rotation_error_deg(
                o32["alpha"], o32["beta"], o32["gamma"], q_true[:n]))),
                   "ref_fp64_median_rot_err_deg": float(np.median(rotation_error_deg(
                       o64["alpha"], o64["beta"], o64["gamma"], q_true[:n]))),
                   "ref_fp32_vs_fp64_max_deg": float(euler_dev_deg(o32["alpha"], o32["beta"], o32["gamma"],
                                                                   o64["alpha"], o64["beta"], o64["gamma"]).max()),
                   "chosen": accuracy_vs_oracle(chosen, o32, o64, q_true, n)}
            if plain_out is not None:
                acc["plain_fp32"] = accuracy_vs_oracle(plain_out, o32, o64, q_true, n)
            line["accuracy_vs_reference"] = acc
            line["ref_median_rot_err_deg"] = acc["ref_median_rot_err_deg"]
            line["median_dev_vs_ref_deg"] = acc["chosen"]["median_dev_vs_ref_deg"]
            line["frac_within_0p05deg"] = acc["chosen"]["frac_within_0p05deg"]
            # the target's form: the median rotation error against the reference's on the same inputs
            line["median_rot_err_diff_vs_ref_deg"] = abs(acc["chosen"]["median_rot_err_deg"]
                                                         - acc["ref_median_rot_err_deg"])
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "subtomograms/s", "cores": os.cpu_count(),
                                    "kind": "port", "sample": f"failed: {exc!r}"[:200]}
    print(json.dumps(line))


def run_reference(args):
    """The oracle restatement of the reference's alternation on the host cores, on the first
    ``--cpu-sample`` subtomograms of the same batch the GPU arm aligns (same generator, same
    seeds, built on the CPU)."""
    _, rank, _ = dist_env()
    if rank != 0:  # under torchrun rank 0 alone times the host cores; the others exit 0
        return
    import torch

    torch.set_num_threads(os.cpu_count() or 1)
    rng = np.random.default_rng(args.seed)
    template = make_template(rng)
    sample = max(1, args.cpu_sample)
    vols, q, _ = make_batch(template, np.random.default_rng(args.seed + 1), args.batch, "cpu", count=sample)
    vols = vols.numpy()
    times = []
    for it in range(args.warmup + args.steps):
        sec, _ = cpu_align(sample, template, vols)
        if it >= args.warmup:
            times.append(sec)
    per = float(np.mean(times))
    value = 1.0 / per
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "subtomograms/s",
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per * sample * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.batch} subtomograms 64^3, L=32, march 8/16/24/32, C=10, 1 Newton step, "
                               f"shift r=5 uf=8, 0 dB", "batch_per_gpu": args.batch, "box": N_BOX, "L": L_MAX,
                   "parallelism": "host cores"},
        "cpu_baseline": {"value": value, "unit": "subtomograms/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": f"the first {sample} subtomograms of the batch per step through the oracle "
                                   f"restatement (FP64 expansion, FP32 search, shift match)"},
        "e2e": {"value": value, "unit": "subtomograms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def highband_oracle(template, vols, L, Li, uf, radius, n, gpu_runs):
    """The FP64 oracle on the first n subtomograms at 128^3: the streamed FP64 expansion of the
    template and the volumes, sigma, the orientation search in FP64, and the shift match in FP64
    at the GPU run's own orientation (so the shift's error is the shift stage's); each GPU run's
    rotation, shift, rotation-score and shift-peak deviations from it."""
    from matcha_b200.core import fle_tables as T
    from oracle import fle as F
    from oracle import matcha as M
    from oracle import pipeline as OP
    from oracle import shift as OS

    N = template.shape[0]
    r = min(N // 2, int(N // 2 * 0.95))
    t0 = time.perf_counter()
    tb = T.lap_eig_ball(N, L, r)
    ff = OP.FoldedFLE(tb, N, float(r), dense=False)
    v = np.asarray(vols[:n], dtype=np.float64)
    a = ff.evaluate_t_streamed(np.concatenate([template[None].astype(np.float64), v]))
    sigma = F.compute_sigma(tb, a[0], a[1:])
    al, be, ga, score = M.search_orientations(sigma, list(Li) + [L], L, K=2, candidates=10, num_steps=1,
                                              dtype=np.float64)
    ref = OS.load_reference_full(template, N, 1.0)
    out = {"sample": n, "seconds": None}
    for name, g in gpu_runs.items():
        ang = [np.asarray(g[k][:n], dtype=np.float64) for k in ("alpha", "beta", "gamma")]
        rot = euler_dev_deg(*ang, al, be, ga)
        tr = np.asarray(g["tracker"][:n], dtype=np.float64)
        deg = OS.euler_zyz_deg_from_quat_conj(tr)
        sh, pk = [], []
        for i in range(n):
            s_i, p_i = OS.estimate_shift_like_relion(ref, v[i], np.zeros(3), deg[i], uf, radius)
            sh.append(s_i)
            pk.append(p_i)
        sh, pk = np.array(sh), np.array(pk)
        rs = np.asarray(g["rotation_score"][:n], dtype=np.float64)
        ss = np.asarray(g["shift_score"][:n], dtype=np.float64)
        out[name] = {"median_rot_dev_deg": float(np.median(rot)), "max_rot_dev_deg": float(rot.max()),
                     "max_shift_dev_px": float(np.abs(np.asarray(g["shift"][:n]) - sh).max()),
                     "max_rotation_score_rel_dev": float(np.max(np.abs(rs - score) / np.abs(score))),
                     "max_shift_peak_rel_dev": float(np.max(np.abs(ss - pk) / np.abs(pk)))}
    out["seconds"] = time.perf_counter() - t0
    return out


def run_highband(args):
    """Config 5: one and three alternations at 128^3, L=64 (1500-blob template, -5 dB, shifts in
    +-8 px) on one GPU: throughput and the tracker's rotation error of the chosen precision
    (expansion BF16 hi+lo; shift match on the tensor cores where its kernels cover the box),
    its deviations from the plain-FP32 run over the whole batch, and both runs' deviations from
    the FP64 oracle on a sample."""
    import torch

    from matcha_b200.pipeline import AlignmentStep, StepConfig

    dev = torch.device("cuda:0")
    N, L, B = 128, 64, (args.batch if args.batch != 1000 else 512)
    if args.split_degree is None:
        args.split_degree = 40  # BF16 with the split correction above l = 40
    Li, uf, radius = [16, 32, 48], 8, 8
    rng = np.random.default_rng(args.seed)
    template = make_template(rng, N=N, n_blobs=1500, window=12)
    vols, q_true, _ = make_batch(template, np.random.default_rng(args.seed + 1), B, dev, snr_db=-5.0, max_shift=8.0)
    ident = torch.zeros((B, 4), device=dev, dtype=torch.float64)
    ident[:, 0] = 1
    z3 = torch.zeros((B, 3), device=dev)
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(1, args.steps)

    def one_precision(precision, split_degree=None):
        step = AlignmentStep(StepConfig(N=N, L=L, Li=Li, batch=B, shift_search_radius=radius,
                                        shift_upsample_factor=uf, precision=precision,
                                        expansion_split_degree=split_degree), dev)
        step.set_template(template)
        tracker = ident.clone()
        for _ in range(max(1, args.warmup)):
            tracker.copy_(ident)
            out = step(vols, vols, tracker, z3)
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(n):
            tracker.copy_(ident)
            out = step(vols, vols, tracker, z3)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / n
        res = {k: out[k].cpu().numpy() for k in ("alpha", "beta", "gamma", "shift", "shift_score",
                                                   "rotation_score", "tracker")}
        # one more alternation with every library launch timed (CUDA events; not the number above)
        from matcha_b200 import _native as nat

        tracker.copy_(ident)
        nat.profile_start(256)
        step(vols, vols, tracker, z3)
        nat.profile_stop()
        prof, _ = nat.profile_read()
        res["kernel_ms"] = {k: round(v["ms"], 3) for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])}
        fle = step.correlator.fle
        prec = f"expansion {fle.precision}" + (f" (plain BF16 up to degree {split_degree}: "
                                               f"{fle.split_tiles()[0]} of {fle.split_tiles()[1]} GEMM tiles split)"
                                               if split_degree is not None else "") + \
            f", upsampled DFT {step.shifter.effective_precision}"
        three = None
        if precision != "fp32" and split_degree is None:
            tracker.copy_(ident)
            local = torch.zeros((B, 3), device=dev)
            e0.record(st)
            step.run_alternations(vols, tracker, local, z3, z3, 3)
            e1.record(st)
            torch.cuda.synchronize()
            ms3 = e0.elapsed_time(e1)
            err3 = tracker_error_deg(tracker.cpu().numpy(), q_true)
            three = {"ms_per_batch": ms3, "value": B / (ms3 * 1e-3), "median_rot_err_deg": float(np.median(err3)),
                     "p90_rot_err_deg": float(np.percentile(err3, 90))}
        del step
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        return ms, res, prec, three

    ms, chosen, prec, three = one_precision("auto", None)
    err1 = rotation_error_deg(chosen["alpha"], chosen["beta"], chosen["gamma"], q_true)
    line = {
        "metric": "subtomograms/s at 128^3 L=64 (one alternation), high-bandlimit shape",
        "value": B / (ms * 1e-3), "unit": "subtomograms/s", "ms_per_alternation": ms, "steps": n,
        "dtype": "f32+bf16x3", "data": "synthetic",
        "config": {"workload": f"{B} subtomograms 128^3, L=64, march 16/32/48/64, C=10, 1 Newton step, "
                               f"shift r=8 uf=8, -5 dB, 1500 blobs", "precision": prec},
        "median_rot_err_deg": float(np.median(err1)), "p90_rot_err_deg": float(np.percentile(err1, 90)),
        "three_alternations": three, "kernel_ms_per_alternation": chosen.pop("kernel_ms"),
    }
    runs = {"chosen": chosen}
    if args.split_degree is not None:
        # the shape's own schedule: plain BF16 up to degree split_degree, the hi+lo split above
        msx, sched, precx, _ = one_precision("auto", args.split_degree)
        kern = sched.pop("kernel_ms")
        runs[f"plain_bf16_to_l{args.split_degree}"] = sched
        ang = lambda d: [np.asarray(d[k], dtype=np.float64) for k in ("alpha", "beta", "gamma")]
        dv = euler_dev_deg(*ang(sched), *ang(chosen))
        line[f"plain_bf16_to_l{args.split_degree}"] = {
            "ms_per_alternation": msx, "value": B / (msx * 1e-3), "precision": precx,
            "gemm_tc_kernel_ms": kern.get("gemm_tc_kernel"),
            "vs_chosen": {"median_rot_dev_deg": float(np.median(dv)), "max_rot_dev_deg": float(dv.max()),
                          "frac_within_0p05deg": float(np.mean(dv < 0.05)),
                          "shift_equal_frac": float(np.mean(np.all(np.abs(sched["shift"] - chosen["shift"]) < 1e-6,
                                                                   axis=1)))}}
    if not args.no_fp32:
        ms32, plain, prec32, _ = one_precision("fp32")
        plain.pop("kernel_ms")
        runs["plain_fp32"] = plain
        ang = lambda d: [np.asarray(d[k], dtype=np.float64) for k in ("alpha", "beta", "gamma")]
        dev_deg = euler_dev_deg(*ang(chosen), *ang(plain))
        line["plain_fp32"] = {
            "ms_per_alternation": ms32, "value": B / (ms32 * 1e-3), "precision": prec32,
            "chosen_vs_plain": {
                "median_rot_dev_deg": float(np.median(dev_deg)), "max_rot_dev_deg": float(dev_deg.max()),
                "frac_within_0p05deg": float(np.mean(dev_deg < 0.05)),
                "shift_equal_frac": float(np.mean(np.all(np.abs(chosen["shift"] - plain["shift"]) < 1e-6, axis=1))),
                "max_shift_peak_rel_dev": float(np.max(np.abs(chosen["shift_score"] - plain["shift_score"])
                                                       / np.abs(plain["shift_score"]))),
                "median_rotation_score_rel_dev": float(np.median(np.abs(chosen["rotation_score"] - plain["rotation_score"])
                                                                 / np.abs(plain["rotation_score"])))}}
    if args.cpu_sample > 0 and not args.no_cpu_baseline:
        line["vs_fp64_oracle"] = highband_oracle(template, vols[:args.cpu_sample].cpu().numpy(), L, Li, uf, radius,
                                                 min(args.cpu_sample, B), runs)
    print(json.dumps(line))


def run_mixed(args):
    """One alternation of a mixed batch of boxes 48, 64 and 96 as one CUDA graph replay."""
    import torch

    from matcha_b200.mixed import BoxSpec, MixedAlignment
    from matcha_b200.pipeline import StepConfig

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(args.seed)
    total = 4096
    boxes = {48: (24, [6, 12, 18], 150), 64: (32, [8, 16, 24], 400), 96: (48, [12, 24, 36], 900)}
    which = rng.integers(0, 3, total)
    counts = {N: int(np.sum(which == k)) for k, N in enumerate(boxes)}
    specs, data = [], {}
    for N, (L, Li, blobs) in boxes.items():
        tmpl = make_template(rng, N=N, n_blobs=blobs, window=12 if N > 64 else None)
        B = counts[N]
        snr = rng.uniform(-10.0, 5.0, B)
        vols, q, _ = make_batch(tmpl, np.random.default_rng(args.seed + N), B, dev, snr_db=snr, max_shift=6.0)
        data[N] = (vols, q)
        specs.append(BoxSpec(StepConfig(N=N, L=L, Li=Li, batch=B, shift_search_radius=6, shift_upsample_factor=8),
                             tmpl))
    t0 = time.time()
    mixed = MixedAlignment(specs, dev, tune=True)
    cap = mixed.capture(counts)
    setup_s = time.time() - t0
    for N in counts:
        cap.volumes[N].copy_(data[N][0])
    st = torch.cuda.current_stream()
    for _ in range(max(1, args.warmup)):
        cap.restore()
        cap.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(1, args.steps)
    e0.record(st)
    for _ in range(n):
        cap.restore()
        out = cap.replay()
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    per_box = {}
    for N, o in out.items():
        err = rotation_error_deg(*(o[k].cpu().numpy() for k in ("alpha", "beta", "gamma")), data[N][1])
        spec = mixed.boxes[N][0]
        per_box[str(N)] = {"count": counts[N], "L": spec.cfg.L, "median_rot_err_deg": float(np.median(err)),
                           "shift_precision": mixed.boxes[N][1].shifter.effective_precision,
                           "shift_tile_rows": spec.cfg.shift_tile_rows,
                           "tile_timings_ms": {str(k): v for k, v in spec.timings.items()}}
    # where the time goes: one eager alternation per box size with every library launch timed
    # (CUDA events around each launch; not the graph-replay number above)
    from matcha_b200 import _native as nat

    for N in counts:
        cap.restore()
        nat.profile_start(256)
        mixed({N: (cap.volumes[N], cap.tracker[N], cap.shift[N])})
        nat.profile_stop()
        prof, _ = nat.profile_read()
        per_box[str(N)]["kernel_ms"] = {k: round(v["ms"], 3)
                                        for k, v in sorted(prof.items(), key=lambda kv: -kv[1]["ms"])}
    print(json.dumps({
        "metric": "subtomograms/s, mixed boxes 48/64/96 (one alternation, one CUDA graph replay)",
        "value": total / (ms * 1e-3), "unit": "subtomograms/s", "ms_per_step": ms, "steps": n,
        "data": "synthetic", "config": {"workload": "4096 subtomograms, boxes {48,64,96}^3 drawn uniformly, L "
                                                    "{24,32,48}, templates of 150/400/900 blobs, shifts +-6, SNR "
                                                    "U[-10,5] dB, C=10, 1 Newton step, uf=8"},
        "setup_s": setup_s, "boxes": per_box}))


def main():
    args = parse()
    if args.mixed:
        run_mixed(args)
        return
    if args.highband:
        run_highband(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
