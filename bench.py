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
# DRAM bytes (read + write) of updft23_tc_kernel per subtomogram, from an ncu capture of the same kernel
# at 200 subtomograms (dram__bytes_read.sum + dram__bytes_write.sum divided by 200)
UPDFT23_DRAM_BYTES_PER_SUBTOMO = 1_526_000


def parse():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=1000)
    p.add_argument("--cpu-sample", type=int, default=2, help="subtomograms per CPU-baseline step")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-fp32", action="store_true", help="skip the plain-FP32 comparison run")
    p.add_argument("--seed", type=int, default=0)
    p.add_argument("--highband", action="store_true",
                   help="the high-bandlimit shape instead of the metric's: 128^3, L=64, march 16/32/48/64, "
                        "shift r=8, -5 dB (a reported extra, not the metric; --batch defaults to 64)")
    return p.parse_args()


# ---------------------------------------------------------------- synthetic data (numpy, host)
def make_template(rng, N=N_BOX, n_blobs=400, window=None):
    """Gaussian blobs in two lobes under a soft spherical mask; window (voxels) evaluates each
    blob only within that distance of its centre per axis (for large boxes)."""
    g = np.arange(N) - N // 2
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    vol = np.zeros((N, N, N))
    lobes = [(26.0, np.array([-3.0, 1.0, 0.0])), (18.0, np.array([6.0, -4.0, 3.0]))]
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


def make_batch(template, rng, B, device, snr_db=0.0, max_shift=5.0):
    """Rotated (reference rotate_volumes convention), shifted, noisy subtomograms on the device."""
    import torch
    import torch.nn.functional as TF
    from scipy.spatial.transform import Rotation as R

    N = template.shape[0]
    q = rng.standard_normal((B, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    shifts = rng.uniform(-max_shift, max_shift, (B, 3)).astype(np.float32)
    mats = torch.tensor(R.from_quat(np.roll(q, -1, axis=1)).as_matrix(), dtype=torch.float32, device=device)
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
    out = torch.empty((B, N, N, N), device=device, dtype=torch.float32)
    sh = torch.from_numpy(shifts).to(device)
    noise_gen = torch.Generator(device=device)
    noise_gen.manual_seed(int(rng.integers(1 << 31)))
    for s in range(0, B, 50):
        e = min(B, s + 50)
        rc = (mats[s:e] @ coords).permute(0, 2, 1).reshape(e - s, N + 1, N + 1, N + 1, 3)
        v = TF.grid_sample(tp.expand(e - s, -1, -1, -1, -1), rc, mode="bilinear", align_corners=True)
        v = v[:, 0, :N, :N, :N]
        ph = torch.exp(-2j * np.pi * (kz[None] * sh[s:e, 0, None, None, None] + ky[None] * sh[s:e, 1, None, None, None]
                                      + kx[None] * sh[s:e, 2, None, None, None]))
        v = torch.fft.ifftn(torch.fft.fftn(v, dim=(1, 2, 3)) * ph, dim=(1, 2, 3)).real
        power = (v[:, mask] ** 2).mean(dim=1)
        noise = torch.randn(v.shape, device=device, generator=noise_gen) * torch.sqrt(
            power * 10.0 ** (-snr_db / 10.0))[:, None, None, None]
        out[s:e] = v + noise
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
def cpu_align(sample, template, vols, q_true, threads=None):
    """Oracle pipeline on a few subtomograms; returns (seconds per subtomogram, outputs)."""
    from matcha_b200.core import fle_tables as T
    from oracle import fle as OF
    from oracle import pipeline as OP
    from oracle import shift as OS

    radius = min(N_BOX // 2, int(N_BOX // 2 * 0.95))
    tb = T.lap_eig_ball(N_BOX, L_MAX, radius)
    ff = OP.FoldedFLE(tb, N_BOX, float(radius))
    a_t = ff.evaluate_t(template[None])[0]
    ref = OS.load_reference_full(template, N_BOX, 1.0)
    v = vols[:sample].astype(np.float64)
    tracker = np.tile([1.0, 0, 0, 0], (sample, 1))
    t0 = time.perf_counter()
    out = OP.align_batch(ff, a_t, ref, v, v, tracker, np.zeros((sample, 3)), L_MAX, LI, uf=UPSAMPLE,
                         shift_radius=SHIFT_RADIUS)
    dt = time.perf_counter() - t0
    return dt / sample, out


# ---------------------------------------------------------------- our implementation
def run_ours(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device(f"cuda:{local}")
    from matcha_b200.pipeline import AlignmentStep, StepConfig

    rng = np.random.default_rng(args.seed)
    template = make_template(rng)
    B = args.batch
    vols, q_true, shifts = make_batch(template, np.random.default_rng(args.seed + 1 + rank), B, dev)
    step = AlignmentStep(StepConfig(N=N_BOX, L=L_MAX, Li=LI, batch=B, shift_search_radius=SHIFT_RADIUS,
                                    shift_upsample_factor=UPSAMPLE), dev)
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
    # per-stage breakdown (one extra untimed step)
    st = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    tracker.copy_(ident)
    ev[0].record(st)
    sigma, norms = step.correlator.get_sigma_upto(vols, L_MAX)
    ev[1].record(st)
    a, b, g, sc = step.matcher.search_orientations(sigma)
    ev[2].record(st)
    step(vols, vols, tracker, zeros3)  # full step (includes a second sigma/search)
    ev[3].record(st)
    torch.cuda.synchronize()
    t_sigma = ev[0].elapsed_time(ev[1])
    t_search = ev[1].elapsed_time(ev[2])
    t_full = ev[2].elapsed_time(ev[3])
    stages = {"fle_sigma_ms": t_sigma, "search_ms": t_search, "shift_ms": max(0.0, t_full - t_sigma - t_search)}
    # per-kernel timing of the candidates for the roofline (launch stream events)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0, b0, g0 = step.matcher._grid_search_so3fft(sigma)
    torch.cuda.synchronize()
    e0.record(st)
    step.matcher.march(a0, b0, g0, sigma)
    e1.record(st)
    torch.cuda.synchronize()
    t_march = e0.elapsed_time(e1)
    # timed region
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        clk.wait_first(one)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        step.shifter.profile(args.steps)  # CUDA events between the shift match's kernel groups
        torch.cuda.nvtx.range_push("timed")  # lets a profiler select the timed launches
        start.record(st)
        for _ in range(args.steps):
            out = one()
        end.record(st)
        torch.cuda.nvtx.range_pop()
        torch.cuda.synchronize()
    ms = start.elapsed_time(end) / args.steps
    shift_prof, shift_calls = step.shifter.profile_read()
    step.shifter.profile(0)
    if world > 1:
        tms = torch.tensor([ms], device=dev)
        dist.all_reduce(tms, op=dist.ReduceOp.MAX)
        ms = float(tms.item())
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
    if world > 1:
        t2 = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
        e2e_ms = float(t2.item())
    # the same step with the plain FP32 kernels (the expansion GEMM and the upsampled DFT on
    # CUDA cores instead of the BF16 hi+lo tensor-core split): the comparison the metric names
    plain = None
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
        e32s, e32e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e32s.record(st)
        for _ in range(n32):
            tracker.copy_(ident)
            step32(vols, vols, tracker, zeros3)
        e32e.record(st)
        torch.cuda.synchronize()
        ms32 = e32s.elapsed_time(e32e) / n32
        if world > 1:
            t32 = torch.tensor([ms32], device=dev)
            dist.all_reduce(t32, op=dist.ReduceOp.MAX)
            ms32 = float(t32.item())
        plain = {"value": world * B / (ms32 * 1e-3), "ms_per_step": ms32, "steps": n32,
                 "chosen_speedup": ms32 / ms}
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
    step.prepare(vols, zeros3, tracker)
    ep1.record(st)
    torch.cuda.synchronize()
    ms_prep = ep0.elapsed_time(ep1)
    if world > 1:
        t3 = torch.tensor([ms3], device=dev)
        dist.all_reduce(t3, op=dist.ReduceOp.MAX)
        ms3 = float(t3.item())
    # rotation error of the tracker after the third alternation (the last run's)
    trk = tracker.cpu().numpy()
    err3 = tracker_error_deg(trk, q_true)
    alternations = {"value": world * B / (ms3 * 1e-3), "unit": "subtomograms/s", "alternations": 3,
                    "ms_per_batch": ms3, "runs": n3, "prepare_ms_per_alternation": ms_prep,
                    "median_rot_err_deg": float(np.median(err3)), "p90_rot_err_deg": float(np.percentile(err3, 90))}
    # accuracy of one more chosen-path step on the full batch (the pieces of the end-to-end
    # runs overwrote the step's output buffers)
    tracker.copy_(ident)
    out = one()
    al, be, ga = (out[k].cpu().numpy() for k in ("alpha", "beta", "gamma"))
    err = rotation_error_deg(al, be, ga, q_true)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    # roofline of the dominant kernel, the fused passes 2+3 of the shift match's upsampled DFT
    # (tcgen05, BF16 hi+lo split): algorithmic FLOP per subtomogram = the three split GEMM
    # segments of pass 2 (rows U*N/2, N-tile 2U, K 2N) and pass 3 (rows U^2, U columns, K N + 2
    # with the Nyquist pair), 2*M*N*K each; its time per launch from the events recorded
    # around it in every timed step
    U = int(np.ceil(UPSAMPLE * (2 * SHIFT_RADIUS + 1)))
    flop_sub = 3 * (2 * (U * N_BOX // 2) * (2 * U) * (2 * N_BOX) + 2 * U * U * U * (N_BOX + 2))
    t_k = shift_prof["updft_pass23"] / max(1, shift_calls)
    achieved = flop_sub * B / (t_k * 1e-3) / 1e12 if t_k > 0 else None
    clocks = clk.summary()
    peak = float(peaks.get("bf16_tflops_sustained", 1400.0))
    line = {
        "metric": METRIC,
        "value": world * B / (ms * 1e-3),
        "unit": "subtomograms/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{B} subtomograms 64^3, L=32, march 8/16/24/32, C=10, 1 Newton step, "
                               f"shift r=5 uf=8, 0 dB", "batch_per_gpu": B, "box": N_BOX, "L": L_MAX,
                   "parallelism": f"replicas x{world}", "l2": "inputs 1.05 GB per step > 126 MB L2"},
        "median_rot_err_deg": float(np.median(err)),
        "p90_rot_err_deg": float(np.percentile(err, 90)),
        "stages_ms": stages,
        "roofline": {"kernel": "updft23_tc_kernel", "bound": "tensor", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": (achieved / peak) if achieved else None,
                     "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (kernel timed inside long steps)",
                     "kernel_ms": t_k, "flop_per_subtomogram": flop_sub,
                     "traffic": (UPDFT23_DRAM_BYTES_PER_SUBTOMO * B) if UPDFT23_DRAM_BYTES_PER_SUBTOMO else None,
                     "traffic_unit": "bytes per launch"},
        "shift_kernel_ms_per_step": {k: v / max(1, shift_calls) for k, v in shift_prof.items()},
        "plain_fp32": plain,
        "three_alternations": alternations,
        "e2e": {"value": world * B / (e2e_ms * 1e-3), "unit": "subtomograms/s",
                "h2d_bytes_per_step": int(B * N_BOX ** 3 * 4), "d2h_bytes_per_step": int(B * 8 * 4)},
        "gpu_launches": KERNELS_PER_STEP * args.steps,
        "clocks": clocks,
    }
    if not args.no_cpu_baseline and world == 1:
        try:
            import torch as _t

            sec, _ = cpu_align(args.cpu_sample, template, vols[: args.cpu_sample].cpu().numpy(), q_true)
            line["cpu_baseline"] = {"value": 1.0 / sec, "unit": "subtomograms/s", "cores": os.cpu_count(),
                                    "kind": "port", "sample": f"{args.cpu_sample} subtomograms through the oracle "
                                                              f"(folded exact FLE, sigma, grid, march, shift)"}
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "subtomograms/s", "cores": os.cpu_count(),
                                    "kind": "port", "sample": f"failed: {exc!r}"[:200]}
    print(json.dumps(line))


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    rng = np.random.default_rng(args.seed)
    template = make_template(rng)
    sample = max(1, args.cpu_sample)
    # inputs: rotated, noisy subtomograms made on the host (no GPU on this arm)
    from scipy.ndimage import map_coordinates
    from scipy.spatial.transform import Rotation as R

    q = rng.standard_normal((sample, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    g = np.linspace(-1, 1, N_BOX + 1)
    wg, hg, dg = np.meshgrid(g, g, g, indexing="ij")
    coords = np.stack([dg.ravel(), hg.ravel(), wg.ravel()], 0)
    vols = np.zeros((sample, N_BOX, N_BOX, N_BOX), dtype=np.float32)
    tp = np.pad(template, ((0, 1), (0, 1), (0, 1)))
    for i in range(sample):
        rc = R.from_quat(np.roll(q[i], -1)).as_matrix() @ coords
        idx = (rc + 1) / 2 * N_BOX  # align_corners=True over N+1 samples
        v = map_coordinates(tp, [idx[2], idx[1], idx[0]], order=1, mode="constant").reshape(N_BOX + 1, N_BOX + 1,
                                                                                              N_BOX + 1)
        v = v[:N_BOX, :N_BOX, :N_BOX]
        vols[i] = v + rng.standard_normal(v.shape) * np.sqrt((v ** 2).mean())
    times = []
    for it in range(args.warmup + args.steps):
        sec, _ = cpu_align(sample, template, vols, q)
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
                         "sample": f"{sample} subtomograms per step through the oracle restatement"},
        "e2e": {"value": value, "unit": "subtomograms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_highband(args):
    """One and three alternations at 128^3, L=64 (1500-blob template, -5 dB, shifts in +-8 px):
    throughput and the tracker's rotation error, on one GPU."""
    import torch

    from matcha_b200.pipeline import AlignmentStep, StepConfig

    dev = torch.device("cuda:0")
    N, L, B = 128, 64, (args.batch if args.batch != 1000 else 64)
    rng = np.random.default_rng(args.seed)
    template = make_template(rng, N=N, n_blobs=1500, window=12)
    vols, q_true, _ = make_batch(template, np.random.default_rng(args.seed + 1), B, dev, snr_db=-5.0, max_shift=8.0)
    step = AlignmentStep(StepConfig(N=N, L=L, Li=[16, 32, 48], batch=B, shift_search_radius=8,
                                    shift_upsample_factor=8), dev)
    step.set_template(template)
    ident = torch.zeros((B, 4), device=dev, dtype=torch.float64)
    ident[:, 0] = 1
    tracker = ident.clone()
    z3 = torch.zeros((B, 3), device=dev)
    for _ in range(max(1, args.warmup)):
        tracker.copy_(ident)
        out = step(vols, vols, tracker, z3)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = max(1, args.steps)
    e0.record(st)
    for _ in range(n):
        tracker.copy_(ident)
        out = step(vols, vols, tracker, z3)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n
    err1 = rotation_error_deg(*(out[k].cpu().numpy() for k in ("alpha", "beta", "gamma")), q_true)
    tracker.copy_(ident)
    local = torch.zeros((B, 3), device=dev)
    e0.record(st)
    step.run_alternations(vols, tracker, local, z3, z3, 3)
    e1.record(st)
    torch.cuda.synchronize()
    ms3 = e0.elapsed_time(e1)
    err3 = tracker_error_deg(tracker.cpu().numpy(), q_true)
    print(json.dumps({
        "metric": "subtomograms/s at 128^3 L=64 (one alternation), high-bandlimit shape",
        "value": B / (ms * 1e-3), "unit": "subtomograms/s", "ms_per_alternation": ms, "steps": n,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{B} subtomograms 128^3, L=64, march 16/32/48/64, C=10, 1 Newton step, "
                               f"shift r=8 uf=8, -5 dB, 1500 blobs", "precision": "bf16x3 expansion, "
                               "fp32 upsampled DFT (box 128 is outside the tensor-core shift kernels)"},
        "median_rot_err_deg": float(np.median(err1)), "p90_rot_err_deg": float(np.percentile(err1, 90)),
        "three_alternations": {"ms_per_batch": ms3, "value": B / (ms3 * 1e-3),
                               "median_rot_err_deg": float(np.median(err3)),
                               "p90_rot_err_deg": float(np.percentile(err3, 90))},
    }))


def main():
    args = parse()
    if args.highband:
        run_highband(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
