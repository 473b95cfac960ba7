"""Small, self-contained runs of each stage of the alignment path, for profilers.

    python bench_cases.py shift  200   # ShiftMatcher.search_shifts, 64^3, uf 8, r 5
    python bench_cases.py search 296   # Matcha.search_orientations, L 32, C 10
    python bench_cases.py fle    256   # CrossCorrelationMatcher.get_sigma, 64^3, L 32
    python bench_cases.py prepare 1000 # shifted patch, masked normalisation, rotation, 64^3
    python bench_cases.py reader 1000  # MRC decode of 1000 64^3 files into pinned memory
    python bench_cases.py graph 64     # one alternation, 64^3 L 32: eager calls vs a CUDA graph
    python bench_cases.py shift 1000 --stages   # plus ShiftMatcher.profile per kernel group
    python bench_cases.py shift 64 --box 128 --radius 8 --kernels   # 128^3, r 8: time per kernel
    python bench_cases.py fftbound 4 --box 128  # cuFFT of the 2x oversampled grid (comparison only)

Each case builds its inputs on the device from a fixed seed (random volumes, Haar rotations,
random shifts; a synthetic sigma with a known optimum for the search), runs the stage three
times untimed, then ``--reps`` more times between CUDA events and prints the mean time per
call.  A kernel profiler attached to the process sees the same launches the bench makes for
that stage, on a batch small enough to capture quickly.
"""
from __future__ import annotations

import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import numpy as np
import torch


class _Cfg(dict):
    __getattr__ = dict.__getitem__


def _shift(B: int, dev, box=64, radius=5, precision="bf16x3"):
    from matcha_b200.core.ShiftMatcher import ShiftMatcher

    N = box
    cfg = _Cfg(N=N, voxel_size=1.0, num_subtomograms_per_batch=B, shift_upsample_factor=8,
               shift_search_radius=radius, do_ctf_correction=False, box_size=N)
    sm = ShiftMatcher(cfg, dev, torch.complex64, precision=precision)
    rng = np.random.default_rng(0)
    sm.set_reference(rng.standard_normal((N, N, N)).astype(np.float32))
    vols = torch.randn(B, N, N, N, device=dev)
    q = rng.standard_normal((B, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    z = torch.from_numpy(rng.uniform(-2, 2, (B, 3)).astype(np.float32)).to(dev)
    run = lambda: sm.search_shifts(subtomos=vols, ctfs=None, shift_zyx=z, rotation_tracker=q)
    run.matcher = sm
    return run


def _search(B: int, dev):
    from matcha_b200.core.Matcha import Matcha
    from matcha_b200.core.wigner_index import compute_size

    L = 32
    rng = np.random.default_rng(0)
    n = compute_size(L + 1)
    sig = (rng.standard_normal((B, n)) + 1j * rng.standard_normal((B, n))).astype(np.complex64)
    st = torch.from_numpy(sig).to(dev)
    m = Matcha(batchsize=B, device=dev, L_max=L, matcha_config=dict(Li=[8, 16, 24, 32], candidates=10,
                                                                   num_steps=1))
    return lambda: m.search_orientations(st)


def _fle(B: int, dev):
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher

    N = 64
    cc = CrossCorrelationMatcher(N=N, device=dev, batchsize=B, bandlimit=32, radius=30, precision_mode="fast",
                                 precision="bf16x3")
    rng = np.random.default_rng(0)
    cc.set_template(rng.standard_normal((N, N, N)).astype(np.float32))
    vols = torch.randn(B, N, N, N, device=dev)
    return lambda: cc.get_sigma_upto(vols, 32)


def _prepare(B: int, dev):
    from matcha_b200 import _native as nat

    N = 64
    lib = nat.load()
    rng = np.random.default_rng(0)
    vols = torch.randn(B, N, N, N, device=dev)
    shift = torch.from_numpy(rng.uniform(-2, 2, (B, 3)).astype(np.float32)).to(dev)
    q = rng.standard_normal((B, 4))
    tracker = torch.from_numpy(q / np.linalg.norm(q, axis=1, keepdims=True)).to(dev)
    work, out = torch.empty((B, N, N, N, 2), device=dev), torch.empty_like(vols)
    stats = torch.empty((B, 2), dtype=torch.float64, device=dev)

    def run():
        nat.check(lib.mtb_prepare_subtomos(nat.ptr(vols), B, N, nat.ptr(shift), nat.ptr(tracker), 30.0,
                                           nat.ptr(work), nat.ptr(stats), nat.ptr(out), nat.stream_ptr(dev)),
                  "mtb_prepare_subtomos")

    return run


def _reader(B: int, reps: int) -> int:
    """Host only: writes B 64^3 float32 MRC files to a temporary directory, reads them once
    to warm the page cache, then times ``reps`` reads of all of them into a pinned batch
    (wall clock; the decode uses no GPU)."""
    import os
    import tempfile
    import time

    from matcha_b200.reader import MrcReader, write_mrc

    N = 64
    rng = np.random.default_rng(0)
    with tempfile.TemporaryDirectory() as d:
        paths = []
        for i in range(B):
            p = os.path.join(d, f"{i}_data.mrc")
            write_mrc(p, rng.standard_normal((N, N, N)).astype(np.float32))
            paths.append(p)
        r = MrcReader(0)
        out = torch.empty((B, N, N, N), dtype=torch.float32, pin_memory=torch.cuda.is_available())
        st = r.read_into(paths, out, (N, N, N))
        if st.any():
            print("read failed", file=sys.stderr)
            return 1
        t0 = time.perf_counter()
        for _ in range(reps):
            r.read_into(paths, out, (N, N, N))
        dt = (time.perf_counter() - t0) / reps
        # the reference reader's steps with numpy in place of mrcfile: a thread pool reads each
        # file into an array of its own, torch.stack makes the batch, pin_memory copies it
        from concurrent.futures import ThreadPoolExecutor

        def one(p):
            return torch.from_numpy(np.fromfile(p, dtype="<f4", offset=1024).reshape(N, N, N))

        with ThreadPoolExecutor(max_workers=os.cpu_count()) as ex:
            t0 = time.perf_counter()
            for _ in range(reps):
                batch = torch.stack(list(ex.map(one, paths)))
                if torch.cuda.is_available():
                    batch = batch.pin_memory()
            dt_np = (time.perf_counter() - t0) / reps
    threads = os.cpu_count()
    print(f"reader batch {B}: {dt * 1e3:.3f} ms per batch, {B / dt:.0f} files/s, "
          f"{B * N ** 3 * 4 / dt / 1e9:.2f} GB/s ({threads} hardware threads); per-file arrays + stack"
          f"{' + pin' if torch.cuda.is_available() else ''}: {dt_np * 1e3:.3f} ms per batch, {B / dt_np:.0f} files/s")
    return 0


def _graph(B: int, reps: int) -> int:
    """One alternation (AlignmentStep at 64^3, L 32) on B random volumes: eager calls against
    the replay of its CUDA graph, CUDA events, ``reps`` calls each."""
    from matcha_b200.pipeline import AlignmentStep, StepConfig

    dev = torch.device("cuda:0")
    rng = np.random.default_rng(0)
    step = AlignmentStep(StepConfig(batch=B), dev)
    step.set_template(rng.standard_normal((64, 64, 64)).astype(np.float32))
    cap = step.capture(B)
    cap.volumes.copy_(torch.randn(B, 64, 64, 64, device=dev))
    tracker = cap.tracker.clone()
    zeros = torch.zeros((B, 3), device=dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = {}
    for name, fn in (("eager", lambda: step(cap.volumes, cap.volumes, tracker, zeros)), ("graph", cap.replay)):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        times[name] = e0.elapsed_time(e1) / reps
    print(f"graph batch {B}: eager {times['eager']:.3f} ms, graph replay {times['graph']:.3f} ms per alternation")
    return 0


def _fftbound(B: int, reps: int, box: int) -> int:
    """A lower bound for the FFT-plus-shell form of the expansion (the reference's NUFFT path)
    at box N: one complex64 FFT of each volume's 2x oversampled (2N)^3 grid, the NUFFT's own
    FFT alone (no spreading, no spherical-harmonic or radial step), timed with cuFFT through
    torch.fft on B volumes.  A comparison measurement only: nothing in the library calls cuFFT."""
    import torch

    dev = torch.device("cuda:0")
    n = 2 * box
    x = torch.randn((B, n, n, n), device=dev, dtype=torch.complex64)
    for _ in range(3):
        torch.fft.fftn(x, dim=(1, 2, 3))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.fft.fftn(x, dim=(1, 2, 3))
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    print(f"fftbound box {box}: ({n})^3 complex64 FFT, {B} volumes: {ms:.3f} ms per call, "
          f"{1e3 * ms / B:.1f} us per volume")
    return 0


CASES = {"shift": _shift, "search": _search, "fle": _fle, "prepare": _prepare, "reader": None, "graph": None,
         "fftbound": None}


def main(argv=None) -> int:
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("case", choices=sorted(CASES))
    p.add_argument("batch", type=int)
    p.add_argument("--reps", type=int, default=5)
    p.add_argument("--stages", action="store_true", help="shift only: time each kernel group with CUDA events")
    p.add_argument("--box", type=int, default=64, help="shift and fftbound: box size")
    p.add_argument("--radius", type=int, default=5, help="shift only: search radius (voxels)")
    p.add_argument("--precision", default="bf16x3", help="shift only: bf16x3, fp32 or auto")
    p.add_argument("--kernels", action="store_true",
                   help="time every kernel launch of the library with CUDA events (mtb_profile_*)")
    a = p.parse_args(argv)
    if a.case == "reader":
        return _reader(a.batch, a.reps)
    if not torch.cuda.is_available():
        print("a CUDA device is required", file=sys.stderr)
        return 2
    if a.case == "graph":
        return _graph(a.batch, a.reps)
    if a.case == "fftbound":
        return _fftbound(a.batch, a.reps, a.box)
    dev = torch.device("cuda:0")
    if a.case == "shift":
        run = _shift(a.batch, dev, a.box, a.radius, a.precision)
    else:
        run = CASES[a.case](a.batch, dev)
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    print(f"{a.case} batch {a.batch}: {e0.elapsed_time(e1) / a.reps:.3f} ms per call")
    sm = getattr(run, "matcher", None)
    if a.stages and sm is not None:
        sm.profile(a.reps)
        for _ in range(a.reps):
            run()
        torch.cuda.synchronize()
        ms, calls = sm.profile_read()
        sm.profile(0)
        print("  " + ", ".join(f"{k} {v / max(calls, 1):.3f}" for k, v in ms.items()) + " ms per call")
    if a.kernels:
        from matcha_b200 import _native

        _native.profile_start(4096)
        for _ in range(a.reps):
            run()
        table, dropped = _native.profile_read()
        _native.profile_stop()
        for name, row in sorted(table.items(), key=lambda kv: -kv[1]["ms"]):
            print(f"  {name}: {row['ms'] / a.reps:.3f} ms per call ({row['launches'] // a.reps} launches)")
        if dropped:
            print(f"  ({dropped} launches not timed: event pool full)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
