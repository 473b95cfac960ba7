"""The bench's multi-rank host logic, as two gloo ranks on the CPU.

Under torchrun every rank aligns its own batch (replicas: no data-path collective) and the
job's step time is the slowest rank's: ``bench.max_over_ranks`` is an all_reduce(MAX) of the
timing only, ``bench.whole_job_value`` the weak-scaling aggregate, and the reference arm runs on
rank 0 alone.  The same functions run here over ``gloo`` with world size 2.
"""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import bench

    w, r, loc = bench.dist_env()
    dist.init_process_group("gloo", rank=r, world_size=w)
    try:
        ms = [6.5, 7.25][r]  # the ranks' own step times
        mx = bench.max_over_ranks(ms, w, "cpu")
        dist.barrier()
        out.put((r, loc, w, mx, bench.whole_job_value(w, 1000, mx)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_value_with_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [g[0] for g in got] == [0, 1] and [g[1] for g in got] == [0, 1]
    for _, _, w, mx, value in got:
        assert w == 2 and mx == 7.25  # every rank sees the slowest rank's time
        assert value == pytest.approx(2 * 1000 / 7.25e-3)


def test_one_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.whole_job_value(1, 1000, 6.6) == pytest.approx(1000 / 6.6e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Rank 1 of a torchrun job returns at once, printing nothing (the driver reads rank 0's
    line); no host-core work is done there."""
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")

    class A:
        steps, warmup, cpu_sample, batch, seed = 1, 0, 1, 4, 0

    assert bench.run_reference(A()) is None
    assert capsys.readouterr().out == ""
