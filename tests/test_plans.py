"""Launch-geometry rules of the tensor-core shift match and of the SO(3) grid kernel, checked
on the host through their C-ABI queries (mtb_shift_tc_plan, mtb_so3_grid_plan; no device
needed): which boxes and upsampled regions the tensor-core kernels take, how the N-tile is cut
into column parts, and that every plan fits the shared memory and tensor memory it claims."""
import ctypes

import pytest

SMEM_CAP = 227 * 1024 - 2048  # the opt-in limit less the kernels' static barriers
GRID_CAP = 200 * 1024


def _lib():
    from matcha_b200 import _native as nat

    return nat.load()


def _shift_plan(N, U):
    lib = _lib()
    vals = [ctypes.c_int() for _ in range(5)]
    smem = ctypes.c_int64()
    rc = lib.mtb_shift_tc_plan(N, U, *[ctypes.byref(v) for v in vals], ctypes.byref(smem))
    if rc:
        return None
    fused, parts, nt, st1, st3 = (v.value for v in vals)
    return dict(fused=fused, parts=parts, nt=nt, stages1=st1, stages3=st3, smem=smem.value)


@pytest.mark.parametrize("N,U,fused,parts,nt", [(64, 88, 1, 1, 176), (32, 56, 1, 1, 112), (128, 136, 0, 2, 144),
                                                (96, 104, 0, 1, 208), (32, 248, 0, 2, 256), (64, 136, 0, 2, 144),
                                                (48, 2, 0, 1, 16), (64, 124, 0, 1, 256)])
def test_shift_plans_of_the_tested_shapes(N, U, fused, parts, nt):
    p = _shift_plan(N, U)
    assert p is not None
    assert (p["fused"], p["parts"], p["nt"]) == (fused, parts, nt)


@pytest.mark.parametrize("N,U", [(8, 12), (4, 8), (128, 264), (130, 88), (63, 88)])
def test_shift_plan_refuses_what_the_kernels_do_not_cover(N, U):
    assert _shift_plan(N, U) is None


def test_every_shift_plan_fits_its_budgets():
    """Every covered (N, U): the column parts cover 2U, each part's N-tile is a legal MMA width
    (multiple of 16, at most 256) whose double-buffered accumulator fits the 512 TMEM columns,
    at least two pipeline stages, and the shared memory within the opt-in limit."""
    boxes = [16, 32, 48, 64, 80, 96, 128]
    for N in boxes:
        for U in list(range(1, 40)) + list(range(40, 257, 7)) + [256]:
            p = _shift_plan(N, U)
            assert p is not None, (N, U)
            assert p["nt"] % 16 == 0 and p["nt"] <= 256, (N, U, p)
            assert p["parts"] * (p["nt"] // 2) >= U, (N, U, p)
            assert p["stages1"] >= 2 and (p["fused"] or p["stages3"] >= 2), (N, U, p)
            assert 2 * p["nt"] <= 512 or p["fused"], (N, U, p)
            assert p["smem"] <= SMEM_CAP, (N, U, p)
            if p["fused"]:
                assert N in (16, 32, 64) and 2 * U <= 256, (N, U, p)


def _grid_plan(L0, K):
    lib = _lib()
    jb, staged, smem = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64()
    rc = lib.mtb_so3_grid_plan(L0, K, ctypes.byref(jb), ctypes.byref(staged), ctypes.byref(smem))
    return None if rc else (jb.value, bool(staged.value), smem.value)


@pytest.mark.parametrize("L0,K,jb,staged", [(8, 2, 8, False), (12, 2, 2, False), (16, 2, 2, False)])
def test_grid_plans_of_the_benchmark_marches(L0, K, jb, staged):
    p = _grid_plan(L0, K)
    assert p is not None and p[:2] == (jb, staged)


def test_every_grid_plan_fits():
    for L0 in range(1, 21):
        for K in (1, 2):
            p = _grid_plan(L0, K)
            assert p is not None, (L0, K)
            assert p[0] in (1, 2, 4, 8) and p[2] <= GRID_CAP, (L0, K, p)


def test_capacity_plan_is_the_affine_fit_of_two_probes(monkeypatch):
    """matcha_b200.autotune.plan_capacity on the host logic alone: the step's memory measured at
    two capacities (here a stand-in of fixed + per-subtomogram bytes), the margin on the slope,
    the batch's own volumes added, and the largest capacity within the budget."""
    torch = pytest.importorskip("torch")
    from matcha_b200 import autotune
    from matcha_b200.pipeline import StepConfig

    fixed, per = 700_000_000, 3_000_000
    monkeypatch.setattr(autotune, "step_bytes", lambda cfg, cap, dev: fixed + per * cap)
    cfg = StepConfig(N=64, L=32, batch=128)
    plan = autotune.plan_capacity(cfg, "cpu", budget_bytes=20_000_000_000, probe=(128, 384), margin=1.1)
    slope = int(-(-1.1 * per // 1))  # ceil(margin x per)
    assert plan.bytes_per_subtomo == slope + 4 * 64 ** 3
    assert plan.bytes_fixed == fixed + per * 128 - slope * 128
    assert plan.capacity == (20_000_000_000 - plan.bytes_fixed) // plan.bytes_per_subtomo
    assert plan.bytes_fixed + plan.capacity * plan.bytes_per_subtomo <= 20_000_000_000
    del torch
