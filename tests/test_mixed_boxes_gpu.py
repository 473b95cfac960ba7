"""Boxes that are not powers of two (48 and 96: radix-6 / radix-12 x 8 FFTs in the shift match;
80: direct DFTs) through the whole alternation, against the oracle at 48^3; the mixed-box batch of
matcha_b200.mixed against per-box steps, eager and as one captured graph; the capacity
planner of matcha_b200.autotune against the memory a step really holds."""
import numpy as np
import pytest
import torch

from tests.helpers import blob_template, euler_dist_deg, make_subtomograms

pytestmark = pytest.mark.gpu


def test_box48_alternation_matches_oracle(cuda_device):
    from matcha_b200.core import fle_tables as T
    from matcha_b200.pipeline import AlignmentStep, StepConfig
    from oracle import pipeline as OP
    from oracle import shift as OS

    N, L, Li, B, r = 48, 24, [6, 12, 18], 4, 4
    rng = np.random.default_rng(48)
    tmpl = blob_template(rng, N, 150, 14, (1.0, 2.5), mask_radius=0.45 * N)
    vols, q, _ = make_subtomograms(tmpl, rng, B, 3.0)
    rad = min(N // 2, int(N // 2 * 0.95))
    step = AlignmentStep(StepConfig(N=N, L=L, Li=Li, batch=B, shift_search_radius=r, shift_upsample_factor=8,
                                    precision="fp32"), cuda_device)
    step.set_template(tmpl)
    assert step.shifter.effective_precision == "fp32"
    dv = torch.from_numpy(vols).to(cuda_device)
    tracker = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    tracker[:, 0] = 1
    out = step(dv, dv, tracker, torch.zeros((B, 3), device=cuda_device))
    tb = T.lap_eig_ball(N, L, rad)
    ff = OP.FoldedFLE(tb, N, float(rad))
    o = OP.align_batch(ff, ff.evaluate_t(tmpl[None])[0], OS.load_reference_full(tmpl, N, 1.0),
                       vols.astype(np.float64), vols.astype(np.float64), np.tile([1.0, 0, 0, 0], (B, 1)),
                       np.zeros((B, 3)), L, Li, uf=8, shift_radius=r, dtype=np.float64)
    d = euler_dist_deg(*(out[k].cpu().numpy().astype(np.float64) for k in ("alpha", "beta", "gamma")),
                       o["alpha"], o["beta"], o["gamma"])
    assert np.median(d) < 0.01 and np.all(d < 0.2), d
    np.testing.assert_allclose(out["bh_norms"].cpu().numpy(), o["bh_norms"], rtol=1e-5)
    same = np.all(np.abs(out["shift"].cpu().numpy() - o["shift"]) < 1e-6, axis=1)
    assert same.sum() >= B - 1, (out["shift"].cpu().numpy(), o["shift"])
    np.testing.assert_allclose(out["shift_score"].cpu().numpy()[same], o["shift_score"][same], rtol=1e-3)


def _specs():
    from matcha_b200.mixed import BoxSpec
    from matcha_b200.pipeline import StepConfig

    rng = np.random.default_rng(7)
    t32 = blob_template(rng, 32, 40, 10, (1.5, 3.0), mask_radius=14)
    t48 = blob_template(rng, 48, 150, 14, (1.0, 2.5), mask_radius=0.45 * 48)
    return [BoxSpec(StepConfig(N=32, L=16, Li=[4, 8, 12], batch=6, shift_search_radius=3), t32),
            BoxSpec(StepConfig(N=48, L=24, Li=[6, 12, 18], batch=5, shift_search_radius=4, precision="fp32"), t48)], rng


def test_mixed_alignment_per_box_and_as_one_graph(cuda_device):
    from matcha_b200.mixed import MixedAlignment
    from matcha_b200.pipeline import AlignmentStep

    specs, rng = _specs()
    mixed = MixedAlignment(specs, cuda_device, tune=True)
    # the tuner timed tiles for the FP32 shift of box 48 only (box 32 runs the tensor cores; box 48
    # is configured for the FP32 kernels here so that there is something to tune)
    assert mixed.boxes[32][0].timings == {} and len(mixed.boxes[48][0].timings) >= 2
    counts = {32: 6, 48: 5}
    inputs = {}
    for spec in specs:
        N = spec.cfg.N
        vols, _, _ = make_subtomograms(spec.template, rng, counts[N], 2.0)
        inputs[N] = torch.from_numpy(vols).to(cuda_device)
    ident = {N: torch.tensor([[1.0, 0, 0, 0]] * B, dtype=torch.float64, device=cuda_device) for N, B in counts.items()}
    z = {N: torch.zeros((B, 3), device=cuda_device) for N, B in counts.items()}
    eager = mixed({N: (inputs[N], ident[N].clone(), z[N]) for N in counts})
    eager = {N: {k: v.clone() for k, v in o.items()} for N, o in eager.items()}
    keys = ("alpha", "beta", "gamma", "rotation_score", "shift", "shift_score")
    for spec in specs:  # an AlignmentStep of the same configuration gives the same answers
        N = spec.cfg.N
        step = AlignmentStep(mixed.boxes[N][0].cfg, cuda_device)
        step.set_template(spec.template)
        ref = step(inputs[N], inputs[N], ident[N].clone(), z[N])
        for k in keys:
            np.testing.assert_allclose(eager[N][k].cpu().numpy(), ref[k].cpu().numpy(), rtol=1e-6, atol=1e-7)
    cap = mixed.capture(counts)
    for N in counts:
        cap.volumes[N].copy_(inputs[N])
    cap.restore()
    out = cap.replay()
    for N in counts:
        for k in keys:
            np.testing.assert_allclose(out[N][k].cpu().numpy(), eager[N][k].cpu().numpy(), rtol=1e-6, atol=1e-7,
                                       err_msg=f"{N} {k}")


def test_plan_capacity_stays_within_budget(cuda_device):
    from dataclasses import replace

    from matcha_b200 import autotune
    from matcha_b200.pipeline import StepConfig

    cfg = StepConfig(N=32, L=16, Li=[4, 8, 12], batch=1, shift_search_radius=3)
    budget = 3 * 1024 ** 3
    plan = autotune.plan_capacity(cfg, cuda_device, budget_bytes=budget)
    assert plan.bytes_per_subtomo > 4 * 32 ** 3 and plan.capacity > 384
    used = autotune.step_bytes(replace(cfg, batch=plan.capacity), plan.capacity, cuda_device)
    assert used + plan.capacity * 4 * 32 ** 3 <= budget * 1.05, (used, plan)
