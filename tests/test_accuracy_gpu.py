"""Whole-path accuracy against the oracle on the same inputs, at the benchmark's shapes.

The reference's alternation loop (src/matcha/align_subtomograms.py:254-285, 316-361) is run
on identical seeded subtomograms on the GPU through ``AlignmentStep`` and on the CPU through
``oracle.pipeline`` (FP64 expansion), whose orientation search runs twice: in FP64 (the
exact answer) and in FP32, the arithmetic the reference's torch path uses.  The
small shape is 32^3 at L = 16 (march 4/8/12/16, shift radius 3, 16 subtomograms, 40-blob
template); the benchmark shape is 64^3 at L = 32 (march 8/16/24/32, shift radius 5, 8
subtomograms, 400-blob two-lobe template).  Both at 0 dB, upsample factor 8.

Checked per subtomogram, for the FP32 and the BF16 hi+lo (tensor-core) step:
  * sigma within 2e-5 (FP32) / 2e-4 (BF16 hi+lo) relative, bh_norms within 1e-5 / 1e-4;
  * rotations within 0.05 degrees (geodesic) of the FP64 oracle's, after one alternation
    and after each of three - except where the oracle's march ends with two distinct
    candidates whose scores agree to 1e-5 relative: then within 0.05 degrees of one of them;
  * shifts identical on the 1/uf grid, except where the oracle's own correlation grid has
    a near-tie (the GPU's pick within 1e-5 relative of the oracle's maximum);
  * near-ties are at most a quarter of the batch, and a subtomogram decided by one is not
    followed into the next alternation (its inputs differ from then on);
  * against the FP32 oracle (the reference's arithmetic): every deviation beyond 0.05 degrees
    is the FP32 oracle's own distance from the exact answer, dev(GPU, FP32) <= dev(FP64, FP32)
    + 0.05 degrees.  With one Newton step per march stage, accept/reject decisions whose
    score gain is below FP32 resolution move the FP32 result by up to a few tenths of a degree.
"""
import numpy as np
import pytest
import torch

from tests.helpers import blob_template, euler_dist_deg, make_subtomograms, quat_dist_deg

pytestmark = pytest.mark.gpu

CASES = {
    "32_L16": dict(N=32, L=16, Li=[4, 8, 12], B=16, r=3, uf=8, seed=101, max_shift=3.0,
                   blobs=dict(n_blobs=40, centre_radius=12, sigma_range=(1.5, 3.0), mask_radius=14)),
    "64_L32": dict(N=64, L=32, Li=[8, 16, 24], B=8, r=5, uf=8, seed=102, max_shift=5.0,
                   blobs=dict(n_blobs=400, centre_radius=None, sigma_range=(1.0, 2.5), mask_radius=0.45 * 64,
                              lobes=[(26.0, (-3.0, 1.0, 0.0)), (18.0, (6.0, -4.0, 3.0))])),
}
ROT_TOL_DEG = 0.05
TIE_REL = 1e-5


def _radius(N):
    return min(N // 2, int(N // 2 * 0.95))


@pytest.fixture(scope="module", params=list(CASES))
def case(request):
    """Inputs and the oracle's outputs (one alternation on the raw volumes, and three
    alternations with the preparation), computed once per shape."""
    from matcha_b200.core import fle_tables as T
    from oracle import fle as OF
    from oracle import pipeline as OP
    from oracle import shift as OS

    c = dict(CASES[request.param])
    rng = np.random.default_rng(c["seed"])
    tmpl = blob_template(rng, c["N"], **c["blobs"])
    vols, q, _ = make_subtomograms(tmpl, rng, c["B"], c["max_shift"])
    N, L, B, rad = c["N"], c["L"], c["B"], _radius(c["N"])
    tb = T.lap_eig_ball(N, L, rad)
    ff = OP.FoldedFLE(tb, N, float(rad))
    a_t = ff.evaluate_t(tmpl[None])[0]
    ref = OS.load_reference_full(tmpl, N, 1.0)
    ident = np.tile([1.0, 0, 0, 0], (B, 1))
    z3 = np.zeros((B, 3))
    v64 = vols.astype(np.float64)
    one = OP.align_batch(ff, a_t, ref, v64, v64, ident, z3, L, c["Li"], uf=c["uf"], shift_radius=c["r"],
                         dtype=np.float64)
    one32 = OP.align_batch(ff, a_t, ref, v64, v64, ident, z3, L, c["Li"], uf=c["uf"], shift_radius=c["r"],
                           dtype=np.float32)
    a_v = ff.evaluate_t(v64)
    sigma = OF.compute_sigma(tb, a_t, a_v)
    three = OP.run_alternations(ff, a_t, ref, vols, ident, z3, z3, z3, L, c["Li"], float(rad), 3, uf=c["uf"],
                                shift_radius=c["r"], dtype=np.float64)
    c.update(name=request.param, template=tmpl, vols=vols, q=q, oracle_one=one, oracle_one32=one32,
             oracle_three=three,
             oracle_sigma=sigma, oracle_norms=np.linalg.norm(a_v, axis=1), ref_fourier=ref, radius=rad)
    return c


def _step(c, dev, precision):
    from matcha_b200.pipeline import AlignmentStep, StepConfig

    step = AlignmentStep(StepConfig(N=c["N"], L=c["L"], Li=c["Li"], batch=c["B"], shift_search_radius=c["r"],
                                    shift_upsample_factor=c["uf"], precision=precision), dev)
    step.set_template(c["template"])
    return step


def _rotation_ok(gpu_angles, o, i):
    """(ok, tie).  The candidates of the oracle's march whose final scores are within TIE_REL of
    its best are the answers the last bits of an FP32 score sum can pick between; ``tie`` says
    that they hold two distinct rotations (more than a tenth of ROT_TOL_DEG apart).  ``ok``:
    subtomogram i's rotation is within ROT_TOL_DEG of one of them (of the oracle's own answer
    when there is no tie)."""
    a, b, g = (np.float64(x[i]) for x in gpu_angles)
    cand = o["candidates"]
    sc = np.asarray(cand["score"][i], dtype=np.float64)
    tied = np.nonzero(sc.max() - sc <= TIE_REL * abs(sc.max()))[0]
    ang = lambda c: (np.float64(cand["alpha"][i, c]), np.float64(cand["beta"][i, c]), np.float64(cand["gamma"][i, c]))
    best = (np.float64(o["alpha"][i]), np.float64(o["beta"][i]), np.float64(o["gamma"][i]))
    tie = any(euler_dist_deg(*ang(c), *best) > 0.1 * ROT_TOL_DEG for c in tied)
    d = min([euler_dist_deg(a, b, g, *best)] + [euler_dist_deg(a, b, g, *ang(c)) for c in tied])
    return bool(d < ROT_TOL_DEG), tie


def _shift_ok(c, gpu_shift, oracle_out, angles_deg_tracker, i):
    """(ok, tie): identical on the 1/uf grid, or the oracle's own correlation grid has a
    near-tie at the GPU's pick (within TIE_REL of its maximum)."""
    from oracle import shift as OS

    if np.abs(gpu_shift[i] - oracle_out["shift"][i]).max() <= 1e-6:
        return True, False
    prior = oracle_out.get("shift_prior", np.zeros((c["B"], 3)))[i]
    (_, _), parts = OS.estimate_shift_like_relion(c["ref_fourier"], c["vols"][i].astype(np.float64), prior,
                                                  angles_deg_tracker[i], c["uf"], c["r"], return_parts=True)
    grid = parts["grid"]
    U = grid.shape[0]
    idx = np.rint(gpu_shift[i][::-1] * c["uf"] + np.floor(U / 2.0)).astype(int)
    if not np.all((idx >= 0) & (idx < U)):
        return False, True
    return bool(grid.max() - grid[tuple(idx)] <= TIE_REL * abs(grid.max())), True


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_one_alternation_matches_oracle(cuda_device, case, precision):
    from matcha_b200.core.wigner_index import compute_size
    from oracle import shift as OS

    c = case
    B, L = c["B"], c["L"]
    step = _step(c, cuda_device, precision)
    dv = torch.from_numpy(c["vols"]).to(cuda_device)
    sig, norms = step.correlator.get_sigma_upto(dv, L)
    sig = sig[:B].cpu().numpy()
    ref_sig = c["oracle_sigma"][:, :compute_size(L + 1)]
    tol_s, tol_n = (2e-5, 1e-5) if precision == "fp32" else (2e-4, 1e-4)
    for i in range(B):
        assert np.linalg.norm(sig[i] - ref_sig[i]) / np.linalg.norm(ref_sig[i]) < tol_s, i
    np.testing.assert_allclose(norms[:B].cpu().numpy(), c["oracle_norms"], rtol=tol_n)
    tracker = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    tracker[:, 0] = 1
    out = step(dv, dv, tracker, torch.zeros((B, 3), device=cuda_device))
    o, o32 = c["oracle_one"], c["oracle_one32"]
    ang = lambda d: [np.asarray(d[k], dtype=np.float64) for k in ("alpha", "beta", "gamma")]
    gpu = ang({k: out[k].cpu().numpy() for k in ("alpha", "beta", "gamma")})
    dev64 = euler_dist_deg(*gpu, *ang(o))
    dev32 = euler_dist_deg(*gpu, *ang(o32))
    ref_own = euler_dist_deg(*ang(o), *ang(o32))
    print(f"{c['name']} {precision} one alternation: deviation from the FP64 oracle max {dev64.max():.5f} deg "
          f"(median {np.median(dev64):.6f}), from the FP32 oracle max {dev32.max():.4f} deg (median "
          f"{np.median(dev32):.5f}, {np.mean(dev32 < ROT_TOL_DEG):.3f} within {ROT_TOL_DEG}); FP32 oracle vs FP64 "
          f"max {ref_own.max():.4f}")
    ties = 0
    rot_tie = np.zeros(B, dtype=bool)
    gpu_shift = out["shift"].cpu().numpy()
    ang_o = OS.euler_zyz_deg_from_quat_conj(o["tracker"])
    for i in range(B):
        ok, tie = _rotation_ok(gpu, o, i)
        assert ok, (i, dev64[i])
        ties += tie
        rot_tie[i] = tie
        if not tie:
            ok, stie = _shift_ok(c, gpu_shift, o, ang_o, i)
            assert ok, (i, gpu_shift[i], o["shift"][i])
            ties += stie
            if not stie:
                np.testing.assert_allclose(out["shift_score"][i].item(), o["shift_score"][i], rtol=1e-3)
    assert ties <= max(1, B // 4), ties
    # away from the near-ties, the FP32 oracle differs from the exact answer by more than the
    # GPU path does
    keep = ~rot_tie
    assert np.all(dev32[keep] <= ref_own[keep] + ROT_TOL_DEG), (dev32, ref_own)


@pytest.mark.parametrize("precision", ["fp32", "bf16x3"])
def test_three_alternations_match_oracle(cuda_device, case, precision):
    """Three alternations with the preparation; a subtomogram whose rotation or shift went the
    other way of a near-tie is followed no further (its next inputs differ)."""
    from oracle import shift as OS

    c = case
    B = c["B"]
    step = _step(c, cuda_device, precision)
    dv = torch.from_numpy(c["vols"]).to(cuda_device)
    tracker = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    tracker[:, 0] = 1
    z = torch.zeros((B, 3), device=cuda_device)
    outs = step.run_alternations(dv, tracker, z.clone(), z, z, 3)
    followed = np.ones(B, dtype=bool)
    for k, (g, o) in enumerate(zip(outs, c["oracle_three"])):
        gpu = [g[x].cpu().numpy().astype(np.float64) for x in ("alpha", "beta", "gamma")]
        dev = quat_dist_deg(g["tracker"].cpu().numpy(), o["tracker"])
        print(f"{c['name']} {precision} alternation {k + 1}: max tracker deviation "
              f"{dev[followed].max():.4f} deg over {followed.sum()} subtomograms")
        shift = g["shift"].cpu().numpy()
        ang_o = OS.euler_zyz_deg_from_quat_conj(o["tracker"])
        loc = g["local_shifts"].cpu().numpy()
        for i in np.nonzero(followed)[0]:
            ok, tie = _rotation_ok(gpu, o, i)
            assert ok, (k, i, dev[i])
            if tie:
                followed[i] = False
                continue
            assert dev[i] < ROT_TOL_DEG, (k, i, dev[i])
            ok, tie = _shift_ok(c, shift, o, ang_o, i)
            assert ok, (k, i, shift[i], o["shift"][i])
            if tie:
                followed[i] = False
                continue
            np.testing.assert_allclose(loc[i], o["local_shifts"][i], atol=1e-5)
    assert followed.sum() >= B - max(1, B // 4), followed
