"""AlignmentStep: the host-input entry (pipelined copies) against the device-input step."""
import numpy as np
import pytest
import torch

from tests.helpers import blob_template

pytestmark = pytest.mark.gpu


def _step(dev, B):
    from matcha_b200.pipeline import AlignmentStep, StepConfig

    return AlignmentStep(StepConfig(N=16, L=12, Li=[4, 8], batch=B, radius=7, shift_search_radius=1,
                                    shift_upsample_factor=4), dev)


@pytest.mark.parametrize("chunks", [1, 3, 8])
def test_align_host_matches_device_step(cuda_device, chunks):
    B, N = 6, 16
    rng = np.random.default_rng(11)
    tmpl = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    vols = (np.repeat(tmpl[None], B, 0) + 0.05 * rng.standard_normal((B, N, N, N))).astype(np.float32)
    step = _step(cuda_device, B)
    step.set_template(tmpl)
    ident = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    ident[:, 0] = 1
    zeros3 = torch.zeros((B, 3), device=cuda_device)

    t_dev = ident.clone()
    dv = torch.from_numpy(vols).to(cuda_device)
    ref = {k: v.clone() for k, v in step(dv, dv, t_dev, zeros3).items()}
    torch.cuda.synchronize()

    host = torch.from_numpy(vols).pin_memory()
    for _ in range(2):  # the second call reuses the staging buffer
        t_host = ident.clone()
        out = step.align_host(host, t_host, zeros3, chunks=chunks)
        torch.cuda.synchronize()
        assert out["tracker"] is t_host
        for k in ("alpha", "beta", "gamma", "rotation_score", "bh_norms", "shift", "shift_score"):
            np.testing.assert_allclose(out[k].cpu().numpy(), ref[k].cpu().numpy(), rtol=1e-5, atol=1e-6,
                                       err_msg=k)
        np.testing.assert_allclose(t_host.cpu().numpy(), t_dev.cpu().numpy(), atol=1e-6)


def test_align_host_back_to_back_calls(cuda_device):
    """Three calls without a host synchronisation in between, on two different batches:
    the third reuses the first call's staging buffer while the second may still run."""
    B, N = 5, 16
    rng = np.random.default_rng(12)
    tmpl = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    batches = [(np.repeat(tmpl[None], B, 0) + s * rng.standard_normal((B, N, N, N))).astype(np.float32)
               for s in (0.05, 0.2)]
    step = _step(cuda_device, B)
    step.set_template(tmpl)
    ident = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    ident[:, 0] = 1
    zeros3 = torch.zeros((B, 3), device=cuda_device)
    keys = ("alpha", "beta", "gamma", "rotation_score", "shift", "shift_score")
    refs = []
    for v in batches:
        dv = torch.from_numpy(v).to(cuda_device)
        refs.append({k: t.clone() for k, t in step(dv, dv, ident.clone(), zeros3).items()})
    hosts = [torch.from_numpy(v).pin_memory() for v in batches]
    outs = []
    for i in (0, 1, 0):
        o = step.align_host(hosts[i], ident.clone(), zeros3, chunks=2)
        outs.append((i, {k: o[k].clone() for k in keys}))
    torch.cuda.synchronize()
    for i, o in outs:
        for k in keys:
            np.testing.assert_allclose(o[k].cpu().numpy(), refs[i][k].cpu().numpy(), rtol=1e-5, atol=1e-6,
                                       err_msg=k)


def test_align_host_rejects_oversize_batch(cuda_device):
    step = _step(cuda_device, 2)
    host = torch.zeros((3, 16, 16, 16)).pin_memory()
    with pytest.raises(ValueError):
        step.align_host(host, torch.zeros((3, 4), dtype=torch.float64, device=cuda_device),
                        torch.zeros((3, 3), device=cuda_device))


@pytest.mark.parametrize("alternations", [0, 2])
def test_captured_step_matches_eager(cuda_device, alternations):
    """One CUDA graph replayed on two different batches gives what the eager calls give."""
    B, N = 4, 16
    rng = np.random.default_rng(40 + alternations)
    tmpl = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    step = _step(cuda_device, B)
    step.set_template(tmpl)
    cap = step.capture(B, alternations)
    ident = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    ident[:, 0] = 1
    zeros3 = torch.zeros((B, 3), device=cuda_device)
    keys = ("alpha", "beta", "gamma", "rotation_score", "shift", "shift_score")
    for trial in range(2):
        vols = (np.repeat(tmpl[None], B, 0) + (0.05 + 0.1 * trial) * rng.standard_normal((B, N, N, N)))
        dv = torch.from_numpy(vols.astype(np.float32)).to(cuda_device)
        cap.volumes.copy_(dv)
        cap.tracker.copy_(ident)
        if alternations:
            cap.local_shifts.zero_()
        out = cap.replay()
        outs = [out] if alternations == 0 else out
        got = [{k: o[k].cpu().numpy().copy() for k in keys} for o in outs]
        got_tracker = cap.tracker.cpu().numpy().copy()
        t = ident.clone()
        if alternations == 0:
            ref = [step(dv, dv, t, zeros3)]
        else:
            ref = step.run_alternations(dv, t, torch.zeros_like(zeros3), zeros3, zeros3, alternations)
        assert len(ref) == len(got)
        for g, r in zip(got, ref):
            for k in keys:
                np.testing.assert_allclose(g[k], r[k].cpu().numpy(), rtol=1e-6, atol=1e-7, err_msg=k)
        np.testing.assert_allclose(got_tracker, t.cpu().numpy(), atol=1e-12)


def test_captured_step_after_set_template(cuda_device):
    """A template changed after capture is what the next replay uses (set_template writes the
    coefficients, the norm and the shift reference in place)."""
    B, N = 3, 16
    rng = np.random.default_rng(77)
    t1 = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    t2 = blob_template(rng, N, 12, 5, (1.0, 2.0), mask_radius=7).astype(np.float32)
    step = _step(cuda_device, B)
    step.set_template(t1)
    cap = step.capture(B, 0)
    step.set_template(t2)
    ident = torch.zeros((B, 4), dtype=torch.float64, device=cuda_device)
    ident[:, 0] = 1
    vols = (np.repeat(t2[None], B, 0) + 0.05 * rng.standard_normal((B, N, N, N))).astype(np.float32)
    dv = torch.from_numpy(vols).to(cuda_device)
    cap.volumes.copy_(dv)
    cap.tracker.copy_(ident)
    out = cap.replay()
    keys = ("alpha", "beta", "gamma", "rotation_score", "shift", "shift_score")
    got = {k: out[k].cpu().numpy().copy() for k in keys}
    ref = step(dv, dv, ident.clone(), torch.zeros((B, 3), device=cuda_device))
    for k in keys:
        np.testing.assert_allclose(got[k], ref[k].cpu().numpy(), rtol=1e-6, atol=1e-7, err_msg=k)
