"""The allocation-free orientation search against the handle-based one, through the C ABI.

mtb_search_orientations_static serves callers that cannot allocate device memory (a host
program that owns all device memory through its own allocator or a fixed budget, or a
pipeline that cannot afford the device-wide synchronisation of cudaMalloc/cudaFree).  Its
tables and workspace live in a library-owned device array; this test checks that two calls
in a row give the same orientations and scores as mtb_search_orientations.  The file sorts
last so that a run stopping at the first failure has run every other test already.
"""
import ctypes

import numpy as np
import pytest
import torch

from tests.helpers import euler_dist_deg, synthetic_sigma

pytestmark = pytest.mark.gpu


def _cfg(native, Lmax, stages, L0, C, steps, B, flags=0):
    cfg = native.MtbSearchConfig()
    cfg.Lmax, cfg.n_stages, cfg.L0, cfg.K = Lmax, len(stages), L0, 2
    for i, l in enumerate(stages):
        cfg.stages[i] = l
    cfg.candidates, cfg.num_steps, cfg.max_batch, cfg.flags = C, steps, B, flags
    return cfg


def _run(lib, native, fn, first_arg, sig, B):
    out = torch.empty((4, B), device=sig.device, dtype=torch.float32)
    rc = fn(first_arg, native.ptr(sig), sig.stride(0), B, native.ptr(out[0]), native.ptr(out[1]), native.ptr(out[2]),
            native.ptr(out[3]), native.stream_ptr(sig.device))
    assert rc == 0, lib.mtb_last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("flag", ["none", "compat_top_block", "gradient_step"])
def test_static_search_matches_handle_search_twice(cuda_device, flag):
    from matcha_b200 import _native as native

    lib = native.load()
    flags = {"none": 0, "compat_top_block": native.MTB_SEARCH_COMPAT_TOP_BLOCK,
             "gradient_step": native.MTB_SEARCH_GRADIENT_STEP}[flag]
    B, Lmax, stages, C = 24, 16, [4, 8, 12, 16], 10
    rng = np.random.default_rng(2024)
    sig_np, _ = synthetic_sigma(rng, B, Lmax)
    sig = torch.from_numpy(sig_np).to(cuda_device)
    cfg = _cfg(native, Lmax, stages, 4, C, 1, B, flags)
    h = ctypes.c_void_p()
    assert lib.mtb_search_create(ctypes.byref(cfg), ctypes.byref(h)) == 0, lib.mtb_last_error()
    try:
        ref = _run(lib, native, lib.mtb_search_orientations, h, sig, B)
    finally:
        lib.mtb_search_destroy(h)
    for call in range(2):
        got = _run(lib, native, lib.mtb_search_orientations_static, ctypes.byref(cfg), sig, B)
        d = euler_dist_deg(got[0], got[1], got[2], ref[0], ref[1], ref[2])
        assert np.all(d < 0.05), (call, d)
        np.testing.assert_allclose(got[3], ref[3], rtol=0, atol=2e-5 * np.abs(ref[3]).max())


def test_static_search_rejects_oversized_batch(cuda_device):
    from matcha_b200 import _native as native

    lib = native.load()
    B = 400_000  # 4 x B x 10 floats exceed the 4 MiB array
    cfg = _cfg(native, 8, [4, 8], 4, 10, 1, B)
    dummy = torch.zeros((1, 1000), dtype=torch.complex64, device=cuda_device)
    out = torch.zeros(4, device=cuda_device)
    rc = lib.mtb_search_orientations_static(ctypes.byref(cfg), native.ptr(dummy), 1000, B, native.ptr(out),
                                            native.ptr(out), native.ptr(out), native.ptr(out),
                                            native.stream_ptr(cuda_device))
    assert rc == native.MTB_ERR_ARG
    assert b"static scratch" in lib.mtb_last_error()
