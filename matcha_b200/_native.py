"""ctypes binding of the matcha_b200 C ABI (include/matcha_b200.h).

The library is the product's only compute path: importing this module on a machine
without the built library, or calling an entry point without a CUDA device, raises
instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

import torch

from . import build as _build

MTB_OK = 0
MTB_ERR_ARG = 1
MTB_ERR_OOM = 2
MTB_ERR_NUMERIC = 3
MTB_ERR_TIMEOUT = 4
MTB_ERR_CUDA = 5

MTB_MAX_STAGES = 16
MTB_FLE_FP32 = 0
MTB_FLE_BF16X3 = 1
MTB_FLE_BF16_SPLIT = 2
MTB_SHIFT_FP32 = 0
MTB_SHIFT_BF16X3 = 1
MTB_SHIFT_AUTO = 2
MTB_SEARCH_COMPAT_TOP_BLOCK = 1
MTB_SEARCH_GRADIENT_STEP = 2

_lib = None


class MtbSearchConfig(ctypes.Structure):
    _fields_ = [
        ("Lmax", ctypes.c_int),
        ("n_stages", ctypes.c_int),
        ("stages", ctypes.c_int * MTB_MAX_STAGES),
        ("L0", ctypes.c_int),
        ("K", ctypes.c_int),
        ("candidates", ctypes.c_int),
        ("num_steps", ctypes.c_int),
        ("max_batch", ctypes.c_int),
        ("flags", ctypes.c_int),
    ]


class MtbFleConfig(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("max_batch", ctypes.c_int), ("ne", ctypes.c_int), ("n_rep", ctypes.c_int),
        ("n_cols", ctypes.c_int), ("lmax", ctypes.c_int), ("n_lk", ctypes.c_int), ("n_r2", ctypes.c_int),
        ("rep_img", ctypes.c_void_p), ("rep_cos", ctypes.c_void_p), ("rep_phi", ctypes.c_void_p),
        ("rep_r2", ctypes.c_void_p), ("jtab", ctypes.c_void_p), ("col_class", ctypes.c_void_p),
        ("col_l", ctypes.c_void_p), ("col_m", ctypes.c_void_p), ("col_part", ctypes.c_void_p),
        ("col_lk", ctypes.c_void_p), ("col_scale", ctypes.c_void_p), ("coef_col_re", ctypes.c_void_p),
        ("coef_col_im", ctypes.c_void_p), ("coef_sign_re", ctypes.c_void_p), ("coef_sign_im", ctypes.c_void_p),
        ("kpad", ctypes.c_void_p), ("kidx", ctypes.c_void_p), ("precision", ctypes.c_int),
        ("split_degree", ctypes.c_int),
    ]


class MtbShiftConfig(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("max_batch", ctypes.c_int), ("upsample_factor", ctypes.c_int),
        ("search_radius", ctypes.c_int), ("mask_radius", ctypes.c_float), ("cosine_width", ctypes.c_float),
        ("precision", ctypes.c_int), ("tile_rows", ctypes.c_int),
    ]


_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64

# name -> (restype, argtypes); every symbol declared in include/matcha_b200.h
SIGNATURES = {
    "mtb_version": (_I, []),
    "mtb_last_error": (ctypes.c_char_p, []),
    "mtb_search_create": (_I, [ctypes.POINTER(MtbSearchConfig), ctypes.POINTER(_P)]),
    "mtb_search_destroy": (None, [_P]),
    "mtb_so3_grid_topk": (_I, [_P, _P, _I64, _I, _P, _P, _P, _P, _P]),
    "mtb_newton_march": (_I, [_P, _P, _I64, _I, _P, _P, _P, _P, _P]),
    "mtb_score_derivatives": (_I, [_P, _P, _I64, _I, _I, _P, _P, _P, _P, _P]),
    "mtb_search_orientations": (_I, [_P, _P, _I64, _I, _P, _P, _P, _P, _P]),
    "mtb_search_orientations_static": (_I, [ctypes.POINTER(MtbSearchConfig), _P, _I64, _I, _P, _P, _P, _P, _P]),
    "mtb_fle_create": (_I, [ctypes.POINTER(MtbFleConfig), ctypes.POINTER(_P)]),
    "mtb_fle_destroy": (None, [_P]),
    "mtb_fle_forward": (_I, [_P, _P, _I, _P, _I64, _P, _P]),
    "mtb_sigma": (_I, [_P, _P, _I64, _P, _I, _P, _I64, _P]),
    "mtb_sigma_upto": (_I, [_P, _P, _I64, _P, _I, _I, _P, _I64, _P]),
    "mtb_fle_status": (_I, [_P, _P]),
    "mtb_fle_inject_stall": (_I, [_P, _I]),
    "mtb_fle_split_tiles": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "mtb_sigma_backward_template": (_I, [_P, _P, _I64, _P, _I64, _I, _I, _P, _P]),
    "mtb_score_backward": (_I, [_P, _I64, _I, _I, _P, _P, _P, _P, _P, _I64, _P, _P]),
    "mtb_shift_create": (_I, [ctypes.POINTER(MtbShiftConfig), ctypes.POINTER(_P)]),
    "mtb_shift_destroy": (None, [_P]),
    "mtb_shift_set_reference": (_I, [_P, _P, _P]),
    "mtb_shift_status": (_I, [_P, _P]),
    "mtb_shift_precision": (_I, [_P, _P]),
    "mtb_shift_score_grad": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _P, _P]),
    "mtb_shift_profile": (_I, [_P, _I]),
    "mtb_shift_profile_read": (_I, [_P, _P, _P]),
    "mtb_shift_search": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _P]),
    "mtb_shift_begin": (_I, [_P, _P, _P, _I, _P]),
    "mtb_shift_tc_plan": (_I, [_I, _I] + [ctypes.POINTER(_I)] * 5 + [ctypes.POINTER(_I64)]),
    "mtb_so3_grid_plan": (_I, [_I, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I64)]),
    "mtb_shift_finish": (_I, [_P, _P, _P, _I, _P, _P, _P]),
    "mtb_update_rotation": (_I, [_P, _P, _P, _P, _I, _P, _P, _P]),
    "mtb_tracker_rotation": (_I, [_P, _I, _P, _P]),
    "mtb_shift_reference": (_I, [_P, _I, ctypes.c_float, _P, _P, _P]),
    "mtb_reader_create": (_I, [_I, _P]),
    "mtb_reader_destroy": (_I, [_P]),
    "mtb_read_mrc": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P]),
    "mtb_pack_results": (_I, [_P, _P, _P, _P, _P, _I, _P, _P]),
    "mtb_prepare_subtomos": (_I, [_P, _I, _I, _P, _P, ctypes.c_float, _P, _P, _P, _P]),
    "mtb_profile_start": (_I, [_I]),
    "mtb_profile_stop": (_I, []),
    "mtb_profile_read": (_I, [_I, _P, _P, _P, _P, _P]),
}
MTB_PROFILE_NAME_LEN = 64


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = False):
    """Load the shared library (optionally building it first) and declare its symbols."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not os.path.exists(path):
        if build_if_missing:
            _build.build()
        else:
            raise RuntimeError(
                f"matcha_b200 CUDA library not found at {path}; build it with `python -m matcha_b200.build`")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    """Map a C status to the exception type the reference's callers expect."""
    if rc == MTB_OK:
        return
    msg = load().mtb_last_error().decode(errors="replace")
    text = f"{what} failed (status {rc}): {msg}"
    if rc == MTB_ERR_OOM:
        raise torch.cuda.OutOfMemoryError("CUDA out of memory. " + text)
    if rc == MTB_ERR_ARG:
        raise ValueError(text)
    raise RuntimeError(text)


def stream_ptr(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor: matcha_b200 runs on the GPU only")


def profile_start(max_launches: int) -> None:
    """Switch on the library's launch timing (``mtb_profile_start``): every hot-path kernel
    launch from now on is bracketed by CUDA events on its stream, up to ``max_launches``."""
    check(load().mtb_profile_start(int(max_launches)), "mtb_profile_start")


def profile_stop() -> None:
    check(load().mtb_profile_stop(), "mtb_profile_stop")


def profile_read(max_entries: int = 64) -> tuple[dict, int]:
    """Per kernel name, in first-launch order: {"ms": summed device time, "launches": n};
    and the number of launches that found the event pool full.  Synchronises."""
    names = ctypes.create_string_buffer(max_entries * MTB_PROFILE_NAME_LEN)
    ms = (ctypes.c_float * max_entries)()
    launches = (ctypes.c_int * max_entries)()
    n, dropped = ctypes.c_int(0), ctypes.c_int(0)
    check(load().mtb_profile_read(max_entries, names, ms, launches, ctypes.byref(n), ctypes.byref(dropped)),
          "mtb_profile_read")
    out = {}
    for k in range(n.value):
        raw = names.raw[k * MTB_PROFILE_NAME_LEN:(k + 1) * MTB_PROFILE_NAME_LEN]
        out[raw.split(b"\0", 1)[0].decode()] = {"ms": float(ms[k]), "launches": int(launches[k])}
    return out, int(dropped.value)
