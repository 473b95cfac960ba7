"""The C-ABI library loads and exports every entry point include/*.h declares (no GPU needed)."""
import ctypes
import glob
import os
import re

from matcha_b200 import _native


def declared_symbols():
    names = set()
    for path in glob.glob(os.path.join(_native._build.ROOT, "include", "*.h")):
        text = open(path, encoding="utf-8").read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(mtb_[a-z0-9_]+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert {"mtb_search_create", "mtb_search_orientations", "mtb_version"} <= names


def test_library_exports_every_declared_symbol():
    lib = _native.load(build_if_missing=True)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(declared_symbols()) <= set(_native.SIGNATURES), "ctypes signatures missing"
    assert lib.mtb_version() >= 100


def test_bad_arguments_are_rejected_without_gpu_work():
    lib = _native.load()
    out = ctypes.c_void_p()
    assert lib.mtb_search_create(None, ctypes.byref(out)) == _native.MTB_ERR_ARG
    cfg = _native.MtbSearchConfig()
    cfg.Lmax = 0  # invalid
    assert lib.mtb_search_create(ctypes.byref(cfg), ctypes.byref(out)) == _native.MTB_ERR_ARG
    assert b"Lmax" in lib.mtb_last_error()
