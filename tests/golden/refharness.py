"""Load the reference's own Python modules on the CPU, for fixture generation only.

The reference (swing-research/Matcha) depends on packages that are not installed
here (cufinufft, torch_harmonics, spherical, quaternionic, ml_collections, mrcfile,
starfile) and its Wigner-D code is Numba CUDA.  This helper

* sets ``NUMBA_ENABLE_CUDASIM=1`` so the reference's ``@cuda.jit`` kernels run in
  Numba's CPU simulator,
* installs small stand-in modules for the missing imports,
* loads ``matcha.core.WignerDMatrices`` from the reference source with one
  simulator-only substitution applied in memory (numpy bool subtraction in
  ``_complex_powers_cuda`` and ``_complex_powers_and_conjugate_cuda``;
  WignerDMatrices.py:470,548), and pads the
  step-4 range tables with one empty range so the simulator does not raise on the
  read past their end (WignerDMatrices.py:776-789).

It reads the reference tree at fixture-generation time and is never imported by the
product, the GPU tests or the benchmark.  Nothing is copied to disk.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

# must be set before numba is first imported
os.environ["NUMBA_ENABLE_CUDASIM"] = "1"

REF_ROOT = os.environ.get("MATCHA_REFERENCE_ROOT")
if not REF_ROOT:
    raise RuntimeError("set MATCHA_REFERENCE_ROOT to a checkout of swing-research/Matcha to generate fixtures")
REF_SRC = os.path.join(REF_ROOT, "src")


class _ConfigDict(dict):
    """Attribute-access dict standing in for ml_collections.ConfigDict."""

    def __init__(self, *a, type_safe=False, **k):
        super().__init__(*a, **k)

    def __getattr__(self, name):
        try:
            return self[name]
        except KeyError as exc:  # pragma: no cover
            raise AttributeError(name) from exc

    def __setattr__(self, name, value):
        self[name] = value


def _install_stubs():
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    if "ml_collections" not in sys.modules:
        mc = types.ModuleType("ml_collections")
        mc.ConfigDict = _ConfigDict
        sys.modules["ml_collections"] = mc
    for name in ("quaternionic", "spherical", "mrcfile", "starfile", "cufinufft", "torch_harmonics"):
        if name not in sys.modules:
            sys.modules[name] = types.ModuleType(name)
    if REF_SRC not in sys.path:
        sys.path.insert(0, REF_SRC)


def load_wigner_module():
    """Return the reference WignerDMatrices module running under the Numba simulator."""
    _install_stubs()
    if "matcha.core.WignerDMatrices" in sys.modules:
        return sys.modules["matcha.core.WignerDMatrices"]
    import numba.cuda as nc

    path = os.path.join(REF_SRC, "matcha", "core", "WignerDMatrices.py")
    with open(path, encoding="utf-8") as fh:
        src = fh.read()
    bad = "((z_imag > 0) - (z_imag < 0))"
    assert src.count(bad) == 2, "reference source changed; update the simulator patch"
    src = src.replace(bad, "(float(z_imag > 0) - float(z_imag < 0))")
    # numba.njit(cache=True) cannot cache code compiled from a string
    src = src.replace("functools.partial(numba.njit, cache=True)", "functools.partial(numba.njit, cache=False)")
    nc.as_cuda_array = lambda t: t.numpy()
    mod = types.ModuleType("matcha.core.WignerDMatrices")
    mod.__file__ = path
    sys.modules["matcha.core.WignerDMatrices"] = mod
    exec(compile(src, path, "exec"), mod.__dict__)
    return mod


def make_reference_wigner(ell_max, batchsize, num_candidates):
    """Construct a reference WignerDMatrices on CPU with the step-4 tables padded."""
    import numpy as np
    import torch
    from numba import cuda

    mod = load_wigner_module()
    cwd = os.getcwd()
    # the reference caches index tables under ./data; keep them out of the repo
    tmp = os.path.join("/tmp", "matcha_ref_cache")
    os.makedirs(tmp, exist_ok=True)
    os.chdir(tmp)
    try:
        w = mod.WignerDMatrices(ell_max=ell_max, batchsize=batchsize, num_candidates=num_candidates,
                                device=torch.device("cpu"))
    finally:
        os.chdir(cwd)
    s4 = np.asarray(w.start_indices_4.copy_to_host() if hasattr(w.start_indices_4, "copy_to_host") else w.start_indices_4)
    e4 = np.asarray(w.end_indices_4.copy_to_host() if hasattr(w.end_indices_4, "copy_to_host") else w.end_indices_4)
    w.start_indices_4 = cuda.to_device(np.append(s4, 0))
    w.end_indices_4 = cuda.to_device(np.append(e4, 0))
    # deterministic contents for buffers the reference leaves uninitialised
    for name in ("z_alpha_powers_real", "z_alpha_powers_imag", "z_gamma_powers_real",
                 "z_gamma_powers_imag", "Hextra"):
        arr = getattr(w, name)
        arr[:] = 0
    return w


def load_module(dotted):
    """Import a reference module by dotted name (after installing the stubs)."""
    _install_stubs()
    return importlib.import_module(dotted)
