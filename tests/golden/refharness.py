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


# ------------------------------------------------------------------ functional shims for the driver
# The reference's alignment driver (align_subtomograms.py, utils/rotation_ops.py,
# utils/volume_rotation.py, utils/io_utils.py, core/ShiftMatcher.py:913) calls
# quaternionic.array (construction, ``*``, ``conj``, ``normalized``, ``ndarray``,
# ``to_euler_angles``, ``array.from_euler_angles``) and reads templates through
# ``mrcfile.open(path).data``.  These stand-ins restate quaternionic 1.0's published
# conventions ((w, x, y, z) components, Hamilton product, intrinsic z-y-z Euler angles) and
# serve arrays registered in memory in place of MRC files.

def _quaternionic_module():
    import numpy as np

    def _hamilton(a, b):
        w1, x1, y1, z1 = np.moveaxis(a, -1, 0)
        w2, x2, y2, z2 = np.moveaxis(b, -1, 0)
        return np.stack([w1 * w2 - x1 * x2 - y1 * y2 - z1 * z2,
                         w1 * x2 + x1 * w2 + y1 * z2 - z1 * y2,
                         w1 * y2 - x1 * z2 + y1 * w2 + z1 * x2,
                         w1 * z2 + x1 * y2 - y1 * x2 + z1 * w2], -1)

    class QArray(np.ndarray):
        def __new__(cls, data):
            a = np.asarray(data, dtype=np.float64)
            if a.shape[-1] != 4:
                raise ValueError("quaternion arrays have 4 components in the last axis")
            return a.copy().view(cls)

        def __array_finalize__(self, obj):
            pass

        def __getitem__(self, item):
            out = np.ndarray.__getitem__(self, item)
            return out.view(QArray) if isinstance(out, np.ndarray) and out.ndim >= 1 and out.shape[-1] == 4 else out

        def __mul__(self, other):
            return QArray(_hamilton(np.asarray(self), np.asarray(other)))

        @property
        def ndarray(self):
            return np.asarray(self).view(np.ndarray).copy()

        def conj(self):
            return QArray(np.asarray(self) * np.array([1.0, -1.0, -1.0, -1.0]))

        @property
        def normalized(self):
            a = np.asarray(self)
            return QArray(a / np.sqrt((a ** 2).sum(-1, keepdims=True)))

        @property
        def to_euler_angles(self):
            q = np.asarray(self)
            n = (q ** 2).sum(-1)
            out = np.empty(q.shape[:-1] + (3,))
            out[..., 0] = np.arctan2(q[..., 3], q[..., 0]) + np.arctan2(-q[..., 1], q[..., 2])
            out[..., 1] = 2 * np.arccos(np.sqrt((q[..., 0] ** 2 + q[..., 3] ** 2) / n))
            out[..., 2] = np.arctan2(q[..., 3], q[..., 0]) - np.arctan2(-q[..., 1], q[..., 2])
            return out

        @classmethod
        def from_euler_angles(cls, alpha_beta_gamma, beta=None, gamma=None):
            if beta is None:
                abg = np.asarray(alpha_beta_gamma, dtype=np.float64)
                a, b, g = abg[..., 0], abg[..., 1], abg[..., 2]
            else:
                a, b, g = (np.asarray(v, dtype=np.float64) for v in (alpha_beta_gamma, beta, gamma))
            return cls(np.stack([np.cos(b / 2) * np.cos((a + g) / 2), -np.sin(b / 2) * np.sin((a - g) / 2),
                                 np.sin(b / 2) * np.cos((a - g) / 2), np.cos(b / 2) * np.sin((a + g) / 2)], -1))

    mod = types.ModuleType("quaternionic")
    mod.array = QArray
    return mod


MRC_FILES = {}  # path -> ndarray served by the mrcfile stand-in


def _mrcfile_module():
    class _Mrc:
        def __init__(self, data):
            self.data = data

        def __enter__(self):
            return self

        def __exit__(self, *exc):
            return False

    mod = types.ModuleType("mrcfile")
    mod.open = lambda path, *a, **k: _Mrc(MRC_FILES[str(path)])
    return mod


def install_driver_shims():
    """Functional quaternionic and mrcfile stand-ins (replacing the empty stubs) for running
    the reference's alignment driver on the CPU."""
    _install_stubs()
    sys.modules["quaternionic"] = _quaternionic_module()
    sys.modules["mrcfile"] = _mrcfile_module()
