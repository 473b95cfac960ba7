"""Drop-in ``ShiftMatcher`` (src/matcha/core/ShiftMatcher.py) on the B200 kernels.

``set_reference`` computes the reference's once-per-template preparation
(``load_reference_full``: soft low-pass, gridding correction, centred FFT, spherical Fourier
mask, FFT shift; ShiftMatcher.py:377-472) on the device in FP64 (``mtb_shift_reference``).
``search_shifts`` turns each rotation tracker into the reference's ZYZ rotation matrix
(ShiftMatcher.py:503, :913; on the device when the tracker is a CUDA tensor) and runs the
whole per-subtomogram shift match in ``mtb_shift_search``.

Precision of the upsampled DFT: ``precision="fp32"`` (CUDA cores), ``"bf16x3"`` (tcgen05 with
a BF16 hi+lo split; ValueError on a box / upsampled region the tensor-core kernels do not
cover) or ``"auto"`` (the tensor cores where they cover the geometry, FP32 elsewhere;
``effective_precision`` says which ran).  Without the argument it comes from the config: the
namespaced key ``b200: {precision: ...}`` if present, else the reference's ``precision_mode``
("fast" -> "auto", "accurate" -> "fp32").
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
from scipy.spatial.transform import Rotation as R

from .. import _native as nat


def tracker_to_euler_deg(rotation_tracker) -> np.ndarray:
    """np.rad2deg(quaternionic.array(tracker.conj()).to_euler_angles) for (w, x, y, z) trackers."""
    q = np.asarray(rotation_tracker, dtype=np.float64).reshape(-1, 4) * np.array([1.0, -1.0, -1.0, -1.0])
    n = (q ** 2).sum(-1)
    a = np.arctan2(q[:, 3], q[:, 0]) + np.arctan2(-q[:, 1], q[:, 2])
    b = 2 * np.arccos(np.sqrt((q[:, 0] ** 2 + q[:, 3] ** 2) / n))
    g = np.arctan2(q[:, 3], q[:, 0]) - np.arctan2(-q[:, 1], q[:, 2])
    return np.rad2deg(np.stack([a, b, g], -1))


def _cfg(config, key, default=None):
    try:
        return config.get(key, default)
    except AttributeError:
        return getattr(config, key, default)


def resolve_precision(config) -> str:
    """Precision of the shift match from a run config: ``b200.precision`` when the namespaced
    key is present, else from the reference's ``precision_mode`` (setup_utils.py:6-16):
    "fast" -> "auto", anything else -> "fp32"."""
    ns = _cfg(config, "b200", None)
    if ns is not None:
        p = _cfg(ns, "precision", None)
        if p is not None:
            return str(p)
    mode = str(_cfg(config, "precision_mode", "accurate")).strip().lower()
    return "auto" if mode == "fast" else "fp32"


class ShiftMatcher:
    """Stateful shift-search wrapper (ShiftMatcher.py:766-928)."""

    def __init__(self, config, device: torch.device, dtype: torch.dtype, micro_batch_size: int = None,
                 precision: str = None, tile_rows: int = 0):
        if precision is None:
            precision = resolve_precision(config)
        if precision not in ("fp32", "bf16x3", "auto"):
            raise ValueError("precision must be 'fp32' (CUDA cores), 'bf16x3' (tensor cores, hi+lo split) or "
                             "'auto' (tensor cores where the geometry allows)")
        self.precision = precision
        self.tile_rows = int(tile_rows)  # FP32 upsampled DFT tile (0: default); matcha_b200.autotune
        self.config = config
        self.device = torch.device(device)
        self.dtype = dtype
        nb = _cfg(config, "num_subtomograms_per_batch", 1)
        self.micro_batch_size = int(micro_batch_size) if micro_batch_size is not None else max(1, int(nb // 2))
        self.reference_data_fourier = None
        self.N = int(_cfg(config, "N"))
        self.upsample_factor = int(_cfg(config, "shift_upsample_factor", 16))
        self.radius = int(_cfg(config, "shift_search_radius", 2))
        box = float(_cfg(config, "box_size", self.N))
        vox = float(_cfg(config, "voxel_size", 1.0))
        self.mask_radius = box / (2.0 * vox)
        self._h = None
        self._cap = 0
        self._ref_version = 0      # bumped by set_reference
        self._uploaded_version = -1
        self._ref_dev = None
        self._lib = nat.load()

    def _handle(self, B: int):
        if self._h is not None and B <= self._cap:
            return self._h
        self._free()
        cfg = nat.MtbShiftConfig()
        cfg.N = self.N
        cfg.max_batch = max(B, int(_cfg(self.config, "num_subtomograms_per_batch", B) or B))
        cfg.upsample_factor = self.upsample_factor
        cfg.search_radius = self.radius
        cfg.mask_radius = self.mask_radius
        cfg.cosine_width = 5.0
        cfg.precision = {"fp32": nat.MTB_SHIFT_FP32, "bf16x3": nat.MTB_SHIFT_BF16X3, "auto": nat.MTB_SHIFT_AUTO}[
            self.precision]
        cfg.tile_rows = self.tile_rows
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_shift_create(ctypes.byref(cfg), ctypes.byref(h)), "mtb_shift_create")
        self._h, self._cap = h, cfg.max_batch
        self._uploaded_version = -1
        return h

    @property
    def effective_precision(self):
        """"bf16x3" or "fp32": what the upsampled DFT runs in (None before the first search)."""
        if self._h is None:
            return None
        p = ctypes.c_int()
        nat.check(self._lib.mtb_shift_precision(self._h, ctypes.byref(p)), "mtb_shift_precision")
        return "bf16x3" if p.value == nat.MTB_SHIFT_BF16X3 else "fp32"

    def status(self):
        """Raise if a bounded device-side wait of the tensor-core path gave up (synchronises)."""
        if self._h is not None:
            with torch.cuda.device(self.device):
                nat.check(self._lib.mtb_shift_status(self._h, nat.stream_ptr(self.device)), "mtb_shift_status")

    PROFILE_STAGES = ("patch_xy_fft", "z_fft_product", "nyquist", "updft_pass1", "updft_pass23", "finalize")

    def profile(self, n_calls: int):
        """Record the device time of each kernel group of the next ``n_calls`` searches
        (extension; 0 switches it off).  The handle must exist (after a first search)."""
        if self._h is None:
            raise RuntimeError("profile() needs a shift handle: run search_shifts once first")
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_shift_profile(self._h, int(n_calls)), "mtb_shift_profile")

    def profile_read(self):
        """(summed ms per kernel group as a dict, number of calls) of the recorded searches."""
        if self._h is None:
            return {k: 0.0 for k in self.PROFILE_STAGES}, 0
        ms = (ctypes.c_float * len(self.PROFILE_STAGES))()
        calls = ctypes.c_int()
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_shift_profile_read(self._h, ms, ctypes.byref(calls)), "mtb_shift_profile_read")
        return dict(zip(self.PROFILE_STAGES, list(ms))), calls.value

    def _free(self):
        if self._h is not None and self._h.value:
            self._lib.mtb_shift_destroy(self._h)
        self._h = None
        self._cap = 0

    def __del__(self):
        if getattr(self, "_lib", None) is not None:
            self._free()

    @torch.no_grad()
    def score_and_gradient(self, subtomos: torch.Tensor, shift_zyx: torch.Tensor, rot: torch.Tensor,
                           query_xyz: torch.Tensor):
        """The correlation the shift search maximises, as a function of a continuous shift, and
        its gradient (extension, ``mtb_shift_score_grad``): for subtomograms (B, N, N, N) at the
        prior shift_zyx (B, 3), reference rotations rot (B, 9) (row-major matrices as
        ``mtb_tracker_rotation`` gives) and query shifts (B, 3) in (x, y, z), returns
        (score (B,), gradient (B, 3)) float32.  On the 1/uf grid the score is the value
        ``search_shifts`` compares."""
        if self.reference_data_fourier is None:
            raise RuntimeError("ShiftMatcher reference is not initialized. Call `set_reference` first.")
        B = subtomos.shape[0]
        vol = subtomos.to(self.device, torch.float32).contiguous()
        nat.require_cuda(vol, "subtomos")
        sz = torch.as_tensor(shift_zyx, device=self.device, dtype=torch.float32).reshape(B, 3).contiguous()
        r = torch.as_tensor(rot, device=self.device, dtype=torch.float32).reshape(B, 9).contiguous()
        q = torch.as_tensor(query_xyz, device=self.device, dtype=torch.float32).reshape(B, 3).contiguous()
        h = self._handle(B)
        self._upload_reference(h)
        score = torch.empty((B,), device=self.device, dtype=torch.float32)
        grad = torch.empty((B, 3), device=self.device, dtype=torch.float32)
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_shift_score_grad(h, nat.ptr(vol), nat.ptr(sz), nat.ptr(r), None, B, nat.ptr(q),
                                                     nat.ptr(score), nat.ptr(grad), nat.stream_ptr(self.device)),
                      "mtb_shift_score_grad")
        return score, grad

    def _upload_reference(self, h):
        if self._uploaded_version != self._ref_version:
            self._ref_dev = self.reference_data_fourier.to(torch.complex64).contiguous()
            with torch.cuda.device(self.device):
                nat.check(self._lib.mtb_shift_set_reference(h, nat.ptr(self._ref_dev), nat.stream_ptr(self.device)),
                          "mtb_shift_set_reference")
            self._uploaded_version = self._ref_version

    @torch.no_grad()
    def set_reference(self, template_data: np.ndarray):
        """Precompute and cache the Fourier-domain reference (ShiftMatcher.py:805-822):
        ``load_reference_full`` on the device in FP64 (``mtb_shift_reference``)."""
        N = self.N
        t = torch.from_numpy(np.ascontiguousarray(template_data, dtype=np.float64)).to(self.device)
        if tuple(t.shape) != (N, N, N):
            raise ValueError(f"template must be ({N}, {N}, {N})")
        ws = torch.empty((2 * (2 * N ** 3 + 2 * N),), dtype=torch.float64, device=self.device)  # 16 B each
        ref = torch.empty((1, N, N, N), dtype=torch.complex64, device=self.device)
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_shift_reference(nat.ptr(t), N, float(_cfg(self.config, "voxel_size", 1.0)),
                                                    nat.ptr(ws), nat.ptr(ref), nat.stream_ptr(self.device)),
                      "mtb_shift_reference")
        self.reference_data_fourier = ref if self.dtype == torch.complex64 else ref.to(self.dtype)
        self._ref_version += 1

    def get_base_shifts(self, num_subtomograms_per_batch: int, num_base_shifts: int, dtype_real: torch.dtype):
        """Base translation grid (B, S, 3) (ShiftMatcher.py:824-871)."""
        execution = _cfg(self.config, "execution", None)
        grid = None if execution is None else _cfg(execution, "translational_search_grid", None)
        if grid is None:
            base = torch.zeros((num_base_shifts, 3), device=self.device, dtype=dtype_real)
        else:
            base = torch.as_tensor(grid[0], device=self.device, dtype=dtype_real)
            if base.ndim == 1:
                base = base.unsqueeze(0)
            if base.shape[0] != num_base_shifts:
                if base.shape[0] > num_base_shifts:
                    base = base[:num_base_shifts]
                else:
                    pad = torch.zeros((num_base_shifts - base.shape[0], 3), device=self.device, dtype=dtype_real)
                    base = torch.cat((base, pad), dim=0)
        return base.unsqueeze(0).expand(num_subtomograms_per_batch, -1, -1)

    @torch.no_grad()
    def search_shifts(self, *, subtomos: torch.Tensor, ctfs: torch.Tensor, shift_zyx: torch.Tensor,
                      rotation_tracker, micro_batch_size: int = None):
        """(shift (B, 3) in (x, y, z), score (B,)) at the current orientations (ShiftMatcher.py:873-928)."""
        if self.reference_data_fourier is None:
            raise RuntimeError("ShiftMatcher reference is not initialized. Call `set_reference` first.")
        B = subtomos.shape[0]
        if isinstance(rotation_tracker, torch.Tensor) and rotation_tracker.is_cuda:
            # a tracker already on the device: its rotation is built there, with no host sync
            trk = rotation_tracker.to(self.device, torch.float64).reshape(-1, 4).contiguous()
            if trk.shape[0] != B:
                raise ValueError("rotation_tracker must hold one rotation per subtomogram")
            rot = torch.empty((B, 9), device=self.device, dtype=torch.float32)
            with torch.cuda.device(self.device):
                nat.check(self._lib.mtb_tracker_rotation(nat.ptr(trk), B, nat.ptr(rot), nat.stream_ptr(self.device)),
                          "mtb_tracker_rotation")
        else:
            angles = tracker_to_euler_deg(rotation_tracker)
            if angles.shape[0] != B:
                raise ValueError("rotation_tracker must hold one rotation per subtomogram")
            rot = torch.from_numpy(R.from_euler("ZYZ", angles, degrees=True).as_matrix().reshape(B, 9)).to(
                self.device, torch.float32)
        vol = subtomos.to(self.device, torch.float32).contiguous()
        nat.require_cuda(vol, "subtomos")
        sz = torch.as_tensor(shift_zyx, device=self.device, dtype=torch.float32).reshape(B, 3).contiguous()
        ctf = None
        if bool(_cfg(self.config, "do_ctf_correction", True)) and isinstance(ctfs, torch.Tensor):
            ctf = ctfs.to(self.device, torch.float32).reshape(B, self.N, self.N, self.N // 2 + 1).contiguous()
        out = torch.empty((B, 3), device=self.device, dtype=torch.float32)
        score = torch.empty((B,), device=self.device, dtype=torch.float32)
        h = self._handle(B)
        self._upload_reference(h)
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_shift_search(h, nat.ptr(vol), nat.ptr(sz), nat.ptr(rot), nat.ptr(ctf), B,
                                                 nat.ptr(out), nat.ptr(score), nat.stream_ptr(self.device)),
                      "mtb_shift_search")
        return out, score
