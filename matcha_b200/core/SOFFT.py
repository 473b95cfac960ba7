"""Drop-in ``SOFFT`` (src/matcha/core/SOFFT.py) and ``SOFFTMatcher`` (src/matcha/example.py:42-67).

``eval`` materialises the whole (2LK)^3 correlation grid as the reference does;
``SOFFTMatcher.search_orientations`` asks the grid kernel for its single best point
without writing the grid to memory.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import _native as nat
from .wigner_index import dsize


class SOFFT:
    """SO(3) correlation grid through Wigner-d tables (SOFFT.py:6-124)."""

    def __init__(self, L: int, device: torch.device, batchsize: int, oversampling_factor=1):
        self.num_betas = 2 * L * oversampling_factor
        self.num_alphas = 2 * L * oversampling_factor
        self.num_gammas = 2 * L * oversampling_factor
        self.batch_size = int(batchsize)
        self.device = torch.device(device)
        self.L = int(L)
        self.Dsize = dsize(self.L)
        self.K = int(oversampling_factor)
        self._handles = {}

    def _handle(self, candidates: int):
        h = self._handles.get(candidates)
        if h is not None:
            return h
        cfg = nat.MtbSearchConfig()
        cfg.Lmax = self.L
        cfg.n_stages = 1
        cfg.stages[0] = self.L
        cfg.L0 = self.L
        cfg.K = self.K
        cfg.candidates = candidates
        cfg.num_steps = 0
        cfg.max_batch = self.batch_size
        cfg.flags = 0
        lib = nat.load()
        hh = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(lib.mtb_search_create(ctypes.byref(cfg), ctypes.byref(hh)), "mtb_search_create")
        self._handles[candidates] = hh
        self._lib = lib
        return hh

    def __del__(self):
        for h in getattr(self, "_handles", {}).values():
            if h.value:
                self._lib.mtb_search_destroy(h)
        self._handles = {}

    def _run(self, flmn: torch.Tensor, candidates: int, want_grid: bool):
        nat.require_cuda(flmn, "flmn_coeffs_t")
        assert flmn.ndim == 2
        if flmn.dtype != torch.complex64:
            flmn = flmn.to(torch.complex64)
        if flmn.stride(1) != 1:
            flmn = flmn.contiguous()
        B = flmn.shape[0]
        if B > self.batch_size:
            raise ValueError(f"Input batch size {B} exceeds configured batchsize {self.batch_size}.")
        n = self.num_betas
        angles = torch.empty((3, B, candidates), device=flmn.device, dtype=torch.float32)
        grid = torch.empty((B, n, n, n), device=flmn.device, dtype=torch.float32) if want_grid else None
        h = self._handle(candidates)
        with torch.cuda.device(flmn.device):
            nat.check(self._lib.mtb_so3_grid_topk(h, nat.ptr(flmn), flmn.stride(0), B, nat.ptr(angles[0]),
                                                nat.ptr(angles[1]), nat.ptr(angles[2]), nat.ptr(grid),
                                                nat.stream_ptr(flmn.device)), "mtb_so3_grid_topk")
        return angles, grid

    @torch.no_grad()
    def eval(self, flmn_coeffs_t: torch.Tensor):
        """f: (batch, num_betas, num_alphas, num_gammas) float32 (SOFFT.py:67-98)."""
        _, grid = self._run(flmn_coeffs_t, 1, True)
        return grid

    def ids_to_angles(self, ids: torch.Tensor, shape):
        """Grid indices (beta, alpha, gamma) -> Euler angles (SOFFT.py:100-124)."""
        num_betas, num_alphas, num_gammas = shape
        betas = ids[:, :, 0] * (np.pi / (num_betas - 1))
        alphas = ids[:, :, 1] * (2 * np.pi / (num_alphas))
        gammas = ids[:, :, 2] * (2 * np.pi / (num_gammas))
        return alphas, betas, gammas


class SOFFTMatcher:
    """Grid-only orientation search with a Matcha-like API (example.py:42-67)."""

    def __init__(self, batchsize: int, device, L_max: int, oversampling_factor_K: int = 2):
        self.sofft = SOFFT(L=L_max, device=device, batchsize=batchsize, oversampling_factor=oversampling_factor_K)

    @torch.no_grad()
    def search_orientations(self, sigma):
        angles, grid = self.sofft._run(sigma, 1, True)
        best = grid.reshape(grid.shape[0], -1).max(dim=1).values
        return angles[0, :, 0], angles[1, :, 0], angles[2, :, 0], best
