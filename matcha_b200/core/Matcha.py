"""Drop-in ``Matcha`` orientation search (src/matcha/core/Matcha.py) on the B200 kernels.

Same constructor, configuration keys, defaults, errors and return values as the
reference class; the grid search, every Newton step of every march stage and the
reduction over candidates run in ``mtb_search_orientations`` (one grid launch, one
march launch, one reduction launch).
"""
from __future__ import annotations

import ctypes

import torch

from .. import _native as nat
from .SOFFT import SOFFT
from .wigner_index import dsize

_DEFAULTS = {
    "candidates": 10,
    "reinits": 1,
    "num_steps": 5,
    "step_type": "newton",
    "stop_early": False,
    "do_random_sampling": False,
    "reinits_iterations": 0,
    "oversampling_factor_K": 2,
}


def _cfg_get(cfg, key):
    if isinstance(cfg, dict):
        return cfg[key]
    return getattr(cfg, key)


def _cfg_has(cfg, key):
    try:
        return key in cfg
    except TypeError:
        return hasattr(cfg, key)


def _cfg_set(cfg, key, value):
    try:
        cfg[key] = value
    except TypeError:
        setattr(cfg, key, value)


def reduce_over_candidates(alphas, betas, gammas, scores):
    """Best candidate per subtomogram (Matcha.py:19-24); first maximum on ties."""
    scores, idx = torch.max(scores, dim=-1)
    pick = lambda x: torch.gather(x, 1, idx.unsqueeze(-1)).squeeze(-1)
    return pick(alphas), pick(betas), pick(gammas), scores


def march_schedule(Li, Lmax):
    """Stages actually run: sorted(Li) + [Lmax], skipping Li >= Lmax unless last (Matcha.py:76,381-386)."""
    sched = sorted(int(x) for x in Li) + [int(Lmax)]
    return [l for i, l in enumerate(sched) if not (l >= Lmax and i != len(sched) - 1)]


class Matcha:
    """Frequency-marched Newton orientation search (Matcha.py:62-403)."""

    def __init__(self, batchsize: int, device: torch.device, L_max: int, matcha_config=None,
                 compat_top_block: bool = False):
        matcha_config = self._assert_config(matcha_config)
        self.device = torch.device(device)
        self.Lmax = int(L_max)
        self.Li = sorted(_cfg_get(matcha_config, "Li")) + [self.Lmax]
        self.L0 = min(self.Li)
        self.do_random_sampling = _cfg_get(matcha_config, "do_random_sampling")
        self.batchsize = int(batchsize)
        self.candidates = int(_cfg_get(matcha_config, "candidates"))
        self.reinits = int(_cfg_get(matcha_config, "reinits"))
        self.reinits_iterations = _cfg_get(matcha_config, "reinits_iterations")
        self.num_steps = int(_cfg_get(matcha_config, "num_steps"))
        self.stop_early = bool(_cfg_get(matcha_config, "stop_early"))
        self.num_templates = 1
        self.step_type = _cfg_get(matcha_config, "step_type")
        self.base_lr = 1 if self.step_type == "newton" else 5e-7
        self.compat_top_block = bool(compat_top_block)
        if self.reinits != 1:
            # the reference's view(B, C*reinits, ...) against (B, C) angles fails for reinits > 1
            raise ValueError("reinits > 1 is not supported (the reference fails on it too)")
        if self.stop_early:
            raise ValueError("stop_early=True is not supported by matcha_b200")
        if self.step_type not in ("newton", "gradient"):
            raise ValueError(f"unknown step_type {self.step_type!r}")
        K = int(_cfg_get(matcha_config, "oversampling_factor_K"))
        self.SOFFT = SOFFT(L=self.L0, device=self.device, batchsize=self.batchsize, oversampling_factor=K)
        self.stages = march_schedule(_cfg_get(matcha_config, "Li"), self.Lmax)
        self._truncate_dsize_cache = {int(l): dsize(int(l)) for l in set(self.Li)}
        flags = 0
        if self.compat_top_block:
            flags |= nat.MTB_SEARCH_COMPAT_TOP_BLOCK
        if self.step_type == "gradient":
            flags |= nat.MTB_SEARCH_GRADIENT_STEP
        self._cfg = nat.MtbSearchConfig()
        self._cfg.Lmax = self.Lmax
        self._cfg.n_stages = len(self.stages)
        if len(self.stages) > nat.MTB_MAX_STAGES:
            raise ValueError(f"at most {nat.MTB_MAX_STAGES} march stages are supported")
        for i, l in enumerate(self.stages):
            self._cfg.stages[i] = l
        self._cfg.L0 = self.L0
        self._cfg.K = K
        self._cfg.candidates = self.candidates
        self._cfg.num_steps = self.num_steps
        self._cfg.max_batch = self.batchsize
        self._cfg.flags = flags
        lib = nat.load()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(lib.mtb_search_create(ctypes.byref(self._cfg), ctypes.byref(h)), "mtb_search_create")
        self._h = h
        self._lib = lib

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.mtb_search_destroy(h)
            self._h = None

    def _assert_config(self, matcha_config):
        if matcha_config is None:
            matcha_config = {}
        if not _cfg_has(matcha_config, "Li"):
            raise ValueError("Matcha config missing required key: 'Li'")
        for key, default_value in _DEFAULTS.items():
            if not _cfg_has(matcha_config, key):
                _cfg_set(matcha_config, key, default_value)
        return matcha_config

    def _prep_sigma(self, sigma: torch.Tensor) -> torch.Tensor:
        nat.require_cuda(sigma, "sigma")
        if sigma.ndim != 2:
            raise ValueError("sigma must have shape (batch, Dsize)")
        if sigma.dtype != torch.complex64:
            sigma = sigma.to(torch.complex64)
        if sigma.stride(1) != 1:
            sigma = sigma.contiguous()
        if sigma.shape[1] < dsize(self.Lmax):
            raise ValueError(f"sigma has {sigma.shape[1]} columns; dsize(L_max)={dsize(self.Lmax)} needed")
        if sigma.shape[0] > self.batchsize:
            raise ValueError(f"Input batch size {sigma.shape[0]} exceeds configured batchsize {self.batchsize}.")
        return sigma

    @torch.no_grad()
    def _grid_search_so3fft(self, sigma):
        """Top-`candidates` grid peaks as Euler angles, each (B, candidates) (Matcha.py:207-236)."""
        sigma = self._prep_sigma(sigma)
        B = sigma.shape[0]
        out = torch.empty((3, B, self.candidates), device=sigma.device, dtype=torch.float32)
        with torch.cuda.device(sigma.device):
            nat.check(self._lib.mtb_so3_grid_topk(self._h, nat.ptr(sigma), sigma.stride(0), B, nat.ptr(out[0]),
                                                nat.ptr(out[1]), nat.ptr(out[2]), None,
                                                nat.stream_ptr(sigma.device)), "mtb_so3_grid_topk")
        return out[0], out[1], out[2]

    @torch.no_grad()
    def march(self, alphas, betas, gammas, sigma):
        """All march stages for given starting candidates; returns refined angles and scores (B, C)."""
        sigma = self._prep_sigma(sigma)
        B = sigma.shape[0]
        a = alphas.to(device=sigma.device, dtype=torch.float32).contiguous().clone()
        b = betas.to(device=sigma.device, dtype=torch.float32).contiguous().clone()
        g = gammas.to(device=sigma.device, dtype=torch.float32).contiguous().clone()
        if a.shape != (B, self.candidates):
            raise ValueError("angles must have shape (batch, candidates)")
        s = torch.empty_like(a)
        with torch.cuda.device(sigma.device):
            nat.check(self._lib.mtb_newton_march(self._h, nat.ptr(sigma), sigma.stride(0), B, nat.ptr(a), nat.ptr(b),
                                               nat.ptr(g), nat.ptr(s), nat.stream_ptr(sigma.device)),
                    "mtb_newton_march")
        return a, b, g, s

    @torch.no_grad()
    def score_derivatives(self, sigma, alpha, beta, gamma, L: int = None):
        """Score f = Re sum_{l <= L} D^l(alpha, beta, gamma) sigma_l at one point per row of
        sigma, its Euler gradient (B, 3) and Hessian (B, 3, 3) (``mtb_score_derivatives``; the
        quantities of WignerDGradients.get_derivatives, WignerDGradients.py:247-302).
        L defaults to L_max; angles (B,) in radians."""
        L = self.Lmax if L is None else int(L)
        if not 0 <= L <= self.Lmax:
            raise ValueError(f"L must be in [0, {self.Lmax}]")
        nat.require_cuda(sigma, "sigma")
        if sigma.ndim != 2:
            raise ValueError("sigma must have shape (batch, Dsize)")
        if sigma.dtype != torch.complex64:
            sigma = sigma.to(torch.complex64)
        if sigma.stride(1) != 1:
            sigma = sigma.contiguous()
        if sigma.shape[1] < dsize(L):
            raise ValueError(f"sigma has {sigma.shape[1]} columns; dsize(L)={dsize(L)} needed")
        B = sigma.shape[0]
        ang = [torch.as_tensor(t, device=sigma.device).to(torch.float32).reshape(-1).contiguous()
               for t in (alpha, beta, gamma)]
        if any(t.shape[0] != B for t in ang):
            raise ValueError("one (alpha, beta, gamma) per row of sigma")
        out = torch.empty((B, 10), device=sigma.device, dtype=torch.float32)
        with torch.cuda.device(sigma.device):
            nat.check(self._lib.mtb_score_derivatives(self._h, nat.ptr(sigma), sigma.stride(0), B, L,
                                                      nat.ptr(ang[0]), nat.ptr(ang[1]), nat.ptr(ang[2]),
                                                      nat.ptr(out), nat.stream_ptr(sigma.device)),
                      "mtb_score_derivatives")
        h = out[:, 4:]
        H = torch.stack([torch.stack([h[:, 0], h[:, 1], h[:, 2]], -1),
                         torch.stack([h[:, 1], h[:, 3], h[:, 4]], -1),
                         torch.stack([h[:, 2], h[:, 4], h[:, 5]], -1)], -2)
        return out[:, 0], out[:, 1:4], H

    @torch.no_grad()
    def search_orientations(self, sigma):
        """(alpha, beta, gamma, score), each (B,), radians (Matcha.py:369-403)."""
        sigma = self._prep_sigma(sigma)
        B = sigma.shape[0]
        out = torch.empty((4, B), device=sigma.device, dtype=torch.float32)
        with torch.cuda.device(sigma.device):
            nat.check(self._lib.mtb_search_orientations(self._h, nat.ptr(sigma), sigma.stride(0), B, nat.ptr(out[0]),
                                                      nat.ptr(out[1]), nat.ptr(out[2]), nat.ptr(out[3]),
                                                      nat.stream_ptr(sigma.device)), "mtb_search_orientations")
        return out[0], out[1], out[2], out[3]
