"""Drop-in ``CrossCorrelationMatcher`` (src/matcha/core/CrossCorrelationMatcher.py).

``get_sigma`` runs the ball expansion of the whole batch (``mtb_fle_forward``) and the
per-degree contraction with the template (``mtb_sigma``) on the current stream, and
returns the persistent ``sigma`` / ``bh_norms`` buffers zeroed and refilled, as the
reference does.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

from .. import _native as nat
from .FLEBasis3D import FLEBasis3D
from .fle_tables import sht_index as get_sht_index  # noqa: F401  (reference name)
from .wigner_index import compute_size


def _to_complex(dtype):
    if dtype == torch.float32:
        return torch.complex64
    if dtype == torch.float64:
        return torch.complex128
    raise ValueError(f"Unsupported dtype {dtype} for conversion to complex.")


class CrossCorrelationMatcher:
    """Ball expansion + correlation coefficients sigma (CrossCorrelationMatcher.py:37-249)."""

    def __init__(self, N: int, device: torch.device, expansion_epsilon: float = 1e-4, batchsize: int = 1,
                 reduce_memory: bool = True, bandlimit: int = None, micro_batch_split: int = 2,
                 dtype=torch.float32, radius: int = None, jl_zeros_path: str = None, cs_path: str = None,
                 precision_mode: str = "accurate", precision: str = None, split_degree: int = None):
        self.N = N
        self.fle_basis_eps = expansion_epsilon
        self.batchsize = batchsize
        self.reduce_memory = reduce_memory
        self.bandlimit = bandlimit
        self.micro_batch_split = int(micro_batch_split)
        if self.micro_batch_split <= 0:
            raise ValueError("micro_batch_split must be a positive integer.")
        if self.batchsize == 1:
            self.micro_batch_split = 1
        self.micro_batch_size = max(1, min(self.batchsize, (self.batchsize + self.micro_batch_split - 1)
                                          // self.micro_batch_split))
        self.device = torch.device(device)
        self.dtype_real = dtype
        self.dtype = _to_complex(self.dtype_real)
        self.radius = radius
        # the whole batch is expanded in one pass; micro-batching only bounded the
        # reference's NUFFT workspace
        self.fle = FLEBasis3D(N=self.N, bandlimit=self.bandlimit, eps=self.fle_basis_eps,
                              reduce_memory=self.reduce_memory, batchsize=self.batchsize, radius=self.radius,
                              device=self.device, dtype=torch.complex64, jl_zeros_path=jl_zeros_path,
                              cs_path=cs_path, precision_mode=precision_mode, precision=precision,
                              split_degree=split_degree)
        self.lmax = self.fle.lmax
        self.sigma = torch.zeros((self.batchsize, compute_size(self.lmax + 1)), dtype=torch.complex64,
                                 device=self.device)
        self.bh_norms = torch.zeros((self.batchsize,), dtype=torch.float32, device=self.device)
        self._coeffs = torch.zeros((self.batchsize, self.fle.ne), dtype=torch.complex64, device=self.device)
        self.template_coefficients_alphas_torch = None
        self.bh_norm_template = None

    @torch.no_grad()
    def set_template(self, template_data: np.ndarray, mask: torch.Tensor = None):
        """Expand the template (N, N, N); keeps its coefficients and norm (:117-130)."""
        t = torch.from_numpy(np.ascontiguousarray(template_data).copy()).to(dtype=torch.float32, device=self.device)
        a, norms = self.fle._forward(t.unsqueeze(0), True)
        coeffs = F.pad(a[0], (0, 1))
        if self.template_coefficients_alphas_torch is None:
            self.template_coefficients_alphas_torch = coeffs
            self.bh_norm_template = norms[0].clone()
        else:
            # in place: a CUDA graph captured earlier (AlignmentStep.capture) reads these addresses
            self.template_coefficients_alphas_torch.copy_(coeffs)
            self.bh_norm_template.copy_(norms[0])

    @torch.no_grad()
    def get_sigma(self, volumes: torch.Tensor):
        """(sigma (batchsize, Dsize(lmax)) complex64, bh_norms (batchsize,)) (:214-249)."""
        num_volumes = volumes.shape[0]
        if num_volumes > self.batchsize:
            raise ValueError(f"Input batch size {num_volumes} exceeds configured batchsize {self.batchsize}.")
        if self.template_coefficients_alphas_torch is None:
            raise RuntimeError("set_template must be called before get_sigma")
        # rows past the batch read as zero (the rows of the batch are overwritten whole)
        if num_volumes < self.batchsize:
            self.sigma[num_volumes:].zero_()
            self.bh_norms[num_volumes:].zero_()
        if num_volumes == 0:
            return self.sigma, self.bh_norms
        self._expand(volumes)
        dev = self.device
        with torch.cuda.device(dev):
            nat.check(self.fle._lib.mtb_sigma(self.fle._h, nat.ptr(self._coeffs), self._coeffs.stride(0),
                                            nat.ptr(self.template_coefficients_alphas_torch), num_volumes,
                                            nat.ptr(self.sigma), self.sigma.stride(0), nat.stream_ptr(dev)),
                    "mtb_sigma")
        return self.sigma, self.bh_norms

    def _expand(self, volumes: torch.Tensor):
        # the reference's driver passes the rotated patches as complex64 with a zero imaginary
        # part (align_subtomograms.py:240-252); the expansion is of the real part
        if volumes.is_complex():
            volumes = volumes.real
        vol = volumes.to(device=self.device, dtype=torch.float32).contiguous()
        dev = self.device
        with torch.cuda.device(dev):
            nat.check(self.fle._lib.mtb_fle_forward(self.fle._h, nat.ptr(vol), volumes.shape[0],
                                                  nat.ptr(self._coeffs), self._coeffs.stride(0),
                                                  nat.ptr(self.bh_norms), nat.stream_ptr(dev)), "mtb_fle_forward")
        self._n_expanded = int(volumes.shape[0])

    @torch.no_grad()
    def expand(self, volumes: torch.Tensor):
        """Expand a batch (b <= batchsize, N, N, N) and keep its coefficients for
        ``sigma_from_template`` (extension: the template-independent half of get_sigma).
        Returns the coefficients (b, ne) complex64, a view of an internal buffer."""
        if volumes.shape[0] > self.batchsize:
            raise ValueError(f"Input batch size {volumes.shape[0]} exceeds configured batchsize {self.batchsize}.")
        self._expand(volumes)
        return self._coeffs[:self._n_expanded]

    @torch.no_grad()
    def sigma_from_template(self, a_template: torch.Tensor, lmax: int):
        """sigma (b, Dsize(lmax)) of the last expanded batch against the template coefficients
        a_template (ne + 1,) complex64, in a tensor of its own (extension: the differentiable
        half of get_sigma, see ``matcha_b200.autograd.template_sigma``)."""
        n = getattr(self, "_n_expanded", None)
        if n is None:
            raise RuntimeError("expand (or get_sigma) must be called before sigma_from_template")
        if not 0 <= lmax <= self.lmax:
            raise ValueError(f"lmax must be in [0, {self.lmax}]")
        t = a_template.to(device=self.device, dtype=torch.complex64).contiguous()
        if t.shape != (self.fle.ne + 1,):
            raise ValueError(f"a_template must have shape ({self.fle.ne + 1},)")
        out = torch.empty((n, compute_size(lmax + 1)), dtype=torch.complex64, device=self.device)
        if n == 0:
            return out
        with torch.cuda.device(self.device):
            nat.check(self.fle._lib.mtb_sigma_upto(self.fle._h, nat.ptr(self._coeffs), self._coeffs.stride(0),
                                                 nat.ptr(t), n, lmax, nat.ptr(out), out.stride(0),
                                                 nat.stream_ptr(self.device)), "mtb_sigma_upto")
        return out

    @torch.no_grad()
    def get_sigma_upto(self, volumes: torch.Tensor, lmax: int):
        """get_sigma for the degrees l <= lmax only: (sigma (n, Dsize(lmax)), bh_norms (n,)) for
        the n given volumes, in buffers of their own (extension: the reference always fills
        every degree of the expansion; the orientation search reads degrees <= its L_max)."""
        num_volumes = volumes.shape[0]
        if num_volumes > self.batchsize:
            raise ValueError(f"Input batch size {num_volumes} exceeds configured batchsize {self.batchsize}.")
        if self.template_coefficients_alphas_torch is None:
            raise RuntimeError("set_template must be called before get_sigma_upto")
        if not 0 <= lmax <= self.lmax:
            raise ValueError(f"lmax must be in [0, {self.lmax}]")
        n = compute_size(lmax + 1)
        buf = getattr(self, "_sigma_upto", None)
        if buf is None or buf.shape[1] != n:
            buf = torch.empty((self.batchsize, n), dtype=torch.complex64, device=self.device)
            self._sigma_upto = buf
        if num_volumes == 0:
            return buf[:0], self.bh_norms[:0]
        self._expand(volumes)
        dev = self.device
        with torch.cuda.device(dev):
            nat.check(self.fle._lib.mtb_sigma_upto(self.fle._h, nat.ptr(self._coeffs), self._coeffs.stride(0),
                                                 nat.ptr(self.template_coefficients_alphas_torch), num_volumes,
                                                 lmax, nat.ptr(buf), buf.stride(0), nat.stream_ptr(dev)),
                      "mtb_sigma_upto")
        return buf[:num_volumes], self.bh_norms[:num_volumes]
