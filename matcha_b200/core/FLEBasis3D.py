"""Drop-in ``FLEBasis3D`` (src/matcha/core/FLEBasis3D.py) on the B200 kernels.

Same constructor and attributes the callers use (``ne``, ``lmax``, ``ls``, ``ks``,
``ms``, ``mds``, ``lmds``, ``cs``, ``idlm_list``, ``h``, ``N``, ``N1``) and
``evaluate_t``.  The coefficients are the discrete adjoint a = h B^H f of the
reference's basis, computed exactly (FP32 accumulation) instead of through the
reference's NUFFT approximation; the compute runs in ``mtb_fle_forward``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from .. import _native as nat
from . import fle_tables as T


def build_compact_tables(tb: T.FLETables, N1: int, radius: float):
    """Octant representatives, real columns with parity classes, radial table, maps."""
    from scipy.special import spherical_jn

    N = N1 + (N1 % 2)
    R = N // 2
    # representatives: |x|, |y|, |z| of every ball voxel
    g = np.arange(-R, R + N % 2)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    inside = (np.sqrt(x ** 2 + y ** 2 + z ** 2) / radius) <= 1 + 1e-13
    if N > N1:
        inside[N1:], inside[:, N1:], inside[:, :, N1:] = False, False, False
    reps = np.unique(np.stack([np.abs(x[inside]), np.abs(y[inside]), np.abs(z[inside])], 1), axis=0)
    n_rep = reps.shape[0]
    img = np.full((n_rep, 8), -1, dtype=np.int32)
    for s in range(8):
        sx, sy, sz = (-1 if s & 1 else 1), (-1 if s & 2 else 1), (-1 if s & 4 else 1)
        ix, iy, iz = sx * reps[:, 0] + R, sy * reps[:, 1] + R, sz * reps[:, 2] + R
        ok = (ix >= 0) & (ix < N1) & (iy >= 0) & (iy < N1) & (iz >= 0) & (iz < N1)
        # a flipped zero coordinate is the same voxel: count it once
        dup = ((s & 1) & (reps[:, 0] == 0)) | ((s & 2) > 0) & (reps[:, 1] == 0) | ((s & 4) > 0) & (reps[:, 2] == 0)
        ok &= ~dup.astype(bool)
        flat = (ix * N1 + iy) * N1 + iz
        img[ok, s] = flat[ok]
    rr2 = (reps ** 2).sum(1)
    r2_vals, r2_idx = np.unique(rr2, return_inverse=True)
    rnorm = np.sqrt(rr2).astype(np.float64)
    cos_t = np.where(rnorm > 0, reps[:, 2] / np.where(rnorm > 0, rnorm, 1.0), 1.0)
    phi = np.arctan2(reps[:, 1], reps[:, 0]).astype(np.float64)
    # radial functions per distinct (l, k)
    lk_keys = sorted({(int(l), int(k)) for l, k in zip(tb.ls, tb.ks)})
    lk_index = {key: j for j, key in enumerate(lk_keys)}
    lam_of = {(int(l), int(k)): float(lmd) for l, k, lmd in zip(tb.ls, tb.ks, tb.lmds)}
    jtab = np.zeros((r2_vals.size, len(lk_keys)), dtype=np.float64)
    rv = np.sqrt(r2_vals.astype(np.float64)) / radius
    for (l, k), j in lk_index.items():
        jtab[:, j] = spherical_jn(l, lam_of[(l, k)] * rv)
    # real columns: Re (and Im for m > 0) of each coefficient with m >= 0
    cols = []  # (i, part)
    col_of = {}
    for i in range(tb.ne):
        if tb.ms[i] >= 0:
            col_of[(i, 0)] = len(cols)
            cols.append((i, 0))
            if tb.ms[i] > 0:
                col_of[(i, 1)] = len(cols)
                cols.append((i, 1))
    nc = len(cols)
    col_l = np.array([tb.ls[i] for i, _ in cols], dtype=np.int32)
    col_m = np.array([tb.ms[i] for i, _ in cols], dtype=np.int32)
    col_part = np.array([p for _, p in cols], dtype=np.int32)
    x_odd = np.where(col_part == 0, col_m % 2, 1 - col_m % 2)
    y_odd = col_part
    z_odd = (col_l + col_m) % 2
    col_class = (x_odd | (y_odd << 1) | (z_odd << 2)).astype(np.int32)
    col_lk = np.array([lk_index[(int(tb.ls[i]), int(tb.ks[i]))] for i, _ in cols], dtype=np.int32)
    col_scale = np.array([tb.h * tb.cs[i] for i, _ in cols], dtype=np.float64)
    # complex coefficient i from the columns
    partner = {}
    for i in range(tb.ne):
        partner[(int(tb.ls[i]), int(tb.ks[i]), int(tb.ms[i]))] = i
    cre = np.zeros(tb.ne, dtype=np.int32)
    cim = np.full(tb.ne, -1, dtype=np.int32)
    sre = np.ones(tb.ne, dtype=np.int8)
    sim = np.ones(tb.ne, dtype=np.int8)
    for i in range(tb.ne):
        m = int(tb.ms[i])
        if m >= 0:
            cre[i] = col_of[(i, 0)]
            if m > 0:
                cim[i] = col_of[(i, 1)]
        else:
            j = partner[(int(tb.ls[i]), int(tb.ks[i]), -m)]
            s = 1 if (m % 2 == 0) else -1  # (-1)^m
            cre[i] = col_of[(j, 0)]
            cim[i] = col_of[(j, 1)]
            sre[i] = s
            sim[i] = -s
    # sigma gather table: rows mu = -l..l hold idlm[l][sht(mu)], padded with -1
    kpad = np.zeros(tb.lmax + 1, dtype=np.int32)
    kidx = []
    for l in range(tb.lmax + 1):
        rows = [tb.idlm_list[l][T.sht_index(mu)] for mu in range(-l, l + 1)]
        kp = max(len(r) for r in rows)
        kpad[l] = kp
        for r in rows:
            kidx.extend(list(r) + [-1] * (kp - len(r)))
    return dict(n_rep=n_rep, rep_img=img, rep_cos=cos_t.astype(np.float64), rep_phi=phi, rep_r2=r2_idx.astype(np.int32),
                jtab=jtab, n_cols=nc, col_class=col_class, col_l=col_l, col_m=col_m, col_part=col_part, col_lk=col_lk,
                col_scale=col_scale, coef_col_re=cre, coef_col_im=cim, coef_sign_re=sre, coef_sign_im=sim, kpad=kpad,
                kidx=np.array(kidx, dtype=np.int32), reps=reps)


class FLEBasis3D:
    """Fourier-Bessel expansion on the ball (FLEBasis3D.py:24-1586, forward path)."""

    def __init__(self, N, bandlimit, eps, maxitr=None, maxfun=None, max_l=None, mode="complex",
                 sph_harm_solver="nvidia_torch", reduce_memory=True, batchsize=1, radius=1, device="cuda",
                 dtype=torch.complex128, jl_zeros_path="jl_zeros_l=3000_k=2500.mat",
                 cs_path="cs_l=3000_k=2500.mat", precision_mode="accurate", precision=None, split_degree=None):
        if mode not in ("complex", "real"):
            raise AssertionError("mode must be 'real' or 'complex'")
        if mode == "real":
            raise ValueError("mode='real' is not supported by matcha_b200 (the alignment path uses 'complex')")
        assert dtype in [torch.complex64, torch.complex128]
        self.batchsize = int(batchsize)
        self.complexmode = True
        self.reduce_memory = reduce_memory
        self.radius = radius
        self.device = torch.device(device)
        self.dtype = dtype
        self.precision_mode = precision_mode
        self.eps = eps
        if precision is None:
            # the reference's "fast" mode accepts a 1e-4 transform (its NUFFT tolerance); the BF16
            # hi+lo split GEMM is within that, the FP32 CUDA-core GEMM is the "accurate" path
            precision = "bf16x3" if str(precision_mode).strip().lower() == "fast" else "fp32"
        if precision not in ("fp32", "bf16x3"):
            raise ValueError("precision must be 'fp32' (CUDA cores) or 'bf16x3' (tensor cores, hi+lo split)")
        if split_degree is not None and precision != "bf16x3":
            raise ValueError("split_degree applies to precision 'bf16x3' only")
        self.precision = precision
        # with split_degree, the tensor-core GEMM runs the columns of degree <= split_degree in
        # plain BF16 (one MMA per K step) and keeps the hi+lo split above it
        self.split_degree = None if split_degree is None else int(split_degree)
        tb = T.lap_eig_ball(int(N), bandlimit, float(radius), jl_zeros_path, cs_path, maxfun=maxfun, max_l=max_l)
        self.tables = tb
        self.N1, self.N, self.ne, self.lmax = tb.N1, tb.N, tb.ne, tb.lmax
        self.ls, self.ks, self.ms, self.mds, self.lmds, self.cs = tb.ls, tb.ks, tb.ms, tb.mds, tb.lmds, tb.cs
        self.kmax = int(np.max(np.abs(tb.ks)))
        self.mmax = int(np.max(np.abs(tb.ms)))
        self.idlm_list = tb.idlm_list
        self.h = tb.h
        self.R = self.N // 2
        ct = build_compact_tables(tb, self.N1, float(radius))
        self.compact = ct
        keep = []
        cfg = nat.MtbFleConfig()
        cfg.N, cfg.max_batch, cfg.ne, cfg.n_rep = self.N1, self.batchsize, tb.ne, ct["n_rep"]
        cfg.n_cols, cfg.lmax, cfg.n_lk, cfg.n_r2 = ct["n_cols"], tb.lmax, ct["jtab"].shape[1], ct["jtab"].shape[0]
        for name in ("rep_img", "rep_cos", "rep_phi", "rep_r2", "jtab", "col_class", "col_l", "col_m", "col_part",
                     "col_lk", "col_scale", "coef_col_re", "coef_col_im", "coef_sign_re", "coef_sign_im", "kpad",
                     "kidx"):
            arr = np.ascontiguousarray(ct[name])
            keep.append(arr)
            setattr(cfg, name, arr.ctypes.data)
        if precision == "fp32":
            cfg.precision = nat.MTB_FLE_FP32
        elif self.split_degree is None:
            cfg.precision = nat.MTB_FLE_BF16X3
        else:
            cfg.precision, cfg.split_degree = nat.MTB_FLE_BF16_SPLIT, self.split_degree
        lib = nat.load()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            nat.check(lib.mtb_fle_create(ctypes.byref(cfg), ctypes.byref(h)), "mtb_fle_create")
        self._h = h
        self._lib = lib

    def split_tiles(self):
        """(tiles of the tensor-core GEMM that take the hi+lo split, all its tiles); (0, 0) in FP32."""
        a, b = ctypes.c_int(), ctypes.c_int()
        nat.check(self._lib.mtb_fle_split_tiles(self._h, ctypes.byref(a), ctypes.byref(b)), "mtb_fle_split_tiles")
        return a.value, b.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._lib.mtb_fle_destroy(h)
            self._h = None

    def _forward(self, f: torch.Tensor, want_norms: bool):
        nat.require_cuda(f, "volumes")
        f = f.reshape(-1, self.N1, self.N1, self.N1)
        if f.dtype != torch.float32:
            f = f.real.to(torch.float32) if f.is_complex() else f.to(torch.float32)
        f = f.contiguous()
        b = f.shape[0]
        if b > self.batchsize:
            raise ValueError(f"Input batch size {b} exceeds configured batchsize {self.batchsize}.")
        out = torch.empty((b, self.ne), device=f.device, dtype=torch.complex64)
        norms = torch.empty((b,), device=f.device, dtype=torch.float32) if want_norms else None
        with torch.cuda.device(f.device):
            nat.check(self._lib.mtb_fle_forward(self._h, nat.ptr(f), b, nat.ptr(out), out.stride(0), nat.ptr(norms),
                                              nat.stream_ptr(f.device)), "mtb_fle_forward")
        return out, norms

    def status(self):
        """Raise if a bounded device-side wait of the tensor-core path gave up (synchronises)."""
        with torch.cuda.device(self.device):
            nat.check(self._lib.mtb_fle_status(self._h, nat.stream_ptr(self.device)), "mtb_fle_status")

    @torch.no_grad()
    def evaluate_t(self, f: torch.Tensor, return_step=3):
        """Coefficients (b, ne) of real volumes (b, N, N, N) (FLEBasis3D.py:945-976)."""
        if return_step != 3:
            raise ValueError("only the full transform (return_step=3) is available")
        a, _ = self._forward(f, False)
        return a if self.dtype == torch.complex64 else a.to(self.dtype)
