"""Oracle (test infrastructure only): the ball expansion and the correlation coefficients.

``evaluate_t`` is the quantity the reference's fast transform approximates
(src/matcha/core/FLEBasis3D.py:945-976, NUFFT + SHT + radial interpolation at
tolerance 1e-4): the discrete adjoint of the basis,

    a_i = h * sum_{|x| <= radius} f(x) conj(psi_i(x)),   psi_i = c_i j_l(lambda_i r) Y_l^m,

written exactly as the reference's dense definition ``create_denseB``
(FLEBasis3D.py:570-698): voxel (i0, i1, i2) sits at (x, y, z) = (i0 - R, i1 - R, i2 - R),
r = |x| / radius, theta = atan2(sqrt(x^2 + y^2), z), phi = atan2(y, x) in [0, 2 pi), Y_l^m the
orthonormal spherical harmonic with the Condon-Shortley phase, and Y_l^{-m} = (-1)^m conj(Y_l^m).

``compute_sigma`` restates CrossCorrelationMatcher.compute_sigma
(src/matcha/core/CrossCorrelationMatcher.py:133-212): for l <= lmax,
    sigma[Dindex(l, m, mp)] = (-1)^(m+mp) sum_k aT[l, -mp, k] conj(aV[l, -m, k]).
Parity of the fast transform against this definition is the reference's own NUFFT
tolerance (1e-4 relative); cuFINUFFT and torch-harmonics are not installed, so the
fast path itself cannot be run.  Only tests, the smoke check and the CPU baseline
may import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import spherical_jn, sph_harm_y

from . import wigner as W


def ball_geometry(N1: int, radius: float):
    N = N1 + (N1 % 2)
    R = N // 2
    g = np.arange(-R, R + N % 2)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    inside = (r / radius) <= 1 + 1e-13
    if N > N1:
        inside[N1:, :, :] = False
        inside[:, N1:, :] = False
        inside[:, :, N1:] = False
    flat = np.nonzero(inside[:N1, :N1, :N1].reshape(-1))[0]
    xs, ys, zs = x[:N1, :N1, :N1].reshape(-1)[flat], y[:N1, :N1, :N1].reshape(-1)[flat], z[:N1, :N1, :N1].reshape(-1)[flat]
    rr = np.sqrt(xs ** 2 + ys ** 2 + zs ** 2)
    th = np.arctan2(np.sqrt(xs ** 2 + ys ** 2), zs)
    ph = np.arctan2(ys, xs)
    ph = ph + 2 * np.pi * (ph < 0)
    return flat, rr / radius, th, ph


def basis_dense(tables, N1: int, radius: float, cols=None) -> tuple[np.ndarray, np.ndarray]:
    """psi values scaled by h: (n_ball_voxels, ne) complex128, and the flat voxel indices."""
    flat, r, th, ph = ball_geometry(N1, radius)
    idx = np.arange(tables.ne) if cols is None else np.asarray(cols)
    Bm = np.zeros((flat.size, idx.size), dtype=np.complex128)
    for j, i in enumerate(idx):
        l, m, lam, c = int(tables.ls[i]), int(tables.ms[i]), tables.lmds[i], tables.cs[i]
        rad = c * spherical_jn(l, lam * r)
        if m >= 0:
            Y = sph_harm_y(l, m, th, ph)
        else:
            Y = (-1) ** m * np.conj(sph_harm_y(l, -m, th, ph))
        Bm[:, j] = tables.h * rad * Y
    return Bm, flat


def evaluate_t(tables, volumes: np.ndarray, radius: float, Bm=None) -> np.ndarray:
    """Ball coefficients a (b, ne) complex128 of real volumes (b, N1, N1, N1)."""
    volumes = np.asarray(volumes, dtype=np.float64)
    b = volumes.shape[0]
    N1 = volumes.shape[1]
    if Bm is None:
        Bm, flat = basis_dense(tables, N1, radius)
    else:
        Bm, flat = Bm
    f = volumes.reshape(b, -1)[:, flat]
    return f @ np.conj(Bm)


def compute_sigma(tables, a_tmpl: np.ndarray, a_vol: np.ndarray) -> np.ndarray:
    """sigma (b, dsize(lmax)) from template (ne,) and volume (b, ne) coefficients."""
    lmax = tables.lmax
    b = a_vol.shape[0]
    out = np.zeros((b, W.dsize(lmax)), dtype=np.complex128)
    from matcha_b200.core.fle_tables import sht_index

    for l in range(lmax + 1):
        rows = [tables.idlm_list[l][sht_index(-m)] for m in range(-l, l + 1)]
        kmax = max(len(r) for r in rows)
        T = np.zeros((2 * l + 1, kmax), dtype=np.complex128)
        V = np.zeros((b, 2 * l + 1, kmax), dtype=np.complex128)
        for i, r in enumerate(rows):
            T[i, :len(r)] = a_tmpl[r]
            V[:, i, :len(r)] = np.conj(a_vol[:, r])
        # rows are indexed by -mu: T[i] holds aT[l, -(i-l)], V[:, i] holds conj(aV[l, -(i-l)])
        alp = np.einsum("ck,bak->bac", T, V)  # (b, a, c)
        m = np.arange(-l, l + 1)
        phase = (-1.0) ** (m[:, None] + m[None, :])
        out[:, W.dsize(l - 1):W.dsize(l)] = (phase * alp).reshape(b, -1)
    return out
