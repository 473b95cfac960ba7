"""Host-side tables of the Fourier-Bessel ball expansion (FLE), float64.

Restates the index construction of ``FLEBasis3D.lap_eig_ball`` and ``precomp``
(src/matcha/core/FLEBasis3D.py:111-540, 700-799): the Dirichlet-Laplacian
eigenfunctions of the unit ball

    psi_{l k m}(r, theta, phi) = c_{lk} j_l(lambda_{lk} r) Y_l^m(theta, phi),

with lambda_{lk} the k-th positive zero of the spherical Bessel function j_l and
c_{lk} = sqrt(2) / |j_{l+1}(lambda_{lk})|, ordered by lambda (stable), m swept as
0, -1, 1, -2, 2, ...  and truncated at lambda < bandlimit * pi / 2 with the
reference's "-1 then keep +-m pairs" rule.

The reference reads lambda and c from ``jl_zeros_l=3000_k=2500.mat`` and
``cs_l=3000_k=2500.mat``.  Those files are used when the configured paths exist;
otherwise the same numbers are computed here (scipy root bracketing on
``spherical_jn``), for the (l, k) range the sweep actually touches.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np
from scipy.optimize import brentq
from scipy.special import spherical_jn


class BesselZeros:
    """k-th positive zero of j_l, computed on demand and cached per l."""

    def __init__(self, mat_roots=None, mat_cs=None):
        self._roots = {}
        self._mat_roots = mat_roots
        self._mat_cs = mat_cs

    def _compute(self, l: int, count: int) -> np.ndarray:
        # zeros of j_l lie above l (the first near l + 1.86 l^(1/3)) and are about pi apart:
        # bracket sign changes on a 0.05 grid, then refine each with Brent's method
        span = (count + 3) * np.pi + 2.0 * l ** (1.0 / 3.0) + 5.0
        while True:
            xs = np.arange(max(1e-3, float(l)), float(l) + span, 0.05)
            f = spherical_jn(l, xs)
            idx = np.nonzero(np.sign(f[:-1]) * np.sign(f[1:]) < 0)[0]
            if len(idx) >= count:
                break
            span *= 1.5
        fn = lambda t: spherical_jn(l, t)
        return np.array([brentq(fn, xs[i], xs[i + 1], xtol=1e-14, rtol=1e-15, maxiter=200) for i in idx[:count]])

    def root(self, l: int, k: int) -> float:
        """k >= 1."""
        if self._mat_roots is not None:
            return float(self._mat_roots[l, k - 1])
        z = self._roots.get(l)
        if z is None or len(z) < k:
            z = self._compute(l, max(k, 8, 0 if z is None else 2 * len(z)))
            self._roots[l] = z
        return float(z[k - 1])

    def cs(self, l: int, k: int) -> float:
        if self._mat_cs is not None:
            return float(self._mat_cs[l, k - 1])
        return float(np.sqrt(2.0) / abs(spherical_jn(l + 1, self.root(l, k))))


def _load_mat(path, key):
    if not path or not os.path.exists(str(path)):
        return None
    from scipy.io import loadmat

    return loadmat(path)[key]


@dataclass
class FLETables:
    N1: int
    N: int
    radius: float
    ne: int
    ls: np.ndarray
    ks: np.ndarray
    ms: np.ndarray
    mds: np.ndarray
    lmds: np.ndarray
    cs: np.ndarray
    lmax: int
    h: float
    idlm_list: list = field(default_factory=list)


def lap_eig_ball(N1: int, bandlimit, radius: float, jl_zeros_path=None, cs_path=None, maxfun=None,
                 max_l=None) -> FLETables:
    """Select (l, k, m) exactly as FLEBasis3D.lap_eig_ball (FLEBasis3D.py:700-799)."""
    N = N1 + (N1 % 2)
    ne = int(maxfun) if maxfun else int(N ** 3 * np.pi / 6)
    zeros = BesselZeros(_load_mat(jl_zeros_path, "roots_table"), _load_mat(cs_path, "cs"))
    if not max_l:
        max_l = int(2.5 * ne ** (1 / 3))
    max_k = int(2.5 * ne ** (1 / 3))
    cap = max_l * (2 * max_l + 1) * max_k
    ls = np.zeros(cap, dtype=int)
    ks = np.zeros(cap, dtype=int)
    ms = np.zeros(cap, dtype=int)
    mds = np.zeros(cap, dtype=int)
    cs = np.zeros(cap, dtype=np.float64)
    lmds = np.full(cap, np.inf)
    ind = 0
    stop_l = max_l
    largest = 0.0
    for k in range(1, max_k):
        for l in range(stop_l):
            mr = 2 * l + 1
            ks[ind:ind + mr] = k
            ls[ind:ind + mr] = l
            mi = np.arange(mr)
            ms[ind:ind + mr] = (-1) ** mi * ((mi + 1) // 2)
            mds[ind:ind + mr] = 2 * np.abs(ms[ind:ind + mr]) - (ms[ind:ind + mr] < 0)
            lam = zeros.root(l, k)
            lmds[ind:ind + mr] = lam
            cs[ind:ind + mr] = zeros.cs(l, k)
            ind += mr
            if ind >= ne and lam > largest:
                stop_l = l
                break
            largest = max(largest, lam)
    idx = np.argsort(lmds[:ind], kind="stable")
    ls, ks, ms, mds, lmds, cs = (a[idx[:ne]] for a in (ls, ks, ms, mds, lmds, cs))
    if bandlimit:
        ne = int(np.searchsorted(lmds, bandlimit * np.pi / 2, side="left") - 1)
    if ms[ne - 1] < 0:
        ne = ne - 1
    if ne <= 1:
        ne = 1
    ls, ks, ms, mds, lmds, cs = (a[:ne] for a in (ls, ks, ms, mds, lmds, cs))
    lmax = int(np.max(np.abs(ls)))
    idlm = [[[] for _ in range(2 * lmax + 1)] for _ in range(lmax + 1)]
    for i in range(ne):
        idlm[ls[i]][mds[i]].append(i)
    return FLETables(N1=N1, N=N, radius=float(radius), ne=ne, ls=ls, ks=ks, ms=ms, mds=mds, lmds=lmds, cs=cs,
                     lmax=lmax, h=float(radius) ** (-1.5), idlm_list=idlm)


def sht_index(m: int) -> int:
    """Position of order m in the sweep 0, -1, 1, -2, 2, ... (CrossCorrelationMatcher.py:19-34)."""
    if m == 0:
        return 0
    return 2 * m if m > 0 else -2 * m - 1


def ball_offsets(N1: int, radius: float):
    """Voxel offsets (x, y, z) = (i0 - R, i1 - R, i2 - R) inside the ball |x| <= radius
    (FLEBasis3D.py:502-515: points with |x|/radius > 1 + 1e-13 are zeroed)."""
    N = N1 + (N1 % 2)
    R = N // 2
    g = np.arange(-R, R + N % 2)
    x, y, z = np.meshgrid(g, g, g, indexing="ij")
    r = np.sqrt(x ** 2 + y ** 2 + z ** 2) / radius
    inside = r <= 1 + 1e-13
    return x[inside], y[inside], z[inside], inside
