"""Oracle (test infrastructure only): Wigner-d / Wigner-D matrices in float64.

Restates the quantity the reference computes with its H-recursion kernels
(``src/matcha/core/WignerDMatrices.py:673-801`` for the recursion,
``:281-306`` for the fill ``D = eps(m') eps(-m) H z_a^{m'} z_g^{m}``, and
``:969-1012`` for the flat index).  The convention, pinned against the
reference kernels run in Numba's CPU simulator (tests/golden), is

    D^l_{m'm}(alpha, beta, gamma) = exp(+i m' alpha) d^l_{m'm}(beta) exp(+i m gamma)

with the standard (Edmonds) small-d, stored flat as ``[l][m'=-l..l][m=-l..l]``.

Two independent evaluations are provided: the explicit Wigner sum (exact in
rational arithmetic up to the float64 evaluation) and the three-term recurrence in
``l`` for fixed ``(m', m)`` that the CUDA kernels use.  Only tests, the smoke check
and the CPU baseline may import this module.
"""
from __future__ import annotations

from functools import lru_cache
from math import factorial

import numpy as np


def dsize(ell_max: int) -> int:
    """Number of entries of D up to and including degree ell_max (WignerDMatrices.py:48-99)."""
    if ell_max < 0:
        return 0
    L = ell_max
    return (L + 1) * (2 * L + 1) * (2 * L + 3) // 3


def dindex(l: int, mp: int, m: int) -> int:
    """Flat index of D^l_{mp, m} (WignerDMatrices.py:969-1012 with ell_min=0, mp_max>=l)."""
    return dsize(l - 1) + (mp + l) * (2 * l + 1) + (m + l)


@lru_cache(maxsize=None)
def _lmm_table(ell_max: int):
    ls, mps, ms = [], [], []
    for l in range(ell_max + 1):
        for mp in range(-l, l + 1):
            for m in range(-l, l + 1):
                ls.append(l)
                mps.append(mp)
                ms.append(m)
    return np.array(ls), np.array(mps), np.array(ms)


def lmm(ell_max: int):
    """Arrays (l, m', m) for every flat index up to ell_max."""
    return _lmm_table(int(ell_max))


def small_d_explicit(l: int, mp: int, m: int, beta: float) -> float:
    """Edmonds' explicit sum for d^l_{m'm}(beta), float64."""
    c = np.cos(beta / 2.0)
    s = np.sin(beta / 2.0)
    pref = np.sqrt(float(factorial(l + mp) * factorial(l - mp) * factorial(l + m) * factorial(l - m)))
    total = 0.0
    kmin = max(0, m - mp)
    kmax = min(l + m, l - mp)
    for k in range(kmin, kmax + 1):
        num = (-1.0) ** (mp - m + k)
        den = float(factorial(l + m - k) * factorial(k) * factorial(mp - m + k) * factorial(l - mp - k))
        total += num / den * c ** (2 * l + m - mp - 2 * k) * s ** (mp - m + 2 * k)
    return pref * total


def small_d_block_explicit(l: int, beta: float) -> np.ndarray:
    out = np.zeros((2 * l + 1, 2 * l + 1))
    for i, mp in enumerate(range(-l, l + 1)):
        for j, m in enumerate(range(-l, l + 1)):
            out[i, j] = small_d_explicit(l, mp, m, beta)
    return out


def small_d_all(ell_max: int, beta) -> np.ndarray:
    """d^l_{m'm}(beta) for l <= ell_max, flat order, via the recurrence in l.

    ``beta`` may be an array; the result has shape ``beta.shape + (dsize(ell_max),)``.
    Starting value at l0 = max(|m'|, |m|) (closed form), then for l >= l0
        l*sqrt(((l+1)^2-m^2)((l+1)^2-m'^2)) d^{l+1}
          = (2l+1)(l(l+1)cos(beta) - m m') d^l - (l+1) sqrt((l^2-m^2)(l^2-m'^2)) d^{l-1}
    (with d^{l0-1} = 0; for l0 = 0 the first step is d^1 = cos(beta) d^0 when m = m' = 0).
    """
    beta = np.asarray(beta, dtype=np.float64)
    flat = beta.reshape(-1)
    out = np.zeros((flat.size, dsize(ell_max)))
    cb = np.cos(flat)
    ch = np.cos(flat / 2.0)
    sh = np.sin(flat / 2.0)
    for mp in range(-ell_max, ell_max + 1):
        for m in range(-ell_max, ell_max + 1):
            l0 = max(abs(mp), abs(m))
            dl = start_value(l0, mp, m, ch, sh)
            dlm1 = np.zeros_like(dl)
            out[:, dindex(l0, mp, m)] = dl
            for l in range(l0, ell_max):
                if l == 0:
                    dnew = cb * dl
                else:
                    a = (2 * l + 1) * (l * (l + 1) * cb - m * mp)
                    b = (l + 1) * np.sqrt(float((l * l - m * m) * (l * l - mp * mp)))
                    c = l * np.sqrt(float(((l + 1) ** 2 - m * m) * ((l + 1) ** 2 - mp * mp)))
                    dnew = (a * dl - b * dlm1) / c
                dlm1, dl = dl, dnew
                out[:, dindex(l + 1, mp, m)] = dl
    return out.reshape(beta.shape + (dsize(ell_max),))


def start_value(l0: int, mp: int, m: int, ch, sh):
    """d^{l0}_{m'm} with l0 = max(|m'|, |m|), closed form.

    The explicit sum has a single term at l0: with k the only admissible index,
    d = (-1)^(m'-m+k) sqrt((l+m')!(l-m')!(l+m)!(l-m)!) / [(l+m-k)! k! (m'-m+k)! (l-m'-k)!]
        * cos(b/2)^(2l+m-m'-2k) sin(b/2)^(m'-m+2k)
    """
    l = l0
    kmin = max(0, m - mp)
    kmax = min(l + m, l - mp)
    assert kmin == kmax, (l, mp, m)
    k = kmin
    lognum = 0.5 * (_lf(l + mp) + _lf(l - mp) + _lf(l + m) + _lf(l - m))
    logden = _lf(l + m - k) + _lf(k) + _lf(mp - m + k) + _lf(l - mp - k)
    coef = np.exp(lognum - logden) * (-1.0) ** (mp - m + k)
    return coef * ch ** (2 * l + m - mp - 2 * k) * sh ** (mp - m + 2 * k)


def _lf(n: int) -> float:
    from math import lgamma

    return lgamma(n + 1.0)


def wigner_D(alpha, beta, gamma, ell_max: int) -> np.ndarray:
    """Complex D up to ell_max, flat order; leading dims follow the angle arrays."""
    alpha = np.asarray(alpha, dtype=np.float64)
    beta = np.asarray(beta, dtype=np.float64)
    gamma = np.asarray(gamma, dtype=np.float64)
    d = small_d_all(ell_max, beta)
    _, mps, ms = lmm(ell_max)
    phase = np.exp(1j * (alpha[..., None] * mps + gamma[..., None] * ms))
    return d * phase
