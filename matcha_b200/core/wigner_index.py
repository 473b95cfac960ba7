"""Index algebra of the flat Wigner-D layout ``[l][m'=-l..l][m=-l..l]``.

Same layout and sizes as src/matcha/core/WignerDMatrices.py:48-99 (WignerDsize) and
:969-1012 (WignerDindex) with ell_min = 0 and mp_max >= ell.
"""


def dsize(ell_max: int) -> int:
    """Entries of D for degrees 0..ell_max."""
    if ell_max < 0:
        return 0
    L = int(ell_max)
    return (L + 1) * (2 * L + 1) * (2 * L + 3) // 3


def dindex(ell: int, mp: int, m: int) -> int:
    """Flat index of D^ell_{mp, m}."""
    return dsize(ell - 1) + (mp + ell) * (2 * ell + 1) + (m + ell)


def compute_size(n: int) -> int:
    """src/matcha/utils/setup_utils.py:35-37: dsize(n - 1)."""
    return dsize(n - 1)
