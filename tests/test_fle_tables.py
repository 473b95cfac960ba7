"""FLE tables and the octant-parity factorisation, checked on the CPU.

The CUDA path folds each volume into 8 reflection-parity channels and runs one GEMM per
channel; here the same tables drive a numpy evaluation that must equal the dense
definition of the reference's basis (the oracle) to float64 rounding.
"""
import numpy as np
import pytest
from scipy.special import sph_harm_y

from matcha_b200.core import fle_tables as T
from matcha_b200.core.FLEBasis3D import build_compact_tables
from oracle import fle as F


@pytest.fixture(scope="module")
def small():
    tb = T.lap_eig_ball(16, 8, 7)
    return tb


def test_table_sizes_match_reference_selection():
    tb = T.lap_eig_ball(32, 16, 16)
    assert (tb.ne, tb.lmax) == (1006, 19)
    # K_0 is the number of zeros k*pi of j_0 below the bandlimit 16 * pi / 2
    assert len(tb.idlm_list[0][0]) == 7
    # every m < 0 entry has its +|m| partner with the same (l, k)
    keys = {(int(l), int(k), int(m)) for l, k, m in zip(tb.ls, tb.ks, tb.ms)}
    assert all((l, k, -m) in keys for (l, k, m) in keys)


def test_bessel_zeros_and_normalisation():
    z = T.BesselZeros()
    np.testing.assert_allclose([z.root(0, k) for k in range(1, 5)], np.pi * np.arange(1, 5), rtol=1e-13)
    # first zero of j_1 solves tan x = x
    x = z.root(1, 1)
    assert abs(np.tan(x) - x) < 1e-9
    from scipy.integrate import quad
    from scipy.special import spherical_jn
    for l, k in [(0, 1), (3, 2), (7, 1)]:
        lam, c = z.root(l, k), z.cs(l, k)
        val, _ = quad(lambda r: (c * spherical_jn(l, lam * r)) ** 2 * r * r, 0, 1, limit=200)
        assert abs(val - 1) < 1e-10


def test_dense_basis_nearly_orthonormal():
    tb = T.lap_eig_ball(32, 16, 16)
    Bm, _ = F.basis_dense(tb, 32, 16)
    G = Bm.conj().T @ Bm
    assert np.abs(G - np.eye(tb.ne)).max() < 1.2e-3


def _emulate(tb, ct, vols, N1):
    """numpy restatement of fold -> per-class GEMM -> expand, from the compact tables."""
    b = vols.shape[0]
    v = vols.reshape(b, -1)
    f = np.zeros((b, ct["n_rep"], 8))
    for s in range(8):
        idx = ct["rep_img"][:, s]
        ok = idx >= 0
        f[:, ok, s] = v[:, idx[ok]]
    ch = np.zeros_like(f)
    for p in range(8):
        sign = np.array([(-1.0) ** bin(p & s).count("1") for s in range(8)])
        ch[:, :, p] = f @ sign
    # basis columns at the representatives
    reps = ct["reps"]
    r = np.sqrt((reps ** 2).sum(1))
    th = np.arccos(np.clip(ct["rep_cos"], -1, 1))
    cols = np.zeros((ct["n_rep"], ct["n_cols"]))
    for c in range(ct["n_cols"]):
        l, m, part = ct["col_l"][c], ct["col_m"][c], ct["col_part"][c]
        Y = np.conj(sph_harm_y(l, m, th, ct["rep_phi"]))
        ang = Y.imag if part else Y.real
        cols[:, c] = ct["col_scale"][c] * ct["jtab"][ct["rep_r2"], ct["col_lk"][c]] * ang
    C = np.zeros((b, ct["n_cols"]))
    for c in range(ct["n_cols"]):
        C[:, c] = ch[:, :, ct["col_class"][c]] @ cols[:, c]
    a = ct["coef_sign_re"] * C[:, ct["coef_col_re"]] + 1j * np.where(
        ct["coef_col_im"] >= 0, ct["coef_sign_im"] * C[:, np.maximum(ct["coef_col_im"], 0)], 0.0)
    return a


@pytest.mark.parametrize("N1,radius", [(16, 7), (16, 8), (15, 7)])
def test_parity_factorisation_equals_dense_definition(N1, radius):
    tb = T.lap_eig_ball(N1, 6, radius)
    ct = build_compact_tables(tb, N1, float(radius))
    rng = np.random.default_rng(N1 + radius)
    vols = rng.standard_normal((2, N1, N1, N1))
    a = _emulate(tb, ct, vols, N1)
    ref = F.evaluate_t(tb, vols, float(radius))
    np.testing.assert_allclose(a, ref, atol=1e-12 * np.abs(ref).max())


def test_sigma_oracle_matches_closed_form(small):
    # sigma_l = V_l T_l^H when every (l, mu) row has the same k-list
    tb = small
    rng = np.random.default_rng(1)
    vols = rng.standard_normal((3, 16, 16, 16))
    a = F.evaluate_t(tb, vols, 7.0)
    s = F.compute_sigma(tb, a[0], a[1:])
    from oracle import wigner as W
    for l in range(tb.lmax + 1):
        rows = [tb.idlm_list[l][T.sht_index(mu)] for mu in range(-l, l + 1)]
        K = len(rows[0])
        if any(len(r) != K for r in rows):
            continue
        Tm = np.array([a[0][r] for r in rows])
        for bi in range(2):
            Vm = np.array([a[1 + bi][r] for r in rows])
            blk = s[bi, W.dsize(l - 1):W.dsize(l)].reshape(2 * l + 1, 2 * l + 1)
            np.testing.assert_allclose(blk, Vm @ Tm.conj().T, atol=1e-10 * max(1, np.abs(blk).max()))
