"""The expansion tables, the dense adjoint and sigma against the reference's own code.

``tests/golden/fle_ref.npz`` holds the output of the reference's ``lap_eig_ball``
(src/matcha/core/FLEBasis3D.py:700-799) at the four alignment shapes and of its
``create_denseB`` (:570-698) applied as a = B^H f to seeded volumes; ``sigma_ref.npz``
holds its ``compute_sigma`` (src/matcha/core/CrossCorrelationMatcher.py:133-212) on those
coefficients.  These CPU tests pin the host tables and the oracle to them; the GPU
kernels are checked against the same fixtures in ``test_fle_gpu.py``.
"""
import numpy as np
import pytest

from matcha_b200.core import fle_tables as T
from oracle import fle as F
from tests.helpers import golden

SHAPES = [(16, 8), (32, 16), (64, 32), (128, 64)]


@pytest.fixture(scope="module")
def fx():
    return golden("fle_ref.npz")


@pytest.mark.parametrize("N,L", SHAPES)
def test_tables_equal_reference_lap_eig_ball(fx, N, L):
    tb = T.lap_eig_ball(N, L, N // 2)
    tag = f"t{N}"
    assert tb.ne == int(fx[f"{tag}_ne"])
    for k in ("ls", "ks", "ms", "mds"):
        np.testing.assert_array_equal(getattr(tb, k), fx[f"{tag}_{k}"])
    np.testing.assert_allclose(tb.lmds, fx[f"{tag}_lmds"], rtol=1e-13)
    np.testing.assert_allclose(tb.cs, fx[f"{tag}_cs"], rtol=1e-12)


def test_benchmark_shape_coefficient_count(fx):
    """ne at 64^3, L = 32 as the reference computes it: 8252, lmax 42."""
    assert int(fx["t64_ne"]) == 8252
    assert int(fx["t64_ls"].max()) == 42


def test_regenerated_zeros_checked_independently(fx):
    assert float(fx["root_check_err"]) < 1e-9


@pytest.mark.parametrize("tag,N,L,radius", [("c16r8", 16, 8, 8), ("c32r16", 32, 16, 16), ("c32r15", 32, 16, 15)])
def test_oracle_adjoint_equals_reference_dense_basis(fx, tag, N, L, radius):
    tb = T.lap_eig_ball(N, L, radius)
    vols = fx[f"{tag}_volumes"]
    ref = fx[f"{tag}_coeffs"]
    a = F.evaluate_t(tb, vols, float(radius))
    assert np.abs(a - ref).max() < 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("tag,N,L,radius", [("c16r8", 16, 8, 8), ("c32r16", 32, 16, 16)])
def test_oracle_sigma_equals_reference_compute_sigma(fx, tag, N, L, radius):
    sx = golden("sigma_ref.npz")
    tb = T.lap_eig_ball(N, L, radius)
    a = fx[f"{tag}_coeffs"]
    sig = F.compute_sigma(tb, a[0], a)
    ref = sx[f"{tag}_sigma"]
    assert sig.shape == ref.shape
    assert np.abs(sig - ref).max() < 1e-12 * np.abs(ref).max()
    np.testing.assert_allclose(np.linalg.norm(a, axis=1), sx[f"{tag}_norms"], rtol=1e-14)


@pytest.mark.parametrize("tag,N,L,radius", [("c16r8", 16, 8, 8), ("c32r16", 32, 16, 16), ("c32r15", 32, 16, 15)])
def test_streamed_oracle_adjoint_equals_reference_dense_basis(fx, tag, N, L, radius):
    """The basis-free form the 128^3, L = 64 accuracy check uses (one degree at a time, no
    n_rep x ne matrix) gives the reference's dense adjoint too."""
    from oracle import pipeline as OP

    tb = T.lap_eig_ball(N, L, radius)
    ff = OP.FoldedFLE(tb, N, float(radius), dense=False)
    ref = fx[f"{tag}_coeffs"]
    a = ff.evaluate_t_streamed(fx[f"{tag}_volumes"])
    assert np.abs(a - ref).max() < 1e-10 * np.abs(ref).max()
