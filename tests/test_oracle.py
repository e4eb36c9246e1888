"""The CPU oracle is pinned against the reference's own outputs (golden
fixtures made by tests/golden/make_golden.py from the reference build) and
against LAPACK's RFP routines in scipy."""
import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from conftest import load_golden
from oracle import oracle as o

KERNELS = [
    ("kernel_gaussian", ("X1", "X2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_symm", ("X1", "Q1", "N1")),
    ("kernel_gaussian_symm_rfp", ("X1", "Q1", "N1")),
    ("kernel_gaussian_jacobian", ("X1", "X2", "dX2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_jacobian_t", ("X1", "dX1", "X2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_hessian", ("X1", "dX1", "X2", "dX2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_hessian_symm", ("X1", "dX1", "Q1", "N1")),
    ("kernel_gaussian_hessian_symm_rfp", ("X1", "dX1", "Q1", "N1")),
    ("kernel_gaussian_full", ("X1", "dX1", "X2", "dX2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_full_symm", ("X1", "dX1", "Q1", "N1")),
    ("kernel_gaussian_full_symm_rfp", ("X1", "dX1", "Q1", "N1")),
]


@pytest.mark.parametrize("name,args", KERNELS)
def test_oracle_matches_reference_random(name, args):
    g = load_golden("golden_random.npz")
    got = getattr(o, name)(*[g[a] for a in args], float(g["sigma"]))
    np.testing.assert_allclose(got, g[name], rtol=1e-12, atol=1e-12)


def test_oracle_matches_reference_fchl19():
    g = load_golden("golden_fchl19.npz")
    X, dX, Q, N, s = g["X"], g["dX"], g["Q"], g["N"], float(g["sigma"])
    np.testing.assert_allclose(o.kernel_gaussian_symm_rfp(X, Q, N, s),
                               g["kernel_gaussian_symm_rfp"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(o.kernel_gaussian(X[:4], X[2:], Q[:4], Q[2:], N[:4], N[2:], s),
                               g["kernel_gaussian"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(
        o.kernel_gaussian_jacobian(X[:4], X[2:], dX[2:], Q[:4], Q[2:], N[:4], N[2:], s),
        g["kernel_gaussian_jacobian"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(o.kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, s),
                               g["kernel_gaussian_hessian_symm_rfp"], rtol=1e-10, atol=1e-10)
    np.testing.assert_allclose(o.kernel_gaussian_full_symm_rfp(X, dX, Q, N, s),
                               g["kernel_gaussian_full_symm_rfp"], rtol=1e-10, atol=1e-10)
    alpha = o.cho_solve_rfp(g["kernel_gaussian_symm_rfp"].copy(), g["cho_y"], float(g["cho_l2"]))
    np.testing.assert_allclose(alpha, g["cho_alpha"], rtol=1e-8, atol=1e-10)


def test_oracle_matches_reference_fchl19_720():
    g = load_golden("golden_fchl19_720.npz")
    np.testing.assert_allclose(o.kernel_gaussian_symm(g["X"], g["Q"], g["N"], 2.0),
                               g["kernel_gaussian_symm"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("n", [1, 2, 5, 6, 9, 10])
@pytest.mark.parametrize("lower", [False, True])
def test_rfp_layout_matches_lapack(n, lower):
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    A = A + A.T
    ref, info = lapack.dtrttf(np.asfortranarray(A), transr="N", uplo="L" if lower else "U")
    assert info == 0
    np.testing.assert_array_equal(o.full_to_rfp(A, lower), ref)
    np.testing.assert_array_equal(o.rfp_to_full(ref, n, lower), A)


@pytest.mark.parametrize("n", [3, 8, 11])
@pytest.mark.parametrize("lower", [False, True])
def test_oracle_cholesky_factor_matches_dpftrf(n, lower):
    rng = np.random.default_rng(n)
    B = rng.standard_normal((n, n))
    A = B @ B.T + n * np.eye(n)
    y = rng.standard_normal(n)
    arf = o.full_to_rfp(A, lower)
    ref, info = lapack.dpftrf(n, arf.copy(), transr="N", uplo="L" if lower else "U")
    assert info == 0
    mine = arf.copy()
    alpha = o.cho_solve_rfp(mine, y, 0.0, lower)
    np.testing.assert_allclose(mine, ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(A @ alpha, y, rtol=1e-10, atol=1e-10)


def test_oracle_cholesky_not_pd():
    A = -np.eye(4)
    with pytest.raises(RuntimeError, match="info=1"):
        o.cho_solve_rfp(o.full_to_rfp(A), np.ones(4))


def test_oracle_detects_planted_error():
    """A mistake planted in the oracle's inputs must show up as a mismatch
    against the reference fixture (the check is not vacuous)."""
    g = load_golden("golden_random.npz")
    X1 = g["X1"].copy()
    X1[0, 0, 0] += 1e-3
    got = o.kernel_gaussian_symm(X1, g["Q1"], g["N1"], float(g["sigma"]))
    assert np.abs(got - g["kernel_gaussian_symm"]).max() > 1e-8
