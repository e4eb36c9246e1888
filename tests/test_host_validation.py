"""Argument validation happens on the host, in the reference's terms, before
any device work (runs without a GPU)."""
import numpy as np
import pytest

from conftest import make_set
from kernelforge_b200 import kernelmath as km
from kernelforge_b200 import local_kernels as lk


def test_sigma_must_be_positive():
    X, dX, Q, N = make_set(3, 4, 5, 2, 0)
    for bad in (0.0, -1.0, float("nan"), float("inf")):
        with pytest.raises(ValueError, match="sigma"):
            lk.kernel_gaussian_symm(X, Q, N, bad)
        with pytest.raises(ValueError, match="sigma"):
            lk.kernel_gaussian(X, X, Q, Q, N, N, bad)
        with pytest.raises(ValueError, match="sigma"):
            lk.kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, bad)


def test_shape_errors_raise_value_error():
    X, dX, Q, N = make_set(3, 4, 5, 2, 0)
    with pytest.raises(ValueError):
        lk.kernel_gaussian_symm(X[0], Q, N, 1.0)
    with pytest.raises(ValueError, match="Q shape"):
        lk.kernel_gaussian_symm(X, Q[:, :2], N, 1.0)
    with pytest.raises(ValueError, match="N length"):
        lk.kernel_gaussian_symm(X, Q, N[:2], 1.0)
    with pytest.raises(ValueError, match="X2"):
        lk.kernel_gaussian(X, X[:, :, :3], Q, Q, N, N, 1.0)
    with pytest.raises(ValueError, match="dX2"):
        lk.kernel_gaussian_jacobian(X, X, dX[:, :, :, :5], Q, Q, N, N, 1.0)
    with pytest.raises(ValueError, match="dX1"):
        lk.kernel_gaussian_jacobian_t(X, dX[:2], X, Q, Q, N, N, 1.0)
    with pytest.raises(ValueError, match="dX"):
        lk.kernel_gaussian_hessian_symm(X, dX[..., :3], Q, N, 1.0)


def test_empty_derivative_axes_return_empty_arrays():
    # the reference returns (nm1, 0) / (0, nm2) / (0, 0) arrays without touching
    # the kernels when naq is zero (src/local_kernels_bindings.cpp:226-231, :474-483)
    X, dX, Q, N = make_set(3, 4, 5, 2, 0)
    Z = np.zeros_like(N)
    assert lk.kernel_gaussian_jacobian(X, X, dX, Q, Q, N, Z, 1.0).shape == (3, 0)
    assert lk.kernel_gaussian_jacobian_t(X, dX, X, Q, Q, Z, N, 1.0).shape == (0, 3)
    assert lk.kernel_gaussian_hessian(X, dX, X, dX, Q, Q, Z, N, 1.0).shape[0] == 0
    assert lk.kernel_gaussian_hessian_symm(X, dX, Q, Z, 1.0).shape == (0, 0)


def test_precision_keyword_is_validated():
    X, dX, Q, N = make_set(3, 4, 5, 2, 0)
    with pytest.raises(ValueError, match="precision"):
        lk.kernel_gaussian_symm(X, Q, N, 1.0, precision="fp8")


def test_cho_solve_rfp_length_check():
    with pytest.raises(RuntimeError, match="n\\*\\(n\\+1\\)/2"):
        km.cho_solve_rfp(np.zeros(5), np.zeros(3))
    with pytest.raises(RuntimeError, match="square"):
        km.full_to_rfp(np.zeros((3, 4)))


def test_bucket_planning_matches_reference_packing():
    """The host plan (labels ascending, molecules in order inside a bucket) is
    the reference's pack_label_block_sym_T order (src/local_kernels.cpp:332-375)."""
    X, dX, Q, N = make_set(6, 5, 3, 3, 4)
    N[1] = 9      # clamped to max_atoms
    N[2] = -2     # clamped to zero
    labels = sorted({int(Q[a, i]) for a in range(6) for i in range(min(max(N[a], 0), 5))})
    order = [(a, i) for lab in labels for a in range(6)
             for i in range(min(max(int(N[a]), 0), 5)) if Q[a, i] == lab]
    assert len(order) == int(np.clip(N, 0, 5).sum())
