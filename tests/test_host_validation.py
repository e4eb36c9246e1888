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


def test_element_baseline_recovers_per_element_energies():
    """Least squares on element counts, no intercept (models/base.py:401-418)."""
    from kernelforge_b200.feature_maps import element_baseline
    rng = np.random.default_rng(3)
    nm, ma = 60, 7
    N = rng.integers(1, ma + 1, nm).astype(np.int32)
    Q = np.full((nm, ma), -1, np.int32)
    for m in range(nm):
        Q[m, :N[m]] = rng.integers(0, 3, N[m])
    Q[0, :] = 1                      # padding beyond N[0] must not count
    true = np.array([-0.5, -37.8, -54.6])
    counts = np.stack([np.sum(Q[m, :N[m]][:, None] == np.arange(3)[None, :], axis=0)
                       for m in range(nm)])
    y = counts @ true
    coef, cnt = element_baseline(Q, N, y, 3)
    np.testing.assert_allclose(cnt, counts)
    np.testing.assert_allclose(coef, true, rtol=1e-10, atol=1e-10)
    coef2, _ = element_baseline(Q, N, y, 3, molecules=np.arange(30))
    np.testing.assert_allclose(coef2, true, rtol=1e-10, atol=1e-10)


def test_sample_pairs_same_element_seeded_and_proportional():
    from kernelforge_b200.feature_maps import sample_pairs
    rng = np.random.default_rng(1)
    nm, ma = 50, 9
    N = rng.integers(3, ma + 1, nm).astype(np.int32)
    Q = np.full((nm, ma), -1, np.int32)
    for m in range(nm):
        Q[m, :N[m]] = rng.choice(4, N[m], p=[0.5, 0.3, 0.1, 0.1])
    a = sample_pairs(Q, N, 4, 2000, seed=7)
    b = sample_pairs(Q, N, 4, 2000, seed=7)
    flatq = Q.reshape(-1)
    total = 0
    for e, ((pi, pj), (qi, qj)) in enumerate(zip(a, b)):
        np.testing.assert_array_equal(pi, qi)
        np.testing.assert_array_equal(pj, qj)
        assert np.all(flatq[pi] == e) and np.all(flatq[pj] == e)
        assert np.all((pi % ma) < N[pi // ma]) and np.all((pj % ma) < N[pj // ma])
        total += len(pi)
    assert abs(total - 2000) <= 4
    counts = np.array([np.sum(flatq[np.arange(nm * ma) % ma < np.repeat(N, ma)] == e)
                       for e in range(4)])
    for e in range(4):
        assert abs(len(a[e][0]) - 2000 * counts[e] / counts.sum()) <= 1
    sub = sample_pairs(Q, N, 4, 500, seed=7, molecules=np.arange(10))
    for pi, pj in sub:
        assert np.all(pi // ma < 10) and np.all(pj // ma < 10)


def test_judge_feature_model_bound():
    from kernelforge_b200.feature_maps import judge_feature_model
    assert judge_feature_model(1.005, 1.0)["use"] == "feature"
    assert judge_feature_model(1.02, 1.0)["use"] == "exact"
    assert judge_feature_model(float("nan"), 1.0)["use"] == "exact"
