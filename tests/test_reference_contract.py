"""The call contract of the drop-in modules, restated from the reference's public
stubs (python/kernelforge/local_kernels.pyi, kernelmath.pyi) and from what its
tests check of them (tests/test_local_kernels_keywords.py: every function
accepts its public parameter names as keywords; tests/test_rfp.py:191-209: a
two-point Gaussian kernel known answer, here for the local kernels).

The parameter tables below are the stubs' names and order (interface data);
this library may add keyword-only parameters with defaults (``precision``)."""
import inspect

import numpy as np
import pytest

LOCAL_KERNELS = {
    "kernel_gaussian": ["X1", "X2", "Q1", "Q2", "N1", "N2", "sigma"],
    "kernel_gaussian_symm": ["X", "Q", "N", "sigma"],
    "kernel_gaussian_symm_rfp": ["X", "Q", "N", "sigma"],
    "kernel_gaussian_jacobian": ["X1", "X2", "dX2", "Q1", "Q2", "N1", "N2", "sigma"],
    "kernel_gaussian_jacobian_t": ["X1", "dX1", "X2", "Q1", "Q2", "N1", "N2", "sigma"],
    "kernel_gaussian_hessian": ["X1", "dX1", "X2", "dX2", "Q1", "Q2", "N1", "N2", "sigma"],
    "kernel_gaussian_hessian_symm": ["X", "dX", "Q", "N", "sigma"],
    "kernel_gaussian_hessian_symm_rfp": ["X", "dX", "Q", "N", "sigma"],
    "kernel_gaussian_full": ["X1", "dX1", "X2", "dX2", "Q1", "Q2", "N1", "N2", "sigma"],
    "kernel_gaussian_full_symm": ["X", "dX", "Q", "N", "sigma"],
    "kernel_gaussian_full_symm_rfp": ["X", "dX", "Q", "N", "sigma"],
    "kernel_gaussian_local_compute_alpha_desc": ["dX2", "Q2", "N2", "alpha"],
    "kernel_gaussian_local_hessian_matvec": ["X1", "dX1", "X2", "alpha_desc", "Q1", "Q2",
                                             "N1", "N2", "sigma"],
    "kernel_gaussian_local_jacobian_t_matvec": ["X1", "X2", "alpha_desc", "Q1", "Q2", "N1",
                                                "N2", "sigma"],
    "kernel_gaussian_local_full_matvec": ["X1", "dX1", "X2", "alpha_desc_F", "alpha_E", "Q1",
                                          "Q2", "N1", "N2", "sigma"],
}
KERNELMATH = {
    "cho_solve_rfp": (["K_rfp", "y", "l2"], {"l2": 0.0}),
    "full_to_rfp": (["A", "uplo", "transr"], {"uplo": "U", "transr": "N"}),
    "rfp_to_full": (["ARF", "n", "uplo", "transr"], {"uplo": "U", "transr": "N"}),
}


def _split(fn):
    ps = list(inspect.signature(fn).parameters.values())
    pos = [p for p in ps if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]
    extra = [p for p in ps if p not in pos]
    return pos, extra


@pytest.mark.parametrize("name", sorted(LOCAL_KERNELS))
def test_local_kernels_parameter_names(name):
    from kernelforge_b200 import local_kernels as lk
    pos, extra = _split(getattr(lk, name))
    assert [p.name for p in pos] == LOCAL_KERNELS[name]
    assert all(p.default is inspect.Parameter.empty for p in pos)
    # additions are keyword-only and optional
    assert all(p.kind == p.KEYWORD_ONLY and p.default is not p.empty for p in extra)


@pytest.mark.parametrize("name", sorted(KERNELMATH))
def test_kernelmath_parameter_names_and_defaults(name):
    from kernelforge_b200 import kernelmath as km
    names, defaults = KERNELMATH[name]
    pos, extra = _split(getattr(km, name))
    assert [p.name for p in pos] == names
    assert {p.name: p.default for p in pos if p.default is not p.empty} == defaults
    assert not extra


def _dataset(seed=0, nm1=3, nm2=4, ma=4, rep=6):
    rng = np.random.default_rng(seed)
    x1 = 0.3 * rng.normal(size=(nm1, ma, rep))
    x2 = 0.3 * rng.normal(size=(nm2, ma, rep))
    dx1 = rng.normal(size=(nm1, ma, rep, 3 * ma))
    dx2 = rng.normal(size=(nm2, ma, rep, 3 * ma))
    q1 = rng.integers(0, 3, size=(nm1, ma)).astype(np.int32)
    q2 = rng.integers(0, 3, size=(nm2, ma)).astype(np.int32)
    n1 = rng.integers(1, ma + 1, size=nm1).astype(np.int32)
    n2 = rng.integers(1, ma + 1, size=nm2).astype(np.int32)
    return dict(X1=x1, X2=x2, dX1=dx1, dX2=dx2, Q1=q1, Q2=q2, N1=n1, N2=n2,
                X=x1, dX=dx1, Q=q1, N=n1, sigma=2.0)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(LOCAL_KERNELS))
def test_keyword_calls_equal_positional_calls(name):
    """Every function called with its public names as keywords (in reversed
    order) returns what the positional call returns."""
    from kernelforge_b200 import local_kernels as lk
    fn = getattr(lk, name)
    d = _dataset()
    nm2, ma2 = d["X2"].shape[:2]
    naq2 = int(3 * d["N2"].sum())
    rng = np.random.default_rng(1)
    alpha = rng.normal(size=naq2)
    d["alpha"] = alpha
    ad = lk.kernel_gaussian_local_compute_alpha_desc(d["dX2"], d["Q2"], d["N2"], alpha)
    d["alpha_desc"] = ad
    d["alpha_desc_F"] = ad
    d["alpha_E"] = rng.normal(size=nm2)
    names = LOCAL_KERNELS[name]
    args = [d[k] for k in names]
    kwargs = {k: d[k] for k in reversed(names)}
    got_pos, got_kw = fn(*args), fn(**kwargs)
    if isinstance(got_pos, tuple):
        for a, b in zip(got_pos, got_kw):
            np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-13 * np.abs(a).max())
    else:
        np.testing.assert_allclose(got_pos, got_kw, rtol=1e-13,
                                   atol=1e-13 * np.abs(got_pos).max())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32", "split_f16"])
def test_two_point_known_answer(precision):
    """Two one-atom molecules of one element, 1 apart, sigma = 1/sqrt(2):
    K = [[1, exp(-1)], [exp(-1), 1]] (dense and RFP, unpacked by kernelmath)."""
    from kernelforge_b200 import kernelmath as km
    from kernelforge_b200 import local_kernels as lk
    X = np.array([[[0.0]], [[1.0]]])
    Q = np.array([[6], [6]], dtype=np.int32)
    N = np.array([1, 1], dtype=np.int32)
    sigma = 1.0 / np.sqrt(2.0)
    want = np.array([[1.0, np.exp(-1.0)], [np.exp(-1.0), 1.0]])
    tol = 1e-15 if precision == "fp64" else 2e-6
    K = lk.kernel_gaussian_symm(X, Q, N, sigma, precision=precision)
    np.testing.assert_allclose(K, want, rtol=tol, atol=tol)
    K_rfp = lk.kernel_gaussian_symm_rfp(X, Q, N, sigma, precision=precision)
    full = km.rfp_to_full(K_rfp, n=2, uplo="L", transr="N")
    full = np.tril(full) + np.tril(full, -1).T
    np.testing.assert_allclose(full, want, rtol=tol, atol=tol)
    # the asymmetric kernel of the same two points, both ways
    np.testing.assert_allclose(lk.kernel_gaussian(X[:1], X[1:], Q[:1], Q[1:], N[:1], N[1:],
                                                  sigma, precision=precision),
                               [[np.exp(-1.0)]], rtol=tol, atol=tol)
