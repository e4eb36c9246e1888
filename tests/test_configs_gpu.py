"""Parity at the sizes of the benchmark configurations, against the reference's
own CPU FP64 modules (oracle/_ref, built from its sources by
oracle/build_ref.sh) run on the same seeded synthetic molecules:

* 1,000 molecules with 9-21 atoms, default 720-dim FCHL19 (the plain FP64
  energy-only KRR configuration): the symmetric RFP kernel at rtol 1e-12, the
  rectangular test x train kernel, and the KRR fit at lambda 1e-8 (800/200);
* 40 x 40 molecules with 9-30 atoms (a slice of the 1,000 x 1,000 gradient-kernel
  configuration): the Jacobian kernel, FP64 at rtol 1e-10, split fp16 with a
  relative Frobenius error <= 5e-5;
* 20 molecules with 21 atoms (a slice of the 300-molecule Hessian
  configuration): the energy+force RFP kernel, FP64 at rtol 1e-10, split fp16
  with a relative Frobenius error <= 5e-5.

The reference modules are test infrastructure; the tests skip when they are not
built.  Descriptors are the library's synthetic FCHL19 restatement (pinned to
the reference's fchl19_repr at 1e-15 by tests/test_repr_oracle.py)."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
SIGMA = 2.0


@pytest.fixture(scope="module")
def ref():
    if not (os.path.isdir(REF) and any(f.startswith("local_kernels") for f in os.listdir(REF))):
        pytest.skip("reference modules not built (oracle/build_ref.sh)")
    if REF not in sys.path:
        sys.path.insert(0, REF)
    import kernelmath as km
    import local_kernels as lk
    return lk, km


def rel_fro(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def config1():
    from kernelforge_b200 import synthetic
    mols = synthetic.make_molecules(1000, 9, 21, seed=20261204)
    X, Q, N = synthetic.fchl19_batched(mols, dtype=np.float64, device="cuda", chunk=128)
    return X, Q, N, mols.E


def test_config1_kernels_fp64(ref, config1):
    from kernelforge_b200 import local_kernels as lk
    rlk, _ = ref
    X, Q, N, _ = config1
    got = lk.kernel_gaussian_symm_rfp(X, Q, N, SIGMA)
    want = rlk.kernel_gaussian_symm_rfp(X, Q, N, SIGMA)
    assert got.shape == want.shape == (1000 * 1001 // 2,)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    got = lk.kernel_gaussian(X[800:], X[:800], Q[800:], Q[:800], N[800:], N[:800], SIGMA)
    want = rlk.kernel_gaussian(X[800:], X[:800], Q[800:], Q[:800], N[800:], N[:800], SIGMA)
    np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_config1_krr_fit_lambda_1e8(ref, config1):
    """cho_solve_rfp at lambda 1e-8 on the 800 training molecules.  The system's
    condition number is ~1e10, so two FP64 Cholesky solves agree to about
    cond x 1e-16 in alpha; the predictions and the residual are the stable
    quantities and are held to 1e-6."""
    from kernelforge_b200 import kernelmath as km
    from kernelforge_b200 import local_kernels as lk
    rlk, rkm = ref
    X, Q, N, E = config1
    ym = E[:800].mean()
    y = E[:800] - ym
    K = rlk.kernel_gaussian_symm_rfp(X[:800], Q[:800], N[:800], SIGMA)
    a_ref = rkm.cho_solve_rfp(K.copy(), y, 1e-8)
    a_got = km.cho_solve_rfp(lk.kernel_gaussian_symm_rfp(X[:800], Q[:800], N[:800], SIGMA), y,
                             1e-8)
    Kd = rlk.kernel_gaussian_symm(X[:800], Q[:800], N[:800], SIGMA)
    res = np.linalg.norm(Kd @ a_got + 1e-8 * a_got - y) / np.linalg.norm(y)
    assert res < 1e-6
    Kt = rlk.kernel_gaussian(X[800:], X[:800], Q[800:], Q[:800], N[800:], N[:800], SIGMA)
    p_got, p_ref = Kt @ a_got + ym, Kt @ a_ref + ym
    np.testing.assert_allclose(p_got, p_ref, rtol=1e-6, atol=1e-6 * np.abs(p_ref).max())
    mae_got = np.abs(p_got - E[800:]).mean()
    mae_ref = np.abs(p_ref - E[800:]).mean()
    assert abs(mae_got / mae_ref - 1) < 1e-6


@pytest.fixture(scope="module")
def config3_slice():
    from kernelforge_b200 import synthetic
    tr = synthetic.make_molecules(40, 9, 30, seed=20261206)
    te = synthetic.make_molecules(40, 9, 30, seed=20261207)
    X1, Q1, N1 = synthetic.fchl19_batched(tr, dtype=np.float64, device="cuda", chunk=64)
    X2, dX2, Q2, N2 = synthetic.fchl19_batched_grad(te, dtype=np.float64, device="cuda", chunk=4)
    return X1, X2, dX2, Q1, Q2, N1, N2


def test_config3_slice_jacobian(ref, config3_slice):
    from kernelforge_b200 import local_kernels as lk
    rlk, _ = ref
    args = config3_slice
    want = rlk.kernel_gaussian_jacobian(*args, SIGMA)
    assert want.shape == (40, int(3 * args[6].sum()))
    got = lk.kernel_gaussian_jacobian(*args, SIGMA)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-10 * np.abs(want).max())
    got = lk.kernel_gaussian_jacobian(*args, SIGMA, precision="split_f16")
    assert rel_fro(got, want) <= 5e-5


@pytest.fixture(scope="module")
def config4_slice():
    from kernelforge_b200 import synthetic
    mols = synthetic.make_molecules(20, 21, 21, seed=20261208)
    return synthetic.fchl19_batched_grad(mols, dtype=np.float64, device="cuda", chunk=4)


def test_config4_slice_full_symm_rfp(ref, config4_slice):
    from kernelforge_b200 import local_kernels as lk
    rlk, _ = ref
    X, dX, Q, N = config4_slice
    want = rlk.kernel_gaussian_full_symm_rfp(X, dX, Q, N, SIGMA)
    big = 20 + 3 * 20 * 21
    assert want.shape == (big * (big + 1) // 2,)
    got = lk.kernel_gaussian_full_symm_rfp(X, dX, Q, N, SIGMA)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-10 * np.abs(want).max())
    got = lk.kernel_gaussian_full_symm_rfp(X, dX, Q, N, SIGMA, precision="split_f16")
    assert rel_fro(got, want) <= 5e-5
