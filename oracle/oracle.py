"""ctypes front-end of the CPU FP64 oracle (kf_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the kernelforge_b200 package.

Function names and argument orders mirror the reference's pybind module
``kernelforge.local_kernels`` (src/local_kernels_bindings.cpp:759-1537) and
``kernelforge.kernelmath.cho_solve_rfp`` (src/math_bindings.cpp:49-76), so a
test reads the same for the oracle, the reference build and the CUDA path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SRC = os.path.join(_HERE, "kf_oracle.c")
_LIB = os.path.join(_HERE, "libkf_oracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile kf_oracle.c into oracle/libkf_oracle.so (gcc, -O2, OpenMP)."""
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(_SRC):
        subprocess.check_call(
            ["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11", _SRC, "-o", _LIB, "-lm"]
        )
    return _LIB


def _load():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB)
        _lib.kfo_rfp_index_upper.restype = ctypes.c_size_t
        _lib.kfo_rfp_index_upper.argtypes = [ctypes.c_long] * 3
        _lib.kfo_rfp_index_lower.restype = ctypes.c_size_t
        _lib.kfo_rfp_index_lower.argtypes = [ctypes.c_long] * 3
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _naq(n, ma):
    return int(3 * np.clip(np.asarray(n), 0, ma).sum())


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} failed (rc={rc})")


def rfp_index_upper(n, i, j):
    return int(_load().kfo_rfp_index_upper(n, i, j))


def rfp_index_lower(n, i, j):
    return int(_load().kfo_rfp_index_lower(n, i, j))


def full_to_rfp(A, uplo_lower=False):
    A = _d(A)
    n = A.shape[0]
    out = np.zeros(n * (n + 1) // 2)
    _load().kfo_full_to_rfp(_p(A), ctypes.c_long(n), ctypes.c_int(int(uplo_lower)), _p(out))
    return out


def rfp_to_full(arf, n, uplo_lower=False):
    arf = _d(arf)
    out = np.zeros((n, n))
    _load().kfo_rfp_to_full(_p(arf), ctypes.c_long(n), ctypes.c_int(int(uplo_lower)), _p(out))
    return out


def kernel_gaussian(X1, X2, Q1, Q2, N1, N2, sigma):
    X1, X2, Q1, Q2, N1, N2 = _d(X1), _d(X2), _i(Q1), _i(Q2), _i(N1), _i(N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    K = np.zeros((nm1, nm2))
    rc = _load().kfo_kernel_gaussian(
        _p(X1), _p(X2), _p(Q1), _p(Q2), _p(N1), _p(N2), nm1, nm2, ma1, ma2, rep,
        ctypes.c_double(sigma), _p(K))
    _check(rc, "kernel_gaussian")
    return K


def kernel_gaussian_symm(X, Q, N, sigma):
    return kernel_gaussian(X, X, Q, Q, N, N, sigma)


def kernel_gaussian_symm_rfp(X, Q, N, sigma, uplo_lower=False):
    return full_to_rfp(kernel_gaussian_symm(X, Q, N, sigma), uplo_lower)


def kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, sigma):
    X1, X2, dX2, Q1, Q2, N1, N2 = _d(X1), _d(X2), _d(dX2), _i(Q1), _i(Q2), _i(N1), _i(N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    naq2 = _naq(N2, ma2)
    K = np.zeros((nm1, naq2))
    rc = _load().kfo_kernel_gaussian_jacobian(
        _p(X1), _p(X2), _p(dX2), _p(Q1), _p(Q2), _p(N1), _p(N2), nm1, nm2, ma1, ma2, rep, naq2,
        ctypes.c_double(sigma), _p(K))
    _check(rc, "kernel_gaussian_jacobian")
    return K


def kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, sigma):
    X1, X2, dX1, Q1, Q2, N1, N2 = _d(X1), _d(X2), _d(dX1), _i(Q1), _i(Q2), _i(N1), _i(N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    naq1 = _naq(N1, ma1)
    K = np.zeros((naq1, nm2))
    rc = _load().kfo_kernel_gaussian_jacobian_t(
        _p(X1), _p(X2), _p(dX1), _p(Q1), _p(Q2), _p(N1), _p(N2), nm1, nm2, ma1, ma2, rep, naq1,
        ctypes.c_double(sigma), _p(K))
    _check(rc, "kernel_gaussian_jacobian_t")
    return K


def kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma):
    X1, X2, dX1, dX2 = _d(X1), _d(X2), _d(dX1), _d(dX2)
    Q1, Q2, N1, N2 = _i(Q1), _i(Q2), _i(N1), _i(N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    naq1, naq2 = _naq(N1, ma1), _naq(N2, ma2)
    H = np.zeros((naq1, naq2))
    rc = _load().kfo_kernel_gaussian_hessian(
        _p(X1), _p(X2), _p(dX1), _p(dX2), _p(Q1), _p(Q2), _p(N1), _p(N2), nm1, nm2, ma1, ma2,
        rep, naq1, naq2, ctypes.c_double(sigma), _p(H))
    _check(rc, "kernel_gaussian_hessian")
    return H


def kernel_gaussian_hessian_symm(X, dX, Q, N, sigma):
    H = kernel_gaussian_hessian(X, dX, X, dX, Q, Q, N, N, sigma)
    return np.tril(H)


def kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, sigma, uplo_lower=False):
    H = kernel_gaussian_hessian(X, dX, X, dX, Q, Q, N, N, sigma)
    return full_to_rfp(H, uplo_lower)


def kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma):
    X1, X2, dX1, dX2 = _d(X1), _d(X2), _d(dX1), _d(dX2)
    Q1, Q2, N1, N2 = _i(Q1), _i(Q2), _i(N1), _i(N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    naq1, naq2 = _naq(N1, ma1), _naq(N2, ma2)
    K = np.zeros((nm1 + naq1, nm2 + naq2))
    rc = _load().kfo_kernel_gaussian_full(
        _p(X1), _p(X2), _p(dX1), _p(dX2), _p(Q1), _p(Q2), _p(N1), _p(N2), nm1, nm2, ma1, ma2,
        rep, naq1, naq2, ctypes.c_double(sigma), _p(K))
    _check(rc, "kernel_gaussian_full")
    return K


def kernel_gaussian_full_symm(X, dX, Q, N, sigma):
    return kernel_gaussian_full(X, dX, X, dX, Q, Q, N, N, sigma)


def kernel_gaussian_full_symm_rfp(X, dX, Q, N, sigma, uplo_lower=False):
    return full_to_rfp(kernel_gaussian_full_symm(X, dX, Q, N, sigma), uplo_lower)


def cho_solve_rfp(K_rfp, y, l2=0.0, uplo_lower=False):
    """Solve (K + l2 I) alpha = y; K_rfp (float64, contiguous) is overwritten with
    the Cholesky factor, like the reference.  Raises RuntimeError on info != 0."""
    y = _d(y)
    n = y.shape[0]
    if K_rfp.ndim != 1 or K_rfp.shape[0] != n * (n + 1) // 2:
        raise RuntimeError("K_rfp length must be n*(n+1)/2")
    arf = K_rfp if (K_rfp.dtype == np.float64 and K_rfp.flags.c_contiguous) else _d(K_rfp)
    alpha = np.zeros(n)
    info = _load().kfo_cho_solve_rfp(_p(arf), _p(y), ctypes.c_long(n), ctypes.c_double(l2),
                                     ctypes.c_int(int(uplo_lower)), _p(alpha))
    if info != 0:
        raise RuntimeError(f"DPFTRF failed, info={info}")
    return alpha
