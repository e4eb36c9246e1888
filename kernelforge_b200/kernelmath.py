"""Drop-in for the RFP part of the reference's ``kernelforge.kernelmath`` module.

``cho_solve_rfp``, ``full_to_rfp`` and ``rfp_to_full`` keep the reference's
names, arguments, defaults and in/out conventions (src/math_bindings.cpp:49-180,
stub python/kernelforge/kernelmath.pyi):

* arrays are C-order NumPy arrays; the ``uplo`` letter of full_to_rfp /
  rfp_to_full names the C-order triangle, so it is swapped before it reaches
  the Fortran RFP convention ('U' in Python is Fortran 'L'),
  src/math_bindings.cpp:85-121;
* cho_solve_rfp uses TRANSR='N', Fortran UPLO='U' (the packing the local_kernels
  *_rfp functions produce) and overwrites K_rfp with the Cholesky factor when
  K_rfp is a C-contiguous float64 array.

The factorisation and solves run in FP64 on the GPU through libkfb.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._device import require_cuda, stream_handle, to_device

__all__ = ["cho_solve_rfp", "full_to_rfp", "rfp_to_full"]


def _norm_uplo(u) -> str:
    u = str(u)
    return "L" if u in ("l", "L") else "U"


def _norm_tr(t) -> str:
    t = str(t)
    return "T" if t in ("t", "T") else "N"


def _rfp_shape(n: int):
    """(rows, cols) of the column-major RFP matrix for TRANSR='N'."""
    return (n, (n + 1) // 2) if n % 2 else (n + 1, n // 2)


def _n_to_t(arf_n: np.ndarray, n: int) -> np.ndarray:
    rows, cols = _rfp_shape(n)
    return np.ascontiguousarray(arf_n.reshape(cols, rows).T).ravel()


def _t_to_n(arf_t: np.ndarray, n: int) -> np.ndarray:
    rows, cols = _rfp_shape(n)
    return np.ascontiguousarray(arf_t.reshape(rows, cols).T).ravel()


def full_to_rfp(A, uplo="U", transr="N"):
    """Symmetric (n, n) C-order matrix -> RFP vector of length n(n+1)/2."""
    A = np.ascontiguousarray(A, dtype=np.float64)
    if A.ndim != 2 or A.shape[0] != A.shape[1]:
        raise RuntimeError("A must be square (n x n).")
    uplo, transr = _norm_uplo(uplo), _norm_tr(transr)
    n = A.shape[0]
    # C-order triangle 'U' is the Fortran 'L' triangle of the same buffer
    fortran = _lib.KFB_RFP_L if uplo == "U" else _lib.KFB_RFP_U
    if n == 0:
        return np.zeros((0,))
    require_cuda()
    import torch
    # the reference packs only the named C-order triangle of A
    src = np.triu(A) + np.triu(A, 1).T if uplo == "U" else np.tril(A) + np.tril(A, -1).T
    a = to_device(src, torch.float64)
    out = torch.empty((n * (n + 1) // 2,), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kfb_full_to_rfp(a.data_ptr(), n, fortran, _lib.KFB_F64,
                                          out.data_ptr(), stream_handle()))
    res = out.cpu().numpy()
    return _n_to_t(res, n) if transr == "T" else res


def rfp_to_full(ARF, n, uplo="U", transr="N"):
    """RFP vector -> symmetric (n, n) C-order matrix (both triangles filled)."""
    ARF = np.ascontiguousarray(ARF, dtype=np.float64)
    if ARF.ndim != 1:
        raise RuntimeError("ARF must be a 1-D array.")
    n = int(n)
    if ARF.shape[0] != n * (n + 1) // 2:
        raise RuntimeError("ARF length must be n*(n+1)/2.")
    uplo, transr = _norm_uplo(uplo), _norm_tr(transr)
    fortran = _lib.KFB_RFP_L if uplo == "U" else _lib.KFB_RFP_U
    if n == 0:
        return np.zeros((0, 0))
    if transr == "T":
        ARF = _t_to_n(ARF, n)
    require_cuda()
    import torch
    a = to_device(ARF, torch.float64)
    out = torch.empty((n, n), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kfb_rfp_to_full(a.data_ptr(), n, fortran, _lib.KFB_F64,
                                          out.data_ptr(), stream_handle()))
    return out.cpu().numpy()


def cho_solve_rfp(K_rfp, y, l2=0.0):
    """Solve (K + l2 I) alpha = y, K in RFP (TRANSR='N', Fortran UPLO='U').
    K_rfp is overwritten with the Cholesky factor (pass K_rfp.copy() to keep it).
    Raises RuntimeError if the matrix is not positive definite."""
    arr = np.asarray(K_rfp)
    y = np.ascontiguousarray(y, dtype=np.float64)
    if arr.ndim != 1 or y.ndim != 1:
        raise RuntimeError("K_rfp must be 1D RFP and y must be 1D")
    n = y.shape[0]
    if arr.shape[0] != n * (n + 1) // 2:
        raise RuntimeError("K_rfp length must be n*(n+1)/2")
    if n <= 0:
        raise RuntimeError("n must be > 0")
    require_cuda()
    import torch
    k = to_device(np.ascontiguousarray(arr, dtype=np.float64), torch.float64)
    yd = to_device(y, torch.float64)
    alpha = torch.empty((n,), dtype=torch.float64, device="cuda")
    info = ctypes.c_int(0)
    st = _lib.lib().kfb_cho_solve_rfp(k.data_ptr(), yd.data_ptr(), n, float(l2), _lib.KFB_RFP_U,
                                      alpha.data_ptr(), ctypes.byref(info), stream_handle())
    if st == _lib.KFB_ERR_NOT_PD:
        raise RuntimeError(f"DPFTRF failed, info={info.value}")
    _lib.check(st)
    if isinstance(K_rfp, np.ndarray) and K_rfp.dtype == np.float64 and K_rfp.flags.c_contiguous \
            and K_rfp.flags.writeable:
        K_rfp[...] = k.cpu().numpy()
    return alpha.cpu().numpy()
