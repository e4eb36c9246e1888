"""Drop-in for the reference's ``kernelforge.cuda_local_kernels`` module (the
training-kernel part): torch CUDA tensors in, torch CUDA tensors out, the same
names, arguments, shapes and dtypes as src/cuda_local_kernels_bindings.cpp:
725-1048 (stub python/kernelforge/cuda_local_kernels.pyi).

* X float32 (nm, max_atoms, rep), dX float32 (nm, max_atoms, rep, 3*max_atoms),
  Q / N int32 (CUDA or host; they are read on the host to plan the label
  buckets, as the reference does).
* Scalar kernels run on the tcgen05 tensor cores by default
  (``precision="split_f16"``: two-term fp16 split of the descriptors, FP32
  accumulation); ``precision="fp32"`` / ``"fp64"`` select CUDA-core paths.
* RFP outputs use TRANSR='N', Fortran UPLO='L' (unpack with
  ``kernelmath.rfp_to_full(K, n, uplo='U')``) and match ``rfp_potrf``'s default.
* Work is enqueued on torch's current stream.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._device import check_sigma, host_i32, require_cuda, stream_handle

__all__ = ["kernel_gaussian_rect", "kernel_gaussian_symm", "kernel_gaussian_symm_rfp",
           "kernel_gaussian_full_symm", "kernel_gaussian_full_symm_rfp"]


def _check_x(X, name):
    import torch
    if not isinstance(X, torch.Tensor) or not X.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if X.dtype != torch.float32:
        raise RuntimeError(f"{name} must be float32")
    if not X.is_contiguous():
        raise RuntimeError(f"{name} must be contiguous")


def _prec(precision):
    if precision not in _lib.PREC:
        raise ValueError(f"precision must be one of {sorted(_lib.PREC)}")
    return _lib.PREC[precision]


def _naq(N, ma):
    return int(3 * np.clip(N.astype(np.int64), 0, ma).sum())


def kernel_gaussian_rect(X_q, Q_q, N_q, X_t, Q_t, N_t, sigma, *, precision="split_f16"):
    """K (nm_q, nm_t) float64 for two molecule sets."""
    require_cuda()
    import torch
    _check_x(X_q, "X_q")
    _check_x(X_t, "X_t")
    check_sigma(sigma)
    Qq, Nq, Qt, Nt = host_i32(Q_q), host_i32(N_q), host_i32(Q_t), host_i32(N_t)
    nm1, ma1, rep = X_q.shape
    nm2, ma2, _ = X_t.shape
    out = torch.empty((nm1, nm2), dtype=torch.float64, device=X_q.device)
    _lib.check(_lib.lib().kfb_kernel_gaussian(
        X_q.data_ptr(), X_t.data_ptr(), Qq.ctypes.data, Qt.ctypes.data, Nq.ctypes.data,
        Nt.ctypes.data, nm1, nm2, ma1, ma2, rep, float(sigma), _lib.KFB_F32, _prec(precision),
        _lib.KFB_F64, out.data_ptr(), stream_handle()))
    return out


def _symm(X, Q, N, sigma, precision, layout, out_dtype):
    require_cuda()
    import torch
    _check_x(X, "X")
    check_sigma(sigma)
    Qh, Nh = host_i32(Q), host_i32(N)
    nm, ma, rep = X.shape
    count = nm * nm if layout == _lib.KFB_DENSE else nm * (nm + 1) // 2
    out = torch.empty((count,), dtype=out_dtype, device=X.device)
    _lib.check(_lib.lib().kfb_kernel_gaussian_symm(
        X.data_ptr(), Qh.ctypes.data, Nh.ctypes.data, nm, ma, rep, float(sigma), _lib.KFB_F32,
        _prec(precision), layout, _lib.KFB_F64 if out_dtype == torch.float64 else _lib.KFB_F32,
        out.data_ptr(), stream_handle()))
    return out.view(nm, nm) if layout == _lib.KFB_DENSE else out


def kernel_gaussian_symm(X, Q, N, sigma, *, precision="split_f16"):
    """Symmetric K (nm, nm) float64, both triangles."""
    import torch
    return _symm(X, Q, N, sigma, precision, _lib.KFB_DENSE, torch.float64)


def kernel_gaussian_symm_rfp(X, Q, N, sigma, *, precision="split_f16"):
    """Symmetric K in RFP (TRANSR='N', Fortran UPLO='L'), float32 (nm(nm+1)/2,)."""
    import torch
    return _symm(X, Q, N, sigma, precision, _lib.KFB_RFP_L, torch.float32)


def _full_symm(X, dX, Q, N, sigma, precision, layout):
    require_cuda()
    import torch
    _check_x(X, "X")
    _check_x(dX, "dX")
    check_sigma(sigma)
    Qh, Nh = host_i32(Q), host_i32(N)
    nm, ma, rep = X.shape
    if tuple(dX.shape) != (nm, ma, rep, 3 * ma):
        raise RuntimeError("dX shape mismatch")
    naq = _naq(Nh, ma)
    big = nm + naq
    count = big * big if layout == _lib.KFB_DENSE else big * (big + 1) // 2
    out = torch.empty((count,), dtype=torch.float32, device=X.device)
    _lib.check(_lib.lib().kfb_kernel_gaussian_full_symm(
        X.data_ptr(), dX.data_ptr(), Qh.ctypes.data, Nh.ctypes.data, nm, ma, rep, naq,
        float(sigma), _lib.KFB_F32, _prec(precision), layout, out.data_ptr(), stream_handle()))
    return out.view(big, big) if layout == _lib.KFB_DENSE else out


def kernel_gaussian_full_symm(X, dX, Q, N, sigma, *, precision="split_f16"):
    """Symmetric energy+force K (nm+naq, nm+naq) float32, fully filled."""
    return _full_symm(X, dX, Q, N, sigma, precision, _lib.KFB_DENSE)


def kernel_gaussian_full_symm_rfp(X, dX, Q, N, sigma, *, precision="split_f16"):
    """Symmetric energy+force K in RFP (TRANSR='N', Fortran UPLO='L'), float32."""
    return _full_symm(X, dX, Q, N, sigma, precision, _lib.KFB_RFP_L)
