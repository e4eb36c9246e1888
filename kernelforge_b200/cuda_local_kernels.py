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
           "kernel_gaussian_full_symm", "kernel_gaussian_full_symm_rfp", "compute_alpha_desc",
           "kernel_gaussian_full_matvec"]


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
    if isinstance(X, torch.Tensor) and X.device.type == "cpu":
        return _symm_host(X, Q, N, sigma, precision, layout, out_dtype)
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


def _symm_host(X, Q, N, sigma, precision, layout, out_dtype):
    """X a float32 CPU tensor (page-locked for overlap): the library copies it
    in chunks of molecules while the tensor cores start on the molecules that
    have arrived; the output is on the current CUDA device."""
    import torch
    if X.dtype != torch.float32 or X.dim() != 3 or not X.is_contiguous():
        raise RuntimeError("X must be a contiguous float32 tensor (nm, ma, rep)")
    check_sigma(sigma)
    Qh, Nh = host_i32(Q), host_i32(N)
    nm, ma, rep = X.shape
    count = nm * nm if layout == _lib.KFB_DENSE else nm * (nm + 1) // 2
    out = torch.empty((count,), dtype=out_dtype, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_symm_host(
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


def _check_coef(t, name):
    """Coefficient tensors: float32 as in the reference, or float64 (kept in FP64)."""
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise RuntimeError(f"{name} must be a CUDA tensor")
    if t.dtype not in (torch.float32, torch.float64):
        raise RuntimeError(f"{name} must be float32 (or float64)")


def compute_alpha_desc(dX, N, alpha_F):
    """alpha_desc (nm, max_atoms, rep): alpha_desc[b, i, :] =
    dX[b, i, :, :3 N[b]] @ alpha_F[off_b : off_b + 3 N[b]] (zero for padded atoms),
    accumulated in FP64; float32 like the reference, float64 when alpha_F is
    float64.  Reference: compute_alpha_desc_local_cu
    (src/cuda_local_kernels.cu:2348-2379)."""
    require_cuda()
    import torch
    _check_x(dX, "dX")
    _check_coef(alpha_F, "alpha_F")
    Nh = host_i32(N)
    if dX.dim() != 4 or dX.shape[3] != 3 * dX.shape[1]:
        raise RuntimeError("dX must be (nm, max_atoms, rep, 3*max_atoms)")
    nm, ma, rep = dX.shape[0], dX.shape[1], dX.shape[2]
    if Nh.shape != (nm,):
        raise RuntimeError("N length mismatch")
    naq = _naq(Nh, ma)
    if alpha_F.numel() < naq:
        raise RuntimeError("alpha_F length mismatch")
    al = alpha_F.reshape(-1).to(torch.float64)
    out = torch.empty((nm, ma, rep), dtype=torch.float64, device=dX.device)
    _lib.check(_lib.lib().kfb_local_alpha_desc(
        dX.data_ptr(), None, Nh.ctypes.data, nm, ma, rep, _lib.KFB_F32, al.data_ptr(),
        out.data_ptr(), stream_handle()))
    return out if alpha_F.dtype == torch.float64 else out.float()


def kernel_gaussian_full_matvec(X_q, dX_q, Q_q, N_q, X_t, Q_t, N_t, alpha_E, alpha_desc_F,
                                sigma):
    """Contracted energy+force prediction: (E_pred (nm_q,), F_pred (naq_q,)), equal to
    kernel_gaussian_full(query, training) @ [alpha_E; alpha_F] without forming that
    matrix (FP64 arithmetic inside); float32 like the reference, float64 when
    alpha_desc_F is float64.  Reference: kernel_gaussian_full_matvec_local_cu
    (src/cuda_local_kernels.cu:2380-2619)."""
    require_cuda()
    import torch
    _check_x(X_q, "X_q")
    _check_x(dX_q, "dX_q")
    _check_x(X_t, "X_t")
    _check_coef(alpha_E, "alpha_E")
    _check_coef(alpha_desc_F, "alpha_desc_F")
    check_sigma(sigma)
    Qq, Nq, Qt, Nt = host_i32(Q_q), host_i32(N_q), host_i32(Q_t), host_i32(N_t)
    nm1, ma1, rep = X_q.shape
    nm2, ma2, rep2 = X_t.shape
    if rep2 != rep or tuple(dX_q.shape) != (nm1, ma1, rep, 3 * ma1):
        raise RuntimeError("X_q / dX_q / X_t shape mismatch")
    if tuple(alpha_desc_F.shape) != (nm2, ma2, rep) or alpha_E.numel() != nm2:
        raise RuntimeError("alpha_E / alpha_desc_F shape mismatch")
    if Qq.shape != (nm1, ma1) or Nq.shape != (nm1,) or Qt.shape != (nm2, ma2) \
            or Nt.shape != (nm2,):
        raise RuntimeError("Q / N shape mismatch")
    naq1 = _naq(Nq, ma1)
    ad = alpha_desc_F.contiguous().to(torch.float64)
    ae = alpha_E.reshape(-1).to(torch.float64)
    e = torch.empty(nm1, dtype=torch.float64, device=X_q.device)
    f = torch.empty(max(naq1, 1), dtype=torch.float64, device=X_q.device)
    _lib.check(_lib.lib().kfb_local_matvec(
        X_q.data_ptr(), dX_q.data_ptr(), X_t.data_ptr(), ad.data_ptr(), ae.data_ptr(),
        Qq.ctypes.data, Qt.ctypes.data, Nq.ctypes.data, Nt.ctypes.data, nm1, nm2, ma1, ma2,
        rep, float(sigma), _lib.KFB_F32, e.data_ptr(), f.data_ptr(), stream_handle()))
    if alpha_desc_F.dtype == torch.float64:
        return e, f[:naq1]
    return e.float(), f[:naq1].float()
