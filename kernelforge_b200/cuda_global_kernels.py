"""Drop-in for ``kernelforge.cuda_global_kernels.rfp_potrf`` / ``rfp_potrs``
(src/cuda_global_kernels_bindings.cpp:410-461) plus the mixed-precision KRR
solve that replaces the reference's FP32-solve-with-CPU-FP64-fallback
(models/cuda_local_krr.py:640-675).
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._device import require_cuda, stream_handle

__all__ = ["rfp_potrf", "rfp_potrs", "krr_solve_mixed"]


def _uplo(uplo) -> int:
    u = str(uplo).upper()
    if u not in ("L", "U"):
        raise ValueError("uplo must be 'L' or 'U'")
    return _lib.KFB_RFP_L if u == "L" else _lib.KFB_RFP_U


def _dt(t):
    import torch
    if t.dtype == torch.float32:
        return _lib.KFB_F32
    if t.dtype == torch.float64:
        return _lib.KFB_F64
    raise RuntimeError("K_rfp must be float32 (or float64)")


def rfp_potrf(K_rfp, N, l2=0.0, uplo="L"):
    """In-place Cholesky of the RFP matrix K_rfp + l2 I (TRANSR='N').  Returns
    info: 0, or k > 0 if the leading minor of order k is not positive definite."""
    require_cuda()
    if not K_rfp.is_cuda or not K_rfp.is_contiguous():
        raise RuntimeError("K_rfp must be a contiguous CUDA tensor")
    n = int(N)
    if K_rfp.numel() != n * (n + 1) // 2:
        raise RuntimeError("K_rfp must have N*(N+1)/2 elements")
    info = ctypes.c_int(0)
    _lib.check(_lib.lib().kfb_rfp_potrf(K_rfp.data_ptr(), n, float(l2), _uplo(uplo), _dt(K_rfp),
                                        ctypes.byref(info), stream_handle()))
    return int(info.value)


def rfp_potrs(L_rfp, B, uplo="L"):
    """Solve with the factor from rfp_potrf; B (N, nrhs) column-major
    (ldb = N; contiguous (N,) or (N, 1) tensors) is overwritten with X."""
    require_cuda()
    if not B.is_cuda or not B.is_contiguous():
        raise RuntimeError("B must be a contiguous CUDA tensor")
    n = B.shape[0]
    nrhs = 1 if B.dim() == 1 else B.shape[1]
    if L_rfp.numel() != n * (n + 1) // 2:
        raise RuntimeError("L_rfp / B size mismatch")
    if B.dtype != L_rfp.dtype:
        raise RuntimeError("B and L_rfp must have the same dtype")
    _lib.check(_lib.lib().kfb_rfp_potrs(L_rfp.data_ptr(), B.data_ptr(), n, nrhs, _uplo(uplo),
                                        _dt(L_rfp), stream_handle()))


def krr_solve_mixed(K_rfp, y, l2=0.0, uplo="L", tol=1e-10, maxit=500, *, lambda_floor=False,
                    factor="fp64"):
    """(K + l2 I) alpha = y with an FP32 RFP kernel matrix (not modified): a
    Cholesky factor as preconditioner (an FP32-class one with the dominant
    eigenpair deflated, or an FP64-class one), FP64 conjugate-gradient
    refinement of residuals against K.  Returns (alpha float64, info dict).

    Raises RuntimeError if K + l2 I is indefinite at FP32 storage precision;
    with ``lambda_floor=True`` l2 is raised in x10 steps until it is not, and
    info["lambda_eff"] reports the value used.

    ``factor``: precision of the Cholesky factor behind the refinement, both
    this library's tensor-core factorisation (FP64 diagonal blocks and panels,
    int8 digit-plane trailing updates): "fp64" (default) an FP64-class factor
    (6 digit planes of 7 bits), one or two refinement steps; "fp32" an
    FP32-class factor (4 planes, FP32 diagonal blocks), about six steps.  At
    n = 10,000 the whole solve takes 15.9 ms and 22.8 ms respectively on one
    B200.
    """
    require_cuda()
    import torch
    if K_rfp.dtype != torch.float32 or not K_rfp.is_cuda or not K_rfp.is_contiguous():
        raise RuntimeError("K_rfp must be a contiguous float32 CUDA tensor")
    yd = y.to(device=K_rfp.device, dtype=torch.float64).contiguous()
    n = yd.numel()
    if K_rfp.numel() != n * (n + 1) // 2:
        raise RuntimeError("K_rfp must have n*(n+1)/2 elements")
    alpha = torch.empty((n,), dtype=torch.float64, device=K_rfp.device)
    info = _lib.SolveInfo()
    if factor not in ("fp32", "fp64"):
        raise ValueError("factor must be 'fp32' or 'fp64'")
    flags = (_lib.KFB_SOLVE_LAMBDA_FLOOR if lambda_floor else 0) | \
        (_lib.KFB_SOLVE_FP64_FACTOR if factor == "fp64" else 0)
    st = _lib.lib().kfb_krr_solve_mixed(K_rfp.data_ptr(), yd.data_ptr(), n, float(l2),
                                        _uplo(uplo), float(tol), int(maxit), flags,
                                        alpha.data_ptr(), ctypes.byref(info), stream_handle())
    res = {"iterations": info.iterations, "factor_info": info.factor_info, "shift": info.shift,
           "rel_residual": info.rel_residual, "used_cg": bool(info.used_cg),
           "lambda_eff": info.lambda_eff}
    if st == _lib.KFB_ERR_NOT_PD:
        raise RuntimeError(_lib.lib().kfb_last_error().decode())
    if st != _lib.KFB_OK and st != _lib.KFB_ERR_NO_CONVERGENCE:
        _lib.check(st)
    res["converged"] = st == _lib.KFB_OK
    return alpha, res
