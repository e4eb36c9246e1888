"""Drop-in for the reference's ``kernelforge.local_kernels`` module.

Same function names, argument names/order, shapes, dtypes (float64 NumPy
outputs) and exceptions as the pybind11 module (src/local_kernels_bindings.cpp:
759-1537, stub python/kernelforge/local_kernels.pyi).  The work runs on the GPU
through libkfb: inputs are copied to the device, the kernel runs, the result is
copied back.  Every function takes one extra keyword-only argument:

``precision``: ``"fp64"`` (default; FP64 CUDA cores, matches the reference's
FP64 CPU results to rounding), ``"fp32"`` (FP32 CUDA cores) or ``"split_f16"``
(scalar kernels only: tcgen05 tensor cores with a two-term fp16 split of the
descriptors and FP32 accumulation; derivative kernels then use FP32).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._device import check_sigma, host_i32, require_cuda, stream_handle, to_device

__all__ = [
    "kernel_gaussian", "kernel_gaussian_symm", "kernel_gaussian_symm_rfp",
    "kernel_gaussian_jacobian", "kernel_gaussian_jacobian_t", "kernel_gaussian_hessian",
    "kernel_gaussian_hessian_symm", "kernel_gaussian_hessian_symm_rfp", "kernel_gaussian_full",
    "kernel_gaussian_full_symm", "kernel_gaussian_full_symm_rfp",
    "kernel_gaussian_local_compute_alpha_desc", "kernel_gaussian_local_jacobian_t_matvec",
    "kernel_gaussian_local_hessian_matvec", "kernel_gaussian_local_full_matvec",
]


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _prec(precision: str) -> int:
    if precision not in _lib.PREC:
        raise ValueError(f"precision must be one of {sorted(_lib.PREC)}")
    return _lib.PREC[precision]


def _deriv_dtype(precision: str):
    import torch
    return (torch.float64, _lib.KFB_F64) if precision == "fp64" else (torch.float32, _lib.KFB_F32)


def _naq(N, ma):
    return int(3 * np.clip(N.astype(np.int64), 0, ma).sum())


def _check_scalar_shapes(X1, X2, Q1, Q2, N1, N2):
    if X1.ndim != 3 or X2.ndim != 3 or Q1.ndim != 2 or Q2.ndim != 2 or N1.ndim != 1 or N2.ndim != 1:
        raise ValueError(
            "Expect shapes: X1(nm1,max_atoms1,rep), X2(nm2,max_atoms2,rep), Q1(nm1,max_atoms1), "
            "Q2(nm2,max_atoms2), N1(nm1), N2(nm2).")
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    if X2.shape[2] != rep:
        raise ValueError("X2 rep_size mismatch.")
    if Q1.shape != (nm1, ma1):
        raise ValueError("Q1 shape mismatch.")
    if Q2.shape != (nm2, ma2):
        raise ValueError("Q2 shape mismatch.")
    if N1.shape[0] != nm1:
        raise ValueError("N1 length mismatch.")
    if N2.shape[0] != nm2:
        raise ValueError("N2 length mismatch.")


def _check_symm_shapes(X, Q, N):
    if X.ndim != 3 or Q.ndim != 2 or N.ndim != 1:
        raise ValueError("Expect shapes: X(nm,max_atoms,rep), Q(nm,max_atoms), N(nm).")
    nm, ma, _ = X.shape
    if Q.shape != (nm, ma):
        raise ValueError("Q shape mismatch.")
    if N.shape[0] != nm:
        raise ValueError("N length mismatch.")


def _check_dX(dX, X, name):
    nm, ma, rep = X.shape
    if dX.ndim != 4 or dX.shape != (nm, ma, rep, 3 * ma):
        raise ValueError(f"{name} shape mismatch.")


# --------------------------------------------------------------------------
# scalar kernels
# --------------------------------------------------------------------------

def kernel_gaussian(X1, X2, Q1, Q2, N1, N2, sigma, *, precision="fp64"):
    """K[a, b] = sum over same-label atom pairs of exp(-|x1 - x2|^2 / (2 sigma^2)),
    shape (nm1, nm2) float64.  Reference: src/local_kernels.cpp:155-298."""
    X1, X2 = np.asarray(X1), np.asarray(X2)
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    _check_scalar_shapes(X1, X2, Q1, Q2, N1, N2)
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    xt = torch.float32 if precision == "fp32" else torch.float64
    x1 = to_device(_f64(X1), xt)
    x2 = to_device(_f64(X2), xt)
    out = torch.empty((nm1, nm2), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian(
        x1.data_ptr(), x2.data_ptr(), Q1.ctypes.data, Q2.ctypes.data, N1.ctypes.data,
        N2.ctypes.data, nm1, nm2, ma1, ma2, rep, float(sigma),
        _lib.KFB_F64 if xt == torch.float64 else _lib.KFB_F32, prec, _lib.KFB_F64,
        out.data_ptr(), stream_handle()))
    return out.cpu().numpy()


def _symm(X, Q, N, sigma, precision, layout):
    X = np.asarray(X)
    Q, N = host_i32(Q), host_i32(N)
    _check_symm_shapes(X, Q, N)
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    nm, ma, rep = X.shape
    xt = torch.float32 if precision == "fp32" else torch.float64
    x = to_device(_f64(X), xt)
    count = nm * nm if layout == _lib.KFB_DENSE else nm * (nm + 1) // 2
    out = torch.empty((count,), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_symm(
        x.data_ptr(), Q.ctypes.data, N.ctypes.data, nm, ma, rep, float(sigma),
        _lib.KFB_F64 if xt == torch.float64 else _lib.KFB_F32, prec, layout, _lib.KFB_F64,
        out.data_ptr(), stream_handle()))
    res = out.cpu().numpy()
    return res.reshape(nm, nm) if layout == _lib.KFB_DENSE else res


def kernel_gaussian_symm(X, Q, N, sigma, *, precision="fp64"):
    """Symmetric kernel, both triangles, (nm, nm) float64.
    Reference: src/local_kernels.cpp:584-758."""
    return _symm(X, Q, N, sigma, precision, _lib.KFB_DENSE)


def kernel_gaussian_symm_rfp(X, Q, N, sigma, *, precision="fp64"):
    """Symmetric kernel in RFP (TRANSR='N', Fortran UPLO='U'), length nm(nm+1)/2.
    Reference: src/local_kernels.cpp:403-577."""
    return _symm(X, Q, N, sigma, precision, _lib.KFB_RFP_U)


# --------------------------------------------------------------------------
# derivative kernels
# --------------------------------------------------------------------------

def kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, sigma, *, precision="fp64"):
    """+dK/dR2, shape (nm1, naq2).  Reference: src/local_kernels.cpp:791-974."""
    X1, X2, dX2 = np.asarray(X1), np.asarray(X2), np.asarray(dX2)
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    if X1.ndim != 3 or X2.ndim != 3 or dX2.ndim != 4 or Q1.ndim != 2 or Q2.ndim != 2 \
            or N1.ndim != 1 or N2.ndim != 1:
        raise ValueError("Expect shapes: X1(nm1,max_atoms1,rep), X2(nm2,max_atoms2,rep), "
                         "dX2(nm2,max_atoms2,rep,3*max_atoms2), Q1, Q2, N1, N2.")
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    if X2.shape[2] != rep:
        raise ValueError("X2 shape mismatch.")
    _check_dX(dX2, X2, "dX2")
    _check_scalar_shapes(X1, X2, Q1, Q2, N1, N2)
    naq2 = _naq(N2, ma2)
    if naq2 <= 0:
        return np.zeros((nm1, 0))
    if nm1 <= 0 or ma1 <= 0 or rep <= 0:
        raise ValueError("All dims must be positive.")
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    dt, kdt = _deriv_dtype(precision)
    x1, x2, dx2 = to_device(_f64(X1), dt), to_device(_f64(X2), dt), to_device(_f64(dX2), dt)
    out = torch.empty((nm1, naq2), dtype=dt, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_jacobian(
        x1.data_ptr(), x2.data_ptr(), dx2.data_ptr(), Q1.ctypes.data, Q2.ctypes.data,
        N1.ctypes.data, N2.ctypes.data, nm1, nm2, ma1, ma2, rep, naq2, float(sigma), kdt, prec,
        out.data_ptr(), stream_handle()))
    return out.double().cpu().numpy()


def kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, sigma, *, precision="fp64"):
    """+dK/dR1, shape (naq1, nm2); equals -kernel_gaussian_jacobian(X2, X1, dX1, ...).T.
    Reference: src/local_kernels.cpp:991-1166."""
    X1, X2, dX1 = np.asarray(X1), np.asarray(X2), np.asarray(dX1)
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    if X1.ndim != 3 or X2.ndim != 3 or dX1.ndim != 4 or Q1.ndim != 2 or Q2.ndim != 2 \
            or N1.ndim != 1 or N2.ndim != 1:
        raise ValueError("Expect shapes: X1(nm1,max_atoms1,rep), dX1(nm1,max_atoms1,rep,"
                         "3*max_atoms1), X2(nm2,max_atoms2,rep), Q1, Q2, N1, N2.")
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    if X2.shape[2] != rep:
        raise ValueError("X2 shape mismatch.")
    _check_dX(dX1, X1, "dX1")
    _check_scalar_shapes(X1, X2, Q1, Q2, N1, N2)
    naq1 = _naq(N1, ma1)
    if naq1 <= 0:
        return np.zeros((0, nm2))
    if nm2 <= 0 or ma2 <= 0 or rep <= 0:
        raise ValueError("All dims must be positive.")
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    dt, kdt = _deriv_dtype(precision)
    x1, x2, dx1 = to_device(_f64(X1), dt), to_device(_f64(X2), dt), to_device(_f64(dX1), dt)
    out = torch.empty((naq1, nm2), dtype=dt, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_jacobian_t(
        x1.data_ptr(), dx1.data_ptr(), x2.data_ptr(), Q1.ctypes.data, Q2.ctypes.data,
        N1.ctypes.data, N2.ctypes.data, nm1, nm2, ma1, ma2, rep, naq1, float(sigma), kdt, prec,
        out.data_ptr(), stream_handle()))
    return out.double().cpu().numpy()


def _check_pair_deriv(X1, dX1, X2, dX2, Q1, Q2, N1, N2):
    if X1.ndim != 3 or X2.ndim != 3 or dX1.ndim != 4 or dX2.ndim != 4 or Q1.ndim != 2 \
            or Q2.ndim != 2 or N1.ndim != 1 or N2.ndim != 1:
        raise ValueError("Expect shapes: X1(nm1,max_atoms1,rep), dX1(nm1,max_atoms1,rep,"
                         "3*max_atoms1), X2(nm2,max_atoms2,rep), dX2(nm2,max_atoms2,rep,"
                         "3*max_atoms2), Q1, Q2, N1, N2.")
    if X2.shape[2] != X1.shape[2]:
        raise ValueError("X2 rep mismatch.")
    _check_dX(dX1, X1, "dX1")
    _check_dX(dX2, X2, "dX2")
    _check_scalar_shapes(X1, X2, Q1, Q2, N1, N2)


def kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma, *, precision="fp64"):
    """Hessian kernel, shape (naq1, naq2).  Reference: src/local_kernels.cpp:1171-1419."""
    X1, X2, dX1, dX2 = map(np.asarray, (X1, X2, dX1, dX2))
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    _check_pair_deriv(X1, dX1, X2, dX2, Q1, Q2, N1, N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    naq1, naq2 = _naq(N1, ma1), _naq(N2, ma2)
    if naq1 == 0 or naq2 == 0:
        return np.zeros((naq1, naq2))
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    dt, kdt = _deriv_dtype(precision)
    x1, x2 = to_device(_f64(X1), dt), to_device(_f64(X2), dt)
    dx1, dx2 = to_device(_f64(dX1), dt), to_device(_f64(dX2), dt)
    out = torch.empty((naq1, naq2), dtype=dt, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_hessian(
        x1.data_ptr(), dx1.data_ptr(), x2.data_ptr(), dx2.data_ptr(), Q1.ctypes.data,
        Q2.ctypes.data, N1.ctypes.data, N2.ctypes.data, nm1, nm2, ma1, ma2, rep, naq1, naq2,
        float(sigma), kdt, prec, out.data_ptr(), stream_handle()))
    return out.double().cpu().numpy()


def _hess_symm(X, dX, Q, N, sigma, precision, layout):
    X, dX = np.asarray(X), np.asarray(dX)
    Q, N = host_i32(Q), host_i32(N)
    if X.ndim != 3 or dX.ndim != 4 or Q.ndim != 2 or N.ndim != 1:
        raise ValueError("Expect shapes: X(nm,max_atoms,rep), dX(nm,max_atoms,rep,3*max_atoms), "
                         "Q(nm,max_atoms), N(nm).")
    _check_dX(dX, X, "dX")
    _check_symm_shapes(X, Q, N)
    nm, ma, rep = X.shape
    naq = _naq(N, ma)
    if naq == 0:
        return np.zeros((0, 0)) if layout == _lib.KFB_DENSE else np.zeros((0,))
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    dt, kdt = _deriv_dtype(precision)
    x, dx = to_device(_f64(X), dt), to_device(_f64(dX), dt)
    count = naq * naq if layout == _lib.KFB_DENSE else naq * (naq + 1) // 2
    out = torch.empty((count,), dtype=dt, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_hessian_symm(
        x.data_ptr(), dx.data_ptr(), Q.ctypes.data, N.ctypes.data, nm, ma, rep, naq,
        float(sigma), kdt, prec, layout, out.data_ptr(), stream_handle()))
    res = out.double().cpu().numpy()
    return res.reshape(naq, naq) if layout == _lib.KFB_DENSE else res


def kernel_gaussian_hessian_symm(X, dX, Q, N, sigma, *, precision="fp64"):
    """Symmetric Hessian (naq, naq); only the lower triangle is filled, as in the
    reference (src/local_kernels.cpp:1421-1655)."""
    return _hess_symm(X, dX, Q, N, sigma, precision, _lib.KFB_DENSE)


def kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, sigma, *, precision="fp64"):
    """Symmetric Hessian in RFP (TRANSR='N', Fortran UPLO='U').
    Reference: src/local_kernels.cpp:1664-1900."""
    return _hess_symm(X, dX, Q, N, sigma, precision, _lib.KFB_RFP_U)


def kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma, *, precision="fp64"):
    """Energy+force kernel ((nm1+naq1), (nm2+naq2)): [scalar, jacobian; -jacobian_t,
    hessian].  Reference: src/local_kernels.cpp:1918-2188."""
    X1, X2, dX1, dX2 = map(np.asarray, (X1, X2, dX1, dX2))
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    _check_pair_deriv(X1, dX1, X2, dX2, Q1, Q2, N1, N2)
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    naq1, naq2 = _naq(N1, ma1), _naq(N2, ma2)
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    dt, kdt = _deriv_dtype(precision)
    x1, x2 = to_device(_f64(X1), dt), to_device(_f64(X2), dt)
    dx1, dx2 = to_device(_f64(dX1), dt), to_device(_f64(dX2), dt)
    out = torch.empty((nm1 + naq1, nm2 + naq2), dtype=dt, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_full(
        x1.data_ptr(), dx1.data_ptr(), x2.data_ptr(), dx2.data_ptr(), Q1.ctypes.data,
        Q2.ctypes.data, N1.ctypes.data, N2.ctypes.data, nm1, nm2, ma1, ma2, rep, naq1, naq2,
        float(sigma), kdt, prec, out.data_ptr(), stream_handle()))
    return out.double().cpu().numpy()


def _full_symm(X, dX, Q, N, sigma, precision, layout):
    X, dX = np.asarray(X), np.asarray(dX)
    Q, N = host_i32(Q), host_i32(N)
    if X.ndim != 3 or dX.ndim != 4 or Q.ndim != 2 or N.ndim != 1:
        raise ValueError("shape error")
    _check_dX(dX, X, "dX")
    _check_symm_shapes(X, Q, N)
    nm, ma, rep = X.shape
    naq = _naq(N, ma)
    big = nm + naq
    prec = _prec(precision)
    check_sigma(sigma)
    require_cuda()
    import torch
    dt, kdt = _deriv_dtype(precision)
    x, dx = to_device(_f64(X), dt), to_device(_f64(dX), dt)
    count = big * big if layout == _lib.KFB_DENSE else big * (big + 1) // 2
    out = torch.empty((count,), dtype=dt, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_full_symm(
        x.data_ptr(), dx.data_ptr(), Q.ctypes.data, N.ctypes.data, nm, ma, rep, naq,
        float(sigma), kdt, prec, layout, out.data_ptr(), stream_handle()))
    res = out.double().cpu().numpy()
    return res.reshape(big, big) if layout == _lib.KFB_DENSE else res


def kernel_gaussian_full_symm(X, dX, Q, N, sigma, *, precision="fp64"):
    """Symmetric energy+force kernel (nm+naq, nm+naq), fully filled.
    Reference: src/local_kernels.cpp:2201-2498."""
    return _full_symm(X, dX, Q, N, sigma, precision, _lib.KFB_DENSE)


def kernel_gaussian_full_symm_rfp(X, dX, Q, N, sigma, *, precision="fp64"):
    """Symmetric energy+force kernel in RFP (TRANSR='N', Fortran UPLO='U').
    Reference: src/local_kernels.cpp:2511-2815."""
    return _full_symm(X, dX, Q, N, sigma, precision, _lib.KFB_RFP_U)


# --------------------------------------------------------------------------
# contracted energy / force prediction ("J^T alpha")
# --------------------------------------------------------------------------

def kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, alpha):
    """alpha_desc[b, j, :] = dX2[b, j, :, :3 N2[b]] @ alpha[off_b : off_b + 3 N2[b]]
    (zero for padded atoms), shape (nm2, max_atoms2, rep) float64.  Reference:
    src/local_kernels_bindings.cpp:1179-1243, src/local_kernels.cpp:2821-2894."""
    dX2 = np.asarray(dX2)
    alpha = np.asarray(alpha)
    Q2, N2 = host_i32(Q2), host_i32(N2)
    if dX2.ndim != 4 or Q2.ndim != 2 or N2.ndim != 1 or alpha.ndim != 1:
        raise ValueError("shape error")
    nm2, ma2, rep = dX2.shape[0], dX2.shape[1], dX2.shape[2]
    if dX2.shape[3] != 3 * ma2:
        raise ValueError("dX2 shape mismatch")
    if Q2.shape != (nm2, ma2):
        raise ValueError("Q2 shape mismatch")
    if N2.shape[0] != nm2:
        raise ValueError("N2 length mismatch")
    if nm2 <= 0 or ma2 <= 0 or rep <= 0:
        raise ValueError("dimensions must be positive")
    naq2 = _naq(N2, ma2)
    if alpha.shape[0] < naq2:
        raise ValueError("alpha length mismatch")
    require_cuda()
    import torch
    dx2 = to_device(_f64(dX2), torch.float64)
    al = to_device(_f64(alpha), torch.float64)
    out = torch.empty((nm2, ma2, rep), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kfb_local_alpha_desc(
        dx2.data_ptr(), Q2.ctypes.data, N2.ctypes.data, nm2, ma2, rep, _lib.KFB_F64,
        al.data_ptr(), out.data_ptr(), stream_handle()))
    return out.cpu().numpy()


def _check_matvec(X1, dX1, X2, ad, Q1, Q2, N1, N2, ad_name):
    if X1.ndim != 3 or X2.ndim != 3 or ad.ndim != 3 or Q1.ndim != 2 or Q2.ndim != 2 \
            or N1.ndim != 1 or N2.ndim != 1 or (dX1 is not None and dX1.ndim != 4):
        raise ValueError("shape error")
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    if dX1 is not None and dX1.shape != (nm1, ma1, rep, 3 * ma1):
        raise ValueError("dX1 shape mismatch")
    if X2.shape[2] != rep:
        raise ValueError("X2 rep_size mismatch")
    if ad.shape != (nm2, ma2, rep):
        raise ValueError(f"{ad_name} shape mismatch")
    if Q1.shape != (nm1, ma1):
        raise ValueError("Q1 shape mismatch")
    if Q2.shape != (nm2, ma2):
        raise ValueError("Q2 shape mismatch")
    if N1.shape[0] != nm1 or N2.shape[0] != nm2:
        raise ValueError("N1/N2 length mismatch")


def _matvec(X1, dX1, X2, ad, alpha_E, Q1, Q2, N1, N2, sigma, want_e, want_f):
    """Shared body of the three matvecs: (E or None, F or None), float64."""
    nm1, ma1, rep = X1.shape
    nm2, ma2 = X2.shape[0], X2.shape[1]
    naq1 = _naq(N1, ma1)
    E = np.zeros(nm1) if want_e else None
    F = np.zeros(naq1) if want_f else None
    if nm1 == 0 or (want_f and not want_e and naq1 == 0):
        return E, F
    if nm2 <= 0 or ma1 <= 0 or ma2 <= 0 or rep <= 0:
        raise ValueError("dimensions must be positive")
    check_sigma(sigma)
    require_cuda()
    import torch
    x1, x2 = to_device(_f64(X1), torch.float64), to_device(_f64(X2), torch.float64)
    dx1 = to_device(_f64(dX1), torch.float64) if want_f else None
    adt = to_device(_f64(ad), torch.float64)
    ae = to_device(_f64(alpha_E), torch.float64) if alpha_E is not None else None
    e = torch.empty(nm1, dtype=torch.float64, device="cuda") if want_e else None
    f = torch.empty(max(naq1, 1), dtype=torch.float64, device="cuda") if want_f else None
    _lib.check(_lib.lib().kfb_local_matvec(
        x1.data_ptr(), dx1.data_ptr() if dx1 is not None else None, x2.data_ptr(),
        adt.data_ptr(), ae.data_ptr() if ae is not None else None, Q1.ctypes.data,
        Q2.ctypes.data, N1.ctypes.data, N2.ctypes.data, nm1, nm2, ma1, ma2, rep, float(sigma),
        _lib.KFB_F64, e.data_ptr() if e is not None else None,
        f.data_ptr() if f is not None else None, stream_handle()))
    if want_e:
        E = e.cpu().numpy()
    if want_f:
        F = f[:naq1].cpu().numpy()
    return E, F


def kernel_gaussian_local_jacobian_t_matvec(X1, X2, alpha_desc, Q1, Q2, N1, N2, sigma):
    """Energies (nm1,) of force coefficients alpha (alpha_desc =
    kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, alpha)): the energy rows
    of kernel_gaussian_full(query, training) times [0; alpha].  Reference:
    src/local_kernels_bindings.cpp:1358-1427, src/local_kernels.cpp:3155-3262."""
    X1, X2, ad = np.asarray(X1), np.asarray(X2), np.asarray(alpha_desc)
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    _check_matvec(X1, None, X2, ad, Q1, Q2, N1, N2, "alpha_desc")
    return _matvec(X1, None, X2, ad, None, Q1, Q2, N1, N2, sigma, True, False)[0]


def kernel_gaussian_local_hessian_matvec(X1, dX1, X2, alpha_desc, Q1, Q2, N1, N2, sigma):
    """Forces (naq1,) = kernel_gaussian_hessian(X1, dX1, X2, dX2, ...) @ alpha, from
    alpha_desc = kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, alpha).
    Reference: src/local_kernels_bindings.cpp:1246-1356, src/local_kernels.cpp:2895-3154."""
    X1, X2, dX1, ad = map(np.asarray, (X1, X2, dX1, alpha_desc))
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    _check_matvec(X1, dX1, X2, ad, Q1, Q2, N1, N2, "alpha_desc")
    return _matvec(X1, dX1, X2, ad, None, Q1, Q2, N1, N2, sigma, False, True)[1]


def kernel_gaussian_local_full_matvec(X1, dX1, X2, alpha_desc_F, alpha_E, Q1, Q2, N1, N2,
                                      sigma):
    """(E (nm1,), F (naq1,)) = kernel_gaussian_full(query, training) @ [alpha_E; alpha_F]
    with alpha_desc_F = kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, alpha_F).
    Reference: src/local_kernels_bindings.cpp:1429-1530, src/local_kernels.cpp:3263-3425."""
    X1, X2, dX1, ad = map(np.asarray, (X1, X2, dX1, alpha_desc_F))
    alpha_E = np.asarray(alpha_E)
    Q1, Q2, N1, N2 = host_i32(Q1), host_i32(Q2), host_i32(N1), host_i32(N2)
    if alpha_E.ndim != 1:
        raise ValueError("shape error")
    _check_matvec(X1, dX1, X2, ad, Q1, Q2, N1, N2, "alpha_desc_F")
    if alpha_E.shape[0] != X2.shape[0]:
        raise ValueError("alpha_E length mismatch")
    return _matvec(X1, dX1, X2, ad, alpha_E, Q1, Q2, N1, N2, sigma, True, True)
