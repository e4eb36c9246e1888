"""Drop-in for the elemental half of ``kernelforge.cuda_rff_features``
(src/cuda_rff_features_bindings.cpp:70-190): random Fourier features summed
per molecule, their force features (gradients through the descriptor
Jacobians), and the energy-only and energy + force normal equations, on the
tensor cores.

Conventions follow the reference's GPU binding: X (nmol, max_atoms, rep)
float32 CUDA tensor, Q (nmol, max_atoms) int32 element INDICES (0-based, -1 =
padding), N (nmol,) int32, W (nelem, rep, D) and b (nelem, D) float32 CUDA
tensors (``W ~ N(0, 1) / sigma``, ``b ~ U(0, 2 pi)``, models/rff.py:110-112).
Q and N may live on the host or the device (they are read on the host).
"""
from __future__ import annotations

from . import _lib
from ._device import host_i32, require_cuda, stream_handle

__all__ = ["rff_features_elemental", "rff_gramian_elemental_rfp",
           "rff_predict_energy_elemental", "feature_gramian", "rff_gradient_elemental",
           "rff_features_elemental_col_major", "rff_gradient_elemental_col_major",
           "rff_full_gramian_elemental_rfp", "rff_predict_force_elemental",
           "rff_predict_force_elemental_cached_topology"]


def _check_x(X):
    import torch
    if not X.is_cuda or X.dim() != 3:
        raise RuntimeError("X must be a 3D CUDA tensor (nmol, max_atoms, rep)")
    if X.dtype not in (torch.float32, torch.float64):
        raise RuntimeError("X must be float32 (or float64)")
    return X.contiguous(), (_lib.KFB_F64 if X.dtype == torch.float64 else _lib.KFB_F32)


def _check_wb(W, b, rep):
    import torch
    if W.dim() != 3 or b.dim() != 2:
        raise RuntimeError("W must be 3D (nelements, rep_size, D) and b 2D (nelements, D)")
    if W.shape[1] != rep:
        raise RuntimeError("W.shape[1] must equal X.shape[2] (rep_size)")
    if W.shape[2] != b.shape[1] or W.shape[0] != b.shape[0]:
        raise RuntimeError("W and b shapes disagree")
    W = W.to(device="cuda", dtype=torch.float32).contiguous()
    b = b.to(device="cuda", dtype=torch.float32).contiguous()
    return W, b


def rff_features_elemental(X, Q, N, W, b):
    """LZ[m] = sum over atoms of molecule m: sqrt(2/D) cos(x W[e] + b[e]);
    returns (nmol, D) float32, row-major."""
    require_cuda()
    import torch
    X, xdt = _check_x(X)
    nm, ma, rep = X.shape
    W, b = _check_wb(W, b, rep)
    q = host_i32(Q).reshape(nm, ma)
    n = host_i32(N).reshape(nm)
    D = b.shape[1]
    Z = torch.empty((nm, D), dtype=torch.float32, device=X.device)
    _lib.check(_lib.lib().kfb_rff_features_elemental(
        X.data_ptr(), q.ctypes.data, n.ctypes.data, nm, ma, rep, W.data_ptr(), b.data_ptr(),
        W.shape[0], D, xdt, Z.data_ptr(), stream_handle()))
    return Z


def feature_gramian(Z, Y=None, layout="L"):
    """Z^T Z of a (nmol, D) float32 feature matrix, RFP 'L' / 'U' (TRANSR='N')
    or dense ('full'), and Z^T Y in float64 (None without Y)."""
    require_cuda()
    import torch
    if Z.dtype != torch.float32 or not Z.is_cuda or Z.dim() != 2:
        raise RuntimeError("Z must be a 2D float32 CUDA tensor")
    Z = Z.contiguous()
    nm, D = Z.shape
    lay = {"L": _lib.KFB_RFP_L, "U": _lib.KFB_RFP_U, "FULL": _lib.KFB_DENSE}[str(layout).upper()]
    ztz = torch.empty((D * (D + 1) // 2,) if lay != _lib.KFB_DENSE else (D, D),
                      dtype=torch.float32, device=Z.device)
    zty = None
    yp = 0
    if Y is not None:
        yd = Y.to(device=Z.device, dtype=torch.float64).contiguous()
        if yd.numel() != nm:
            raise RuntimeError("Y must be 1D (nmol,)")
        zty = torch.empty((D,), dtype=torch.float64, device=Z.device)
        yp = yd.data_ptr()
    _lib.check(_lib.lib().kfb_feature_gramian(Z.data_ptr(), yp, nm, D, lay, ztz.data_ptr(),
                                              zty.data_ptr() if zty is not None else 0,
                                              stream_handle()))
    return ztz, zty


def rff_gramian_elemental_rfp(X, Q, N, W, b, Y, chunk_size=256):
    """(ZtZ_rfp, ZtY) of the energy-only RFF normal equations: ZtZ_rfp float32,
    RFP TRANSR='N', UPLO='L' (the reference's GPU convention), ZtY float64.
    chunk_size is accepted for signature compatibility; the feature matrix is
    formed once."""
    if int(chunk_size) <= 0:
        raise RuntimeError("chunk_size must be positive")
    Z = rff_features_elemental(X, Q, N, W, b)
    return feature_gramian(Z, Y, "L")


def rff_predict_energy_elemental(X, Q, N, W, b, weights, chunk_size=256):
    """Energies Z @ weights (float64)."""
    import torch
    if int(chunk_size) <= 0:
        raise RuntimeError("chunk_size must be positive")
    Z = rff_features_elemental(X, Q, N, W, b)
    return Z.to(torch.float64) @ weights.to(device=Z.device, dtype=torch.float64)


def _check_dx(dX, X):
    import torch
    nm, ma, rep = X.shape
    if not dX.is_cuda or dX.dtype != X.dtype:
        raise RuntimeError("dX must be a CUDA tensor of X's dtype")
    if tuple(dX.shape) not in ((nm, ma, rep, 3 * ma), (nm, ma, rep, ma, 3)):
        raise RuntimeError("dX must be (nmol, max_atoms, rep, 3*max_atoms) or "
                           "(nmol, max_atoms, rep, max_atoms, 3)")
    return dX.contiguous()


def rff_gradient_elemental(X, dX, Q, N, W, b, chunk_size=64):
    """Force features G (total_naq, D) float32: row 3 off_m + 3 a + t holds
    sqrt(2/D) sum_j sin(x_j W[e_j] + b[e_j]) (W[e_j]^T dX[m, j, :, 3 a + t]), so that
    forces are G @ weights (the transpose of the reference CPU's (D, ngrads))."""
    require_cuda()
    import torch
    if int(chunk_size) <= 0:
        raise RuntimeError("chunk_size must be positive")
    X, xdt = _check_x(X)
    dX = _check_dx(dX, X)
    nm, ma, rep = X.shape
    W, b = _check_wb(W, b, rep)
    q = host_i32(Q).reshape(nm, ma)
    n = host_i32(N).reshape(nm)
    D = b.shape[1]
    naq = int(3 * n.clip(0, ma).sum())
    G = torch.empty((max(naq, 1), D), dtype=torch.float32, device=X.device)
    _lib.check(_lib.lib().kfb_rff_gradient_elemental(
        X.data_ptr(), dX.data_ptr(), q.ctypes.data, n.ctypes.data, nm, ma, rep, W.data_ptr(),
        b.data_ptr(), W.shape[0], D, xdt, G.data_ptr(), stream_handle()))
    return G[:naq]


def rff_features_elemental_col_major(X, Q, N, W, b):
    """Z^T (D, nmol) float32."""
    return rff_features_elemental(X, Q, N, W, b).t().contiguous()


def rff_gradient_elemental_col_major(X, dX, Q, N, W, b, chunk_size=64):
    """G^T (D, total_naq) float32."""
    return rff_gradient_elemental(X, dX, Q, N, W, b, chunk_size).t().contiguous()


def rff_full_gramian_elemental_rfp(X, dX, Q, N, W, b, Y, F, energy_chunk=256, force_chunk=64):
    """(ZtZ_rfp, ZtY) of the energy + force normal equations [Z; G]^T [Z; G] and
    Z^T Y + G^T F: float32 RFP TRANSR='N', UPLO='L', and float64.  The chunk sizes
    are accepted for signature compatibility."""
    import torch
    if int(energy_chunk) <= 0 or int(force_chunk) <= 0:
        raise RuntimeError("chunk sizes must be positive")
    Z = rff_features_elemental(X, Q, N, W, b)
    G = rff_gradient_elemental(X, dX, Q, N, W, b)
    y = torch.cat([Y.reshape(-1).to(device=Z.device, dtype=torch.float64),
                   F.reshape(-1).to(device=Z.device, dtype=torch.float64)])
    if y.numel() != Z.shape[0] + G.shape[0]:
        raise RuntimeError("Y must have nmol entries and F 3 * sum(N)")
    return feature_gramian(torch.cat([Z, G]), y, "L")


def rff_predict_force_elemental(X, dX, Q, N, W, b, weights, chunk_size=64):
    """Forces G @ weights (total_naq,) float64."""
    import torch
    G = rff_gradient_elemental(X, dX, Q, N, W, b, chunk_size)
    return G.to(torch.float64) @ weights.to(device=G.device, dtype=torch.float64)


def rff_predict_force_elemental_cached_topology(X, dX, Q, N, W, b, weights, offsets, atom_maps,
                                                row_meta, total_rows_host, total_grads,
                                                chunk_size=64):
    """rff_predict_force_elemental; the reference's cached topology arguments are
    accepted for signature compatibility (the row plan is rebuilt per call)."""
    return rff_predict_force_elemental(X, dX, Q, N, W, b, weights, chunk_size)
