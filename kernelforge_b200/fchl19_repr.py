"""Drop-in for the reference's ``kernelforge.fchl19_repr`` module (FCHL19
descriptors of one molecule and their Jacobians), computed on the GPU.

Same names, arguments, defaults, shapes and exceptions as the pybind11 module
(src/fchl19_repr_bindings.cpp:222-330): NumPy in, float64 NumPy out, FP64
arithmetic (kernel ``kfb_fchl19_repr``, csrc/repr.cu).  ``generate_batched``
adds the padded many-molecule form the local kernels consume.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from ._device import require_cuda, stream_handle, to_device

__all__ = ["compute_rep_size", "generate_fchl_acsf", "generate_fchl_acsf_and_gradients",
           "generate_batched"]

DEFAULT_ELEMENTS = (1, 6, 7, 8, 16)


def compute_rep_size(nelements, nbasis2, nbasis3, nabasis):
    """Descriptor length nelements nbasis2 + nelements (nelements + 1) / 2 nbasis3 nabasis
    (src/fchl19_repr_bindings.cpp:222-230)."""
    nelements, nbasis2, nbasis3, nabasis = (int(v) for v in (nelements, nbasis2, nbasis3,
                                                               nabasis))
    return nelements * nbasis2 + nelements * (nelements + 1) // 2 * nbasis3 * nabasis


def _params(nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut, acut, two_body_decay,
            three_body_decay, three_body_weight):
    return (int(nRs2), int(nRs3), int(nFourier), float(eta2), float(eta3), float(zeta),
            float(rcut), float(acut), float(two_body_decay), float(three_body_decay),
            float(three_body_weight))


def _run(coords_dev, elem, natoms, nm, ma, nelements, params, dt, want_grad):
    """Device outputs (rep, grad or None) of padded molecules."""
    import torch
    nRs2, nRs3, nFourier = params[:3]
    rep_size = _lib.lib().kfb_fchl19_rep_size(nelements, nRs2, nRs3, nFourier)
    if rep_size <= 0:
        raise ValueError("invalid descriptor sizes")
    tdt = torch.float64 if dt == _lib.KFB_F64 else torch.float32
    rep = torch.empty((nm, ma, rep_size), dtype=tdt, device="cuda")
    grad = torch.empty((nm, ma, rep_size, 3 * ma), dtype=tdt, device="cuda") if want_grad \
        else None
    _lib.check(_lib.lib().kfb_fchl19_repr(
        coords_dev.data_ptr(), elem.ctypes.data, natoms.ctypes.data, nm, ma, nelements,
        *params, dt, rep.data_ptr(), grad.data_ptr() if grad is not None else None,
        stream_handle()))
    return rep, grad


def _one(coords, nuclear_z, elements, params, want_grad):
    z = np.ascontiguousarray(np.asarray(nuclear_z).reshape(-1), dtype=np.int64)
    n = z.shape[0]
    if n == 0:
        raise ValueError("n_atoms must be > 0")
    c = np.asarray(coords, dtype=np.float64)
    if c.ndim == 2:
        if c.shape != (n, 3):
            raise ValueError("coords must have shape (n_atoms, 3)")
    elif c.ndim == 1:
        if c.shape[0] != 3 * n:
            raise ValueError("coords 1D length must be n_atoms*3")
        c = c.reshape(n, 3)
    else:
        raise ValueError("coords must be a 1D or 2D NumPy array")
    elements = [int(e) for e in (elements if elements is not None and len(elements) > 0
                                 else DEFAULT_ELEMENTS)]
    lut = {e: k for k, e in enumerate(elements)}
    try:
        idx = np.array([lut[int(v)] for v in z], dtype=np.int32)
    except KeyError:
        raise RuntimeError("nuclear_z contains an element not present in elements") from None
    require_cuda()
    import torch
    cd = to_device(c.reshape(1, n, 3), torch.float64)
    rep, grad = _run(cd, idx.reshape(1, n), np.array([n], np.int32), 1, n, len(elements),
                     params, _lib.KFB_F64, want_grad)
    rep = rep[0].cpu().numpy()
    if not want_grad:
        return rep
    # (n, rep, 3n): the reference's returned layout (column 3 a + t = atom a, axis t)
    return rep, grad[0].cpu().numpy()


def generate_fchl_acsf(coords, nuclear_z, elements=DEFAULT_ELEMENTS, nRs2=24, nRs3=20,
                       nFourier=1, eta2=0.32, eta3=2.7, zeta=math.pi, rcut=8.0, acut=8.0,
                       two_body_decay=1.8, three_body_decay=0.57, three_body_weight=13.4):
    """FCHL19 descriptor (n_atoms, rep_size) float64 of one molecule.  Reference:
    src/fchl19_repr_bindings.cpp:52-138, src/fchl19_repr.cpp:89-306."""
    return _one(coords, nuclear_z, elements,
                _params(nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut, acut, two_body_decay,
                        three_body_decay, three_body_weight), False)


def generate_fchl_acsf_and_gradients(coords, nuclear_z, elements=DEFAULT_ELEMENTS, nRs2=24,
                                     nRs3=20, nFourier=1, eta2=0.32, eta3=2.7, zeta=math.pi,
                                     rcut=8.0, acut=8.0, two_body_decay=1.8,
                                     three_body_decay=0.57, three_body_weight=13.4):
    """(rep (n_atoms, rep_size), grad (n_atoms, rep_size, 3 n_atoms)) float64, analytic
    Jacobian (column 3 a + t: coordinate t of atom a).  Reference: src/fchl19_repr_bindings.cpp:150-216, src/fchl19_repr.cpp:308-781."""
    if int(nFourier) != 1:
        raise ValueError("gradients are defined for nFourier = 1")
    return _one(coords, nuclear_z, elements,
                _params(nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut, acut, two_body_decay,
                        three_body_decay, three_body_weight), True)


def generate_batched(coords, Z, N, elements=DEFAULT_ELEMENTS, gradients=False,
                     dtype="float32", nRs2=24, nRs3=20, nFourier=1, eta2=0.32, eta3=2.7,
                     zeta=math.pi, rcut=8.0, acut=8.0, two_body_decay=1.8,
                     three_body_decay=0.57, three_body_weight=13.4):
    """Padded descriptors of many molecules in the local kernels' layout: coords
    (nm, max_atoms, 3) (NumPy or torch), nuclear charges Z (nm, max_atoms), N (nm,).
    Returns CUDA tensors X (nm, ma, rep) [and dX (nm, ma, rep, 3 ma)] of ``dtype``."""
    import torch
    require_cuda()
    from ._device import host_i32
    Zh, Nh = host_i32(Z), host_i32(N)
    nm, ma = Zh.shape
    elements = [int(e) for e in elements]
    lut = np.full(max(max(elements), int(Zh.max(initial=0))) + 1, -1, np.int32)
    for k, e in enumerate(elements):
        lut[e] = k
    valid = np.arange(ma)[None, :] < np.clip(Nh, 0, ma)[:, None]
    idx = np.where(valid, lut[np.clip(Zh, 0, None)], 0).astype(np.int32)
    if (valid & ((idx < 0) | (Zh < 0))).any():
        raise RuntimeError("nuclear_z contains an element not present in elements")
    tdt = torch.float64 if dtype in ("float64", np.float64, torch.float64) else torch.float32
    kdt = _lib.KFB_F64 if tdt == torch.float64 else _lib.KFB_F32
    if isinstance(coords, torch.Tensor):
        cd = coords.to(device="cuda", dtype=tdt).contiguous()
    else:
        cd = to_device(np.asarray(coords, np.float64), tdt)
    if tuple(cd.shape) != (nm, ma, 3):
        raise ValueError("coords must have shape (nm, max_atoms, 3)")
    rep, grad = _run(cd, idx, Nh, nm, ma, len(elements),
                     _params(nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut, acut,
                             two_body_decay, three_body_decay, three_body_weight), kdt,
                     gradients)
    return (rep, grad) if gradients else rep
