"""Drop-in for the reference's ``kernelforge.cuda_fchl19_repr`` module (GPU FCHL19
descriptors of padded molecule batches; stub python/kernelforge/cuda_fchl19_repr.pyi):
float32 CUDA tensors in and out, element indices Q in [0, nelements).  Arithmetic is
FP64 inside the kernel (``kfb_fchl19_repr``), results are stored in float32.
``deterministic`` is accepted for signature compatibility: the kernel writes every
Jacobian entry from one thread, so results do not depend on scheduling.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from ._device import host_i32, require_cuda, stream_handle

__all__ = ["generate_fchl_acsf", "generate_fchl_acsf_and_gradients",
           "generate_fchl_acsf_and_gradients_md_single"]


def _check(coords, Q, N, nelements):
    import torch
    if not isinstance(coords, torch.Tensor) or not coords.is_cuda:
        raise RuntimeError("coords must be a CUDA tensor")
    if coords.dtype != torch.float32:
        raise RuntimeError("coords must be float32")
    if coords.dim() != 3 or coords.shape[2] != 3:
        raise RuntimeError("coords must have shape (nm, max_atoms, 3)")
    nm, ma = coords.shape[0], coords.shape[1]
    Qh, Nh = host_i32(Q), host_i32(N)
    if Qh.shape != (nm, ma) or Nh.shape != (nm,):
        raise RuntimeError("Q must be (nm, max_atoms) and N (nm,)")
    if int(nelements) <= 0:
        raise RuntimeError("nelements must be > 0")
    return coords.contiguous(), Qh, Nh, nm, ma


def _run(coords, Q, N, nelements, grad, nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut, acut,
         two_body_decay, three_body_decay, three_body_weight):
    require_cuda()
    import torch
    c, Qh, Nh, nm, ma = _check(coords, Q, N, nelements)
    rep_size = _lib.lib().kfb_fchl19_rep_size(int(nelements), int(nRs2), int(nRs3),
                                              int(nFourier))
    if rep_size <= 0:
        raise RuntimeError("invalid descriptor sizes")
    rep = torch.empty((nm, ma, rep_size), dtype=torch.float32, device=c.device)
    g = torch.empty((nm, ma, rep_size, ma, 3), dtype=torch.float32, device=c.device) \
        if grad else None
    st = _lib.lib().kfb_fchl19_repr(
        c.data_ptr(), Qh.ctypes.data, Nh.ctypes.data, nm, ma, int(nelements), int(nRs2),
        int(nRs3), int(nFourier), float(eta2), float(eta3), float(zeta), float(rcut),
        float(acut), float(two_body_decay), float(three_body_decay), float(three_body_weight),
        _lib.KFB_F32, rep.data_ptr(), g.data_ptr() if g is not None else None,
        stream_handle())
    if st != _lib.KFB_OK:
        raise RuntimeError(_lib.lib().kfb_last_error().decode())
    return (rep, g) if grad else rep


def generate_fchl_acsf(coords, Q, N, nelements, nRs2=24, nRs3=20, nFourier=1, eta2=0.32,
                       eta3=2.7, zeta=math.pi, rcut=8.0, acut=8.0, two_body_decay=1.8,
                       three_body_decay=0.57, three_body_weight=13.4, deterministic=False):
    """rep (nm, max_atoms, rep_size) float32; padded slots are zero.  Reference:
    src/cuda_fchl19_repr_bindings.cpp:170-231."""
    return _run(coords, Q, N, nelements, False, nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut,
                acut, two_body_decay, three_body_decay, three_body_weight)


def generate_fchl_acsf_and_gradients(coords, Q, N, nelements, nRs2=24, nRs3=20, nFourier=1,
                                     eta2=0.32, eta3=2.7, zeta=math.pi, rcut=8.0, acut=8.0,
                                     two_body_decay=1.8, three_body_decay=0.57,
                                     three_body_weight=13.4, deterministic=False):
    """(rep (nm, ma, rep_size), grad (nm, ma, rep_size, ma, 3)) float32.  Reference:
    src/cuda_fchl19_repr_bindings.cpp:233-261."""
    return _run(coords, Q, N, nelements, True, nRs2, nRs3, nFourier, eta2, eta3, zeta, rcut,
                acut, two_body_decay, three_body_decay, three_body_weight)


def generate_fchl_acsf_and_gradients_md_single(coords, Q, N, nelements, nRs2=24, nRs3=20,
                                               nFourier=1, eta2=0.32, eta3=2.7, zeta=math.pi,
                                               rcut=8.0, acut=8.0, two_body_decay=1.8,
                                               three_body_decay=0.57, three_body_weight=13.4,
                                               deterministic=False):
    """The nm == 1 form of generate_fchl_acsf_and_gradients (same kernel).  Reference:
    src/cuda_fchl19_repr_bindings.cpp:263-290."""
    if coords.dim() != 3 or coords.shape[0] != 1:
        raise RuntimeError("the single-molecule path needs nm == 1")
    return generate_fchl_acsf_and_gradients(coords, Q, N, nelements, nRs2, nRs3, nFourier,
                                            eta2, eta3, zeta, rcut, acut, two_body_decay,
                                            three_body_decay, three_body_weight)
