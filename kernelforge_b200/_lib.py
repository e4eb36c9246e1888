"""ctypes binding of libkfb.so (include/kfb.h).

The library is built in-tree (kernelforge_b200/libkfb.so, see build.py).  There
is no CPU fallback: importing works without a GPU (so the CPU test suite can
check the exports), but every compute call raises if no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkfb.so")

KFB_OK, KFB_ERR_INVALID_ARG, KFB_ERR_NOT_PD, KFB_ERR_ALLOC = 0, 1, 2, 3
KFB_ERR_CUDA, KFB_ERR_TIMEOUT, KFB_ERR_NO_CONVERGENCE, KFB_ERR_UNSUPPORTED = 4, 5, 6, 7
KFB_F32, KFB_F64 = 0, 1
PREC = {"fp64": 0, "fp32": 1, "split_f16": 2}
KFB_DENSE, KFB_RFP_U, KFB_RFP_L = 0, 1, 2
KFB_SOLVE_LAMBDA_FLOOR = 1
KFB_SOLVE_FP64_FACTOR = 2

# every function declared in include/kfb.h
EXPORTS = (
    "kfb_last_error", "kfb_abi_version", "kfb_set_timing", "kfb_last_kernel_ms", "kfb_kernel_gaussian", "kfb_kernel_gaussian_symm",
    "kfb_kernel_gaussian_symm_host",
    "kfb_kernel_gaussian_jacobian", "kfb_kernel_gaussian_jacobian_t",
    "kfb_kernel_gaussian_hessian", "kfb_kernel_gaussian_hessian_symm",
    "kfb_kernel_gaussian_full", "kfb_kernel_gaussian_full_symm", "kfb_full_to_rfp",
    "kfb_rfp_to_full", "kfb_rfp_add_diag", "kfb_rfp_potrf", "kfb_rfp_potrs",
    "kfb_cho_solve_rfp", "kfb_krr_solve_mixed", "kfb_rff_features_elemental",
    "kfb_rff_gradient_elemental", "kfb_feature_gramian", "kfb_ridge_solve_mixed", "kfb_pair_gaussian", "kfb_cosmlp_create", "kfb_cosmlp_destroy",
    "kfb_cosmlp_params", "kfb_cosmlp_grads", "kfb_cosmlp_sync", "kfb_cosmlp_optimizer_state",
    "kfb_cosmlp_set_steps", "kfb_cosmlp_pair_step", "kfb_cosmlp_features_elemental",
    "kfb_local_alpha_desc", "kfb_local_matvec", "kfb_fchl19_rep_size", "kfb_fchl19_repr",
    "kfb_kernel_gaussian_symm_noalloc", "kfb_path_log_clear", "kfb_path_log_read",
    "kfb_gemm_f64_i8",
)


class KfbError(RuntimeError):
    """A libkfb call failed (CUDA error, timeout, allocation, no convergence)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("factor_info", ctypes.c_int),
                ("shift", ctypes.c_double), ("rel_residual", ctypes.c_double),
                ("used_cg", ctypes.c_int), ("lambda_eff", ctypes.c_double)]


_lib = None
P = ctypes.c_void_p
I = ctypes.c_int
D = ctypes.c_double

_SIGS = {
    "kfb_last_error": (ctypes.c_char_p, []),
    "kfb_abi_version": (I, []),
    "kfb_set_timing": (I, [I]),
    "kfb_last_kernel_ms": (D, []),
    "kfb_kernel_gaussian": (I, [P, P, P, P, P, P, I, I, I, I, I, D, I, I, I, P, P]),
    "kfb_kernel_gaussian_symm": (I, [P, P, P, I, I, I, D, I, I, I, I, P, P]),
    "kfb_kernel_gaussian_symm_host": (I, [P, P, P, I, I, I, D, I, I, I, I, P, P]),
    "kfb_kernel_gaussian_jacobian": (I, [P, P, P, P, P, P, P, I, I, I, I, I, I, D, I, I, P, P]),
    "kfb_kernel_gaussian_jacobian_t": (I, [P, P, P, P, P, P, P, I, I, I, I, I, I, D, I, I, P, P]),
    "kfb_kernel_gaussian_hessian": (I, [P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, D, I, I, P,
                                        P]),
    "kfb_kernel_gaussian_hessian_symm": (I, [P, P, P, P, I, I, I, I, D, I, I, I, P, P]),
    "kfb_kernel_gaussian_full": (I, [P, P, P, P, P, P, P, P, I, I, I, I, I, I, I, D, I, I, P, P]),
    "kfb_kernel_gaussian_full_symm": (I, [P, P, P, P, I, I, I, I, D, I, I, I, P, P]),
    "kfb_full_to_rfp": (I, [P, I, I, I, P, P]),
    "kfb_rfp_to_full": (I, [P, I, I, I, P, P]),
    "kfb_rfp_add_diag": (I, [P, I, D, I, I, P]),
    "kfb_rfp_potrf": (I, [P, I, D, I, I, ctypes.POINTER(I), P]),
    "kfb_rfp_potrs": (I, [P, P, I, I, I, I, P]),
    "kfb_cho_solve_rfp": (I, [P, P, I, D, I, P, ctypes.POINTER(I), P]),
    "kfb_krr_solve_mixed": (I, [P, P, I, D, I, D, I, I, P, ctypes.POINTER(SolveInfo), P]),
    "kfb_rff_features_elemental": (I, [P, P, P, I, I, I, P, P, I, I, I, P, P]),
    "kfb_rff_gradient_elemental": (I, [P, P, P, P, I, I, I, P, P, I, I, I, P, P]),
    "kfb_feature_gramian": (I, [P, P, I, I, I, P, P, P]),
    "kfb_ridge_solve_mixed": (I, [P, P, I, I, D, D, I, I, P, ctypes.POINTER(SolveInfo), P]),
    "kfb_pair_gaussian": (I, [P, ctypes.c_longlong, P, P, I, I, D, I, P, P]),
    "kfb_cosmlp_create": (I, [I, I, I, I, I, ctypes.POINTER(P)]),
    "kfb_cosmlp_destroy": (None, [P]),
    "kfb_cosmlp_params": (I, [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P),
                              ctypes.POINTER(P)]),
    "kfb_cosmlp_grads": (I, [P, ctypes.POINTER(P), ctypes.POINTER(P), ctypes.POINTER(P),
                             ctypes.POINTER(P)]),
    "kfb_cosmlp_sync": (I, [P, I, P]),
    "kfb_cosmlp_optimizer_state": (I, [P, P, P, P]),
    "kfb_cosmlp_set_steps": (I, [P, P]),
    "kfb_cosmlp_pair_step": (I, [P, I, P, ctypes.c_longlong, I, P, P, P, I, ctypes.c_float, I,
                                 ctypes.POINTER(D), P]),
    "kfb_cosmlp_features_elemental": (I, [P, P, P, P, I, I, I, I, P, P]),
    "kfb_local_alpha_desc": (I, [P, P, P, I, I, I, I, P, P, P]),
    "kfb_local_matvec": (I, [P, P, P, P, P, P, P, P, P, I, I, I, I, I, D, I, P, P, P]),
    "kfb_fchl19_rep_size": (I, [I, I, I, I]),
    "kfb_fchl19_repr": (I, [P, P, P, I, I, I, I, I, I, D, D, D, D, D, D, D, D, I, P, P, P]),
    "kfb_kernel_gaussian_symm_noalloc": (I, [P, P, P, I, I, I, D, I, I, P, P]),
    "kfb_path_log_clear": (I, []),
    "kfb_path_log_read": (I, [ctypes.c_char_p, I]),
    "kfb_gemm_f64_i8": (I, [I, I, I, D, P, I, P, I, D, P, I, I, P]),
}


def lib():
    """The loaded libkfb (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: build it with `python -m kernelforge_b200.build`")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def path_log_clear() -> None:
    """Empty this thread's code-path log (kfb_path_log_clear)."""
    lib().kfb_path_log_clear()


def path_log() -> list:
    """The names of the paths taken since the last clear, in call order."""
    n = lib().kfb_path_log_read(None, 0)
    buf = ctypes.create_string_buffer(n + 1)
    lib().kfb_path_log_read(buf, n + 1)
    s = buf.value.decode()
    return s.split(",") if s else []


def check(status: int) -> None:
    """Raise the reference's exception type for a failed call."""
    if status == KFB_OK:
        return
    msg = lib().kfb_last_error().decode(errors="replace")
    if status == KFB_ERR_INVALID_ARG:
        raise ValueError(msg)
    raise KfbError(status, msg)
