"""Device staging helpers for the NumPy- and torch-facing modules.

PyTorch is used only for device memory and the current CUDA stream; all compute
goes through libkfb.  There is no CPU fallback: without a CUDA device the
compute calls raise.
"""
from __future__ import annotations

import math

import numpy as np


def require_cuda() -> None:
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("kernelforge_b200 computes on a CUDA (sm_100) device; none is available")


def stream_handle() -> int:
    import torch
    return torch.cuda.current_stream().cuda_stream


def to_device(a: np.ndarray, dtype):
    """Host array -> contiguous CUDA tensor of `dtype` (pinned staging for large arrays)."""
    import torch
    t = torch.from_numpy(np.ascontiguousarray(a))
    if t.numel() * t.element_size() > (1 << 20):
        t = t.pin_memory()
    return t.to(device="cuda", dtype=dtype, non_blocking=False)


def host_i32(a) -> np.ndarray:
    """Labels / atom counts as a C-contiguous host int32 array (torch tensors are
    copied to the host)."""
    try:
        import torch
        if isinstance(a, torch.Tensor):
            a = a.detach().cpu().numpy()
    except ImportError:
        pass
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)


def check_sigma(sigma) -> None:
    s = float(sigma)
    if not math.isfinite(s) or s <= 0.0:
        raise ValueError("sigma must be > 0")
