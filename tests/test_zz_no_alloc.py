"""The allocation-free entry point kfb_kernel_gaussian_symm_noalloc, called
through the C ABI, gives the same kernel as kfb_kernel_gaussian_symm (FP64,
rtol 1e-12), on two calls in a row (the second call reuses the fixed scratch
array the first call left behind).  It exists for callers that cannot allocate
device memory during a call: frameworks that reserve the device-memory budget
up front, or loops that must not let cudaMalloc / cudaFree synchronise the
device.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import make_set
from oracle import oracle as o

pytestmark = pytest.mark.gpu


def _regular(lib, x, Q, N, sigma, layout, count):
    import torch

    from kernelforge_b200 import _lib
    nm, ma, rep = x.shape
    out = torch.full((count,), float("nan"), dtype=torch.float64, device="cuda")
    st = lib.kfb_kernel_gaussian_symm(x.data_ptr(), Q.ctypes.data, N.ctypes.data, nm, ma, rep,
                                      sigma, _lib.KFB_F64, _lib.PREC["fp64"], layout, _lib.KFB_F64,
                                      out.data_ptr(), torch.cuda.current_stream().cuda_stream)
    assert st == _lib.KFB_OK, lib.kfb_last_error()
    return out


def _noalloc(lib, x, Q, N, sigma, layout, count):
    import torch

    from kernelforge_b200 import _lib
    nm, ma, rep = x.shape
    out = torch.full((count,), float("nan"), dtype=torch.float64, device="cuda")
    st = lib.kfb_kernel_gaussian_symm_noalloc(x.data_ptr(), Q.ctypes.data, N.ctypes.data, nm, ma,
                                              rep, sigma, _lib.KFB_F64, layout, out.data_ptr(),
                                              torch.cuda.current_stream().cuda_stream)
    assert st == _lib.KFB_OK, lib.kfb_last_error()
    return out


@pytest.mark.parametrize("layout_name", ["dense", "rfp_u", "rfp_l"])
def test_noalloc_matches_the_allocating_entry_point_twice(layout_name):
    import torch

    from kernelforge_b200 import _lib
    lib = _lib.lib()
    layout = {"dense": _lib.KFB_DENSE, "rfp_u": _lib.KFB_RFP_U, "rfp_l": _lib.KFB_RFP_L}[layout_name]
    X, _, Q, N = make_set(140, 10, 48, 3, seed=17)
    X *= 0.4
    N[3] = 0
    nm = X.shape[0]
    count = nm * nm if layout == _lib.KFB_DENSE else nm * (nm + 1) // 2
    x = torch.tensor(X, device="cuda")
    ref = _regular(lib, x, Q, N, 2.0, layout, count).cpu().numpy()
    # the CPU oracle of the same layout pins both entry points
    if layout == _lib.KFB_DENSE:
        want = o.kernel_gaussian_symm(X, Q, N, 2.0).ravel()
    else:
        want = o.kernel_gaussian_symm_rfp(X, Q, N, 2.0,
                                          uplo_lower=(layout == _lib.KFB_RFP_L))
    np.testing.assert_allclose(ref, want, rtol=1e-12, atol=1e-12)
    for _ in range(2):
        got = _noalloc(lib, x, Q, N, 2.0, layout, count).cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
    # a different problem in between: the scratch keeps the last call's contents
    X2, _, Q2, N2 = make_set(60, 7, 48, 2, seed=18)
    x2 = torch.tensor(X2 * 0.4, device="cuda")
    c2 = 60 * 60 if layout == _lib.KFB_DENSE else 60 * 61 // 2
    np.testing.assert_allclose(_noalloc(lib, x2, Q2, N2, 2.0, layout, c2).cpu().numpy(),
                               _regular(lib, x2, Q2, N2, 2.0, layout, c2).cpu().numpy(),
                               rtol=1e-12, atol=1e-12)
    got = _noalloc(lib, x, Q, N, 2.0, layout, count).cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_noalloc_rejects_a_problem_larger_than_its_scratch():
    import torch

    from kernelforge_b200 import _lib
    lib = _lib.lib()
    nm, ma, rep = 1600, 10, 720          # 16,000 active atoms: beyond the fixed scratch
    X = np.zeros((nm, ma, rep), dtype=np.float64)
    Q = np.ones((nm, ma), dtype=np.int32)
    N = np.full((nm,), ma, dtype=np.int32)
    x = torch.tensor(X, device="cuda")
    out = torch.full((nm * (nm + 1) // 2,), 7.0, dtype=torch.float64, device="cuda")
    st = lib.kfb_kernel_gaussian_symm_noalloc(x.data_ptr(), Q.ctypes.data, N.ctypes.data, nm, ma,
                                              rep, 2.0, _lib.KFB_F64, _lib.KFB_RFP_U,
                                              out.data_ptr(),
                                              torch.cuda.current_stream().cuda_stream)
    assert st == _lib.KFB_ERR_INVALID_ARG
    assert b"scratch" in lib.kfb_last_error()
    torch.cuda.synchronize()
    assert bool((out == 7.0).all())   # rejected before any device work
    assert ctypes.sizeof(ctypes.c_void_p) == 8
