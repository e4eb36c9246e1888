"""Contracted energy/force prediction on the GPU (kfb_local_alpha_desc,
kfb_local_matvec) against the reference's golden outputs and the oracle.
FP64 inputs: rtol 1e-10 (the reference's own matvec tests use 1e-8 to 1e-12);
float32 inputs (the torch-facing module): FP64 arithmetic on the rounded
inputs, compared with the oracle on the same rounded inputs at rtol 1e-9 and
the float32 outputs at rtol 1e-6."""
import os

import numpy as np
import pytest

from conftest import load_golden, make_set
from oracle import matvec as om

pytestmark = pytest.mark.gpu


def _case(tag):
    g = load_golden("golden_matvec.npz")
    return {k[len(tag) + 1:]: v for k, v in g.items() if k.startswith(tag + "_")}


def close(got, ref, rtol=1e-10):
    ref = np.asarray(ref)
    np.testing.assert_allclose(got, ref, rtol=rtol, atol=rtol * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("tag", ["r", "f"])
def test_golden_alpha_desc(tag):
    from kernelforge_b200 import local_kernels as lk
    c = _case(tag)
    ad = lk.kernel_gaussian_local_compute_alpha_desc(c["dX2"], c["Q2"], c["N2"], c["alpha_F"])
    assert ad.shape == c["alpha_desc"].shape and ad.dtype == np.float64
    close(ad, c["alpha_desc"], 1e-12)


@pytest.mark.parametrize("tag", ["r", "f"])
def test_golden_matvecs(tag):
    from kernelforge_b200 import local_kernels as lk
    c = _case(tag)
    tail = (c["Q1"], c["Q2"], c["N1"], c["N2"], float(c["sigma"]))
    E = lk.kernel_gaussian_local_jacobian_t_matvec(c["X1"], c["X2"], c["alpha_desc"], *tail)
    assert E.shape == c["jacobian_t_matvec"].shape
    close(E, c["jacobian_t_matvec"])
    F = lk.kernel_gaussian_local_hessian_matvec(c["X1"], c["dX1"], c["X2"], c["alpha_desc"],
                                                *tail)
    assert F.shape == c["hessian_matvec"].shape
    close(F, c["hessian_matvec"])
    E, F = lk.kernel_gaussian_local_full_matvec(c["X1"], c["dX1"], c["X2"], c["alpha_desc"],
                                                c["alpha_E"], *tail)
    close(E, c["full_matvec_E"])
    close(F, c["full_matvec_F"])


def _problem(seed, nm1=7, nm2=9, ma1=6, ma2=8, rep=24, species=3, scale=0.35):
    X1, dX1, Q1, N1 = make_set(nm1, ma1, rep, species, seed)
    X2, dX2, Q2, N2 = make_set(nm2, ma2, rep, species, seed + 1)
    rng = np.random.default_rng(seed + 2)
    aE = rng.standard_normal(nm2)
    aF = rng.standard_normal(int(3 * N2.sum()))
    return (X1 * scale, dX1 * 0.3, Q1, N1, X2 * scale, dX2 * 0.3, Q2, N2, aE, aF)


@pytest.mark.parametrize("sigma", [0.2, 0.5, 1.0, 2.0, 5.0])
def test_sigmas_against_oracle(sigma):
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(11)
    ad = om.alpha_desc(dX2, Q2, N2, aF)
    close(lk.kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, aF), ad, 1e-12)
    Er, Fr = om.matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1, N2, sigma)
    E, F = lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1, N2, sigma)
    close(E, Er)
    close(F, Fr)


def test_equals_full_kernel_times_coefficients():
    """E, F equal the GPU's own kernel_gaussian_full(query, training) @ [aE; aF]."""
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(21, nm1=12, nm2=15, rep=40)
    sigma = 1.3
    K = lk.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma)
    v = np.concatenate([aE, aF])
    ad = lk.kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, aF)
    E, F = lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1, N2, sigma)
    close(E, K[:len(N1)] @ v)
    close(F, K[len(N1):] @ v)


def test_chunked_query_rows(monkeypatch):
    """A workspace budget far below one label's rows forces many query chunks."""
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(31, nm1=40, nm2=30, rep=32)
    ad = om.alpha_desc(dX2, Q2, N2, aF)
    Er, Fr = om.matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1, N2, 1.1)
    monkeypatch.setenv("KFB_WORKSPACE_GB", "0.00002")  # ~21 kB: a handful of rows
    E, F = lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1, N2, 1.1)
    close(E, Er)
    close(F, Fr)


def test_edge_cases():
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(41)
    ad = om.alpha_desc(dX2, Q2, N2, aF)
    # query labels absent from the training set: all zero
    Q1x = np.where(Q1 > 0, Q1 + 50, 0).astype(np.int32)
    E, F = lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE, Q1x, Q2, N1, N2, 1.0)
    assert not E.any() and not F.any() and F.shape == (3 * N1.sum(),)
    # empty query molecules and a single query molecule
    N1e = N1.copy()
    N1e[[0, 3]] = 0
    Er, Fr = om.matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1e, N2, 0.9)
    E, F = lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1e, N2, 0.9)
    close(E, Er)
    close(F, Fr)
    assert E[0] == 0.0 and E[3] == 0.0
    E1, F1 = lk.kernel_gaussian_local_full_matvec(X1[:1], dX1[:1], X2, ad, aE, Q1[:1], Q2,
                                                  N1[:1], N2, 0.9)
    Er1, Fr1 = om.matvec(X1[:1], dX1[:1], X2, ad, aE, Q1[:1], Q2, N1[:1], N2, 0.9)
    close(E1, Er1)
    close(F1, Fr1)
    # all query molecules empty
    Z = np.zeros_like(N1)
    F = lk.kernel_gaussian_local_hessian_matvec(X1, dX1, X2, ad, Q1, Q2, Z, N2, 1.0)
    assert F.shape == (0,)
    E = lk.kernel_gaussian_local_jacobian_t_matvec(X1, X2, ad, Q1, Q2, Z, N2, 1.0)
    assert E.shape == (len(N1),) and not E.any()


def test_bad_arguments():
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(51)
    ad = om.alpha_desc(dX2, Q2, N2, aF)
    with pytest.raises(ValueError):
        lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad[:-1], aE, Q1, Q2, N1, N2, 1.0)
    with pytest.raises(ValueError):
        lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE[:-1], Q1, Q2, N1, N2, 1.0)
    with pytest.raises(ValueError):
        lk.kernel_gaussian_local_hessian_matvec(X1, dX1[:, :, :-1], X2, ad, Q1, Q2, N1, N2, 1.0)
    with pytest.raises(ValueError):
        lk.kernel_gaussian_local_jacobian_t_matvec(X1, X2, ad, Q1, Q2, N1, N2, 0.0)
    with pytest.raises(ValueError):
        lk.kernel_gaussian_local_compute_alpha_desc(dX2[..., :-1], Q2, N2, aF)


def test_torch_module_float32():
    import torch
    from kernelforge_b200 import cuda_local_kernels as clk
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(61, nm1=10, nm2=12, rep=48)
    f32 = lambda a: torch.tensor(np.asarray(a, np.float32), device="cuda")
    i32 = lambda a: torch.tensor(np.asarray(a, np.int32), device="cuda")
    r = lambda a: np.asarray(a, np.float32).astype(np.float64)
    ad = clk.compute_alpha_desc(f32(dX2), i32(N2), f32(aF))
    assert ad.dtype == torch.float32 and tuple(ad.shape) == X2.shape
    ad_ref = om.alpha_desc(r(dX2), Q2, N2, r(aF))
    close(ad.double().cpu().numpy(), ad_ref, 1e-6)
    sigma = 1.2
    E, F = clk.kernel_gaussian_full_matvec(f32(X1), f32(dX1), i32(Q1), i32(N1), f32(X2),
                                           i32(Q2), i32(N2), f32(aE), ad, sigma)
    assert E.dtype == torch.float32 and F.dtype == torch.float32
    Er, Fr = om.matvec(r(X1), r(dX1), r(X2), r(ad.cpu().numpy()), r(aE), Q1, Q2, N1, N2, sigma)
    close(E.double().cpu().numpy(), Er, 1e-6)
    close(F.double().cpu().numpy(), Fr, 1e-6)


def test_fp32_inputs_fp64_arithmetic():
    """x_dt = KFB_F32 through the C-ABI: FP64 arithmetic on the float32 values."""
    import ctypes
    import torch
    from kernelforge_b200 import _lib
    X1, dX1, Q1, N1, X2, dX2, Q2, N2, aE, aF = _problem(71)
    r = lambda a: np.asarray(a, np.float32).astype(np.float64)
    ad = om.alpha_desc(r(dX2), Q2, N2, aF)
    Er, Fr = om.matvec(r(X1), r(dX1), r(X2), ad, aE, Q1, Q2, N1, N2, 0.8)
    d = lambda a, dt: torch.tensor(np.asarray(a), dtype=dt, device="cuda")
    x1, dx1, x2 = d(X1, torch.float32), d(dX1, torch.float32), d(X2, torch.float32)
    adt, aet = d(ad, torch.float64), d(aE, torch.float64)
    e = torch.empty(len(N1), dtype=torch.float64, device="cuda")
    f = torch.empty(int(3 * N1.sum()), dtype=torch.float64, device="cuda")
    Q1c, Q2c, N1c, N2c = (np.ascontiguousarray(a, np.int32) for a in (Q1, Q2, N1, N2))
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    _lib.check(_lib.lib().kfb_local_matvec(
        x1.data_ptr(), dx1.data_ptr(), x2.data_ptr(), adt.data_ptr(), aet.data_ptr(),
        Q1c.ctypes.data, Q2c.ctypes.data, N1c.ctypes.data, N2c.ctypes.data, nm1, nm2, ma1, ma2,
        rep, ctypes.c_double(0.8), _lib.KFB_F32, e.data_ptr(), f.data_ptr(),
        torch.cuda.current_stream().cuda_stream))
    close(e.cpu().numpy(), Er, 1e-9)
    close(f.cpu().numpy(), Fr, 1e-9)
