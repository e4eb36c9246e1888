"""Scalar kernels on the GPU against the CPU oracle and the reference's golden
outputs.  FP64 path: reference tolerances (rtol 1e-12).  Split-fp16 tensor-core
and FP32 paths: rtol 2e-5 on entries, atol 2e-6 x max|K| (FP32 arithmetic)."""
import numpy as np
import pytest

from conftest import load_golden, make_set
from oracle import oracle as o

pytestmark = pytest.mark.gpu

F32_RTOL, F32_ATOL = 2e-5, 2e-6


def close32(got, ref):
    np.testing.assert_allclose(got, ref, rtol=F32_RTOL, atol=F32_ATOL * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("seed", [0, 42, 999])
def test_fp64_matches_oracle(seed):
    from kernelforge_b200 import local_kernels as lk
    X1, _, Q1, N1 = make_set(4, 6, 8, 3, seed)
    X2, _, Q2, N2 = make_set(5, 6, 8, 3, seed + 1)
    np.testing.assert_allclose(lk.kernel_gaussian(X1, X2, Q1, Q2, N1, N2, 2.5),
                               o.kernel_gaussian(X1, X2, Q1, Q2, N1, N2, 2.5), rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(lk.kernel_gaussian_symm(X1, Q1, N1, 2.5),
                               o.kernel_gaussian_symm(X1, Q1, N1, 2.5), rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(lk.kernel_gaussian_symm_rfp(X1, Q1, N1, 2.5),
                               o.kernel_gaussian_symm_rfp(X1, Q1, N1, 2.5), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("precision", ["fp64", "fp32", "split_f16"])
def test_golden_random(precision):
    from kernelforge_b200 import local_kernels as lk
    g = load_golden("golden_random.npz")
    s = float(g["sigma"])
    got = [lk.kernel_gaussian(g["X1"], g["X2"], g["Q1"], g["Q2"], g["N1"], g["N2"], s,
                              precision=precision),
           lk.kernel_gaussian_symm(g["X1"], g["Q1"], g["N1"], s, precision=precision),
           lk.kernel_gaussian_symm_rfp(g["X1"], g["Q1"], g["N1"], s, precision=precision)]
    ref = [g["kernel_gaussian"], g["kernel_gaussian_symm"], g["kernel_gaussian_symm_rfp"]]
    for a, b in zip(got, ref):
        if precision == "fp64":
            np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-13)
        else:
            close32(a, b)


@pytest.mark.parametrize("precision", ["fp64", "split_f16"])
def test_golden_fchl19_720(precision):
    from kernelforge_b200 import local_kernels as lk
    g = load_golden("golden_fchl19_720.npz")
    got = lk.kernel_gaussian_symm_rfp(g["X"], g["Q"], g["N"], 2.0, precision=precision)
    if precision == "fp64":
        np.testing.assert_allclose(got, g["kernel_gaussian_symm_rfp"], rtol=1e-12, atol=1e-12)
    else:
        close32(got, g["kernel_gaussian_symm_rfp"])


@pytest.mark.parametrize("rep", [9, 16, 70, 130, 720])
@pytest.mark.parametrize("precision", ["fp64", "fp32", "split_f16"])
def test_multi_tile_ragged(rep, precision):
    """Buckets of several hundred rows: several tiles per label, molecules that
    straddle tile edges, diagonal and off-diagonal tiles, partial K slices."""
    from kernelforge_b200 import local_kernels as lk
    X, _, Q, N = make_set(90, 12, rep, 2, rep, species=[1, 6])
    X *= 0.3
    N[5] = 0
    N[7] = 40   # clamped to max_atoms
    sig = 2.0
    ref = o.kernel_gaussian_symm(X, Q, N, sig)
    got = lk.kernel_gaussian_symm(X, Q, N, sig, precision=precision)
    rfp = lk.kernel_gaussian_symm_rfp(X, Q, N, sig, precision=precision)
    X2, _, Q2, N2 = make_set(50, 9, rep, 2, rep + 1, species=[6, 1])
    X2 *= 0.3
    rect = lk.kernel_gaussian(X, X2, Q, Q2, N, N2, sig, precision=precision)
    rref = o.kernel_gaussian(X, X2, Q, Q2, N, N2, sig)
    if precision == "fp64":
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(rfp, o.full_to_rfp(ref), rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(rect, rref, rtol=1e-12, atol=1e-12)
    else:
        close32(got, ref)
        close32(rfp, o.full_to_rfp(ref))
        close32(rect, rref)


def test_no_shared_labels_gives_zero():
    from kernelforge_b200 import local_kernels as lk
    X1, _, Q1, N1 = make_set(3, 4, 6, 1, 0, species=[1])
    X2, _, Q2, N2 = make_set(4, 4, 6, 1, 1, species=[8])
    for prec in ("fp64", "split_f16"):
        K = lk.kernel_gaussian(X1, X2, Q1, Q2, N1, N2, 1.0, precision=prec)
        assert K.shape == (3, 4) and not K.any()


def test_symmetry_and_psd():
    from kernelforge_b200 import local_kernels as lk
    X, _, Q, N = make_set(30, 8, 20, 3, 3)
    K = lk.kernel_gaussian_symm(X, Q, N, 3.0)
    np.testing.assert_allclose(K, K.T, rtol=0, atol=1e-12)
    assert np.linalg.eigvalsh(K).min() > -1e-10
    assert (K >= 0).all()


def test_torch_api_rfp_lower_and_dtypes():
    import torch

    from kernelforge_b200 import cuda_local_kernels as clk
    g = load_golden("golden_fchl19_720.npz")
    X = torch.tensor(g["X"], dtype=torch.float32, device="cuda")
    Q = torch.tensor(g["Q"], device="cuda")
    N = torch.tensor(g["N"], device="cuda")
    rfp = clk.kernel_gaussian_symm_rfp(X, Q, N, 2.0)
    assert rfp.dtype == torch.float32 and rfp.is_cuda
    K = g["kernel_gaussian_symm"]
    close32(rfp.cpu().numpy(), o.full_to_rfp(K, uplo_lower=True))
    Kd = clk.kernel_gaussian_symm(X, Q, N, 2.0)
    assert Kd.dtype == torch.float64 and tuple(Kd.shape) == K.shape
    close32(Kd.cpu().numpy(), K)
    Kr = clk.kernel_gaussian_rect(X[:3], Q[:3], N[:3], X, Q, N, 2.0)
    close32(Kr.cpu().numpy(), K[:3])


def test_tensor_core_path_is_deterministic_in_value():
    from kernelforge_b200 import local_kernels as lk
    X, _, Q, N = make_set(60, 10, 64, 2, 5)
    a = lk.kernel_gaussian_symm_rfp(X, Q, N, 2.0, precision="split_f16")
    b = lk.kernel_gaussian_symm_rfp(X, Q, N, 2.0, precision="split_f16")
    # atomics may add in a different order: equal to FP32 rounding
    np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6 * np.abs(a).max())


@pytest.mark.parametrize("chunks", ["1", "3", "8"])
@pytest.mark.parametrize("rep", [70, 720])
def test_host_input_pipelined(chunks, rep, monkeypatch):
    """X in (page-locked) host memory: copies in chunks of molecules overlapped
    with the tile waves.  A label that first appears in a late chunk (oxygen
    only in the last molecules) is centred on that chunk's rows; empty
    molecules and clamped counts as in the device-input tests."""
    import torch

    from kernelforge_b200 import cuda_local_kernels as clk
    monkeypatch.setenv("KFB_H2D_CHUNKS", chunks)
    X, _, Q, N = make_set(90, 12, rep, 2, rep + 7, species=[1, 6])
    X = (X * 0.3).astype(np.float32)
    Q[80:, :3] = 8   # a label present only in the last chunk(s)
    N[80:] = np.maximum(N[80:], 3)
    N[5] = 0
    N[7] = 40   # clamped to max_atoms
    sig = 2.0
    Xh = torch.from_numpy(X).pin_memory()
    rfp = clk.kernel_gaussian_symm_rfp(Xh, Q, N, sig)
    assert rfp.is_cuda and rfp.dtype == torch.float32
    ref = o.kernel_gaussian_symm(X.astype(np.float64), Q, N, sig)
    close32(rfp.cpu().numpy(), o.full_to_rfp(ref, uplo_lower=True))
    dev = clk.kernel_gaussian_symm_rfp(torch.tensor(X, device="cuda"), Q, N, sig)
    np.testing.assert_allclose(rfp.cpu().numpy(), dev.cpu().numpy(), rtol=2e-5,
                               atol=2e-6 * float(dev.abs().max()))
    Kd = clk.kernel_gaussian_symm(Xh, Q, N, sig)
    close32(Kd.cpu().numpy(), ref)


@pytest.mark.parametrize("precision", ["fp64", "split_f16"])
def test_host_input_c_abi_f64(precision):
    """kfb_kernel_gaussian_symm_host with FP64 descriptors in host memory: the
    split-fp16 path pipelines the copy, the FP64 path copies once and runs the
    device-input kernel; dense FP64 output against the oracle."""
    import torch

    from kernelforge_b200 import _lib
    from kernelforge_b200._device import stream_handle
    X, _, Q, N = make_set(40, 10, 70, 3, 11)
    X = np.ascontiguousarray(X * 0.3)
    nm, ma, rep = X.shape
    out = torch.empty((nm * nm,), dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().kfb_kernel_gaussian_symm_host(
        X.ctypes.data, Q.ctypes.data, N.ctypes.data, nm, ma, rep, 2.0, _lib.KFB_F64,
        _lib.PREC[precision], _lib.KFB_DENSE, _lib.KFB_F64, out.data_ptr(), stream_handle()))
    torch.cuda.synchronize()
    ref = o.kernel_gaussian_symm(X, Q, N, 2.0)
    got = out.view(nm, nm).cpu().numpy()
    if precision == "fp64":
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12)
    else:
        close32(got, ref)


def test_host_input_more_chunks_than_molecules(monkeypatch):
    """Host-memory descriptors of 5 molecules with 8 chunks requested: one
    molecule per chunk."""
    import torch

    from kernelforge_b200 import cuda_local_kernels as clk
    monkeypatch.setenv("KFB_H2D_CHUNKS", "8")
    X, _, Q, N = make_set(5, 9, 32, 2, 77, species=[1, 6])
    X = (X * 0.3).astype(np.float32)
    rfp = clk.kernel_gaussian_symm_rfp(torch.from_numpy(X).pin_memory(), Q, N, 2.0)
    ref = o.kernel_gaussian_symm(X.astype(np.float64), Q, N, 2.0)
    close32(rfp.cpu().numpy(), o.full_to_rfp(ref, uplo_lower=True))
