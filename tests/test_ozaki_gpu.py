"""FP64-class products on the int8 tensor cores (kfb_gemm_f64_i8) against
NumPy's FP64 product.

Error bound of the digit-slicing scheme with S planes per operand: each
operand row is truncated below 2 max|row| 2^-7S, and the dropped digit pairs
(p + q > S + 1) add at most ~4.03 S K max|A_i| max|B_j| 2^-7S, so per element
    |C - A B^T| <= (6 + 5 S) K 2^-7S max|A_i| max|B_j|
(plus FP64 rounding of the level sums, far below it).  The tests hold every
element to that bound; S = 7 is ~1e-13 relative for K of a few hundred."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gemm(A, B, S, C=None, alpha=1.0):
    import torch

    from kernelforge_b200 import _lib
    m, k = A.shape
    n = B.shape[0]
    a = torch.tensor(A, dtype=torch.float64, device="cuda")
    b = torch.tensor(B, dtype=torch.float64, device="cuda")
    c = (torch.tensor(C, dtype=torch.float64, device="cuda") if C is not None
         else torch.full((m, n), np.nan, dtype=torch.float64, device="cuda"))
    _lib.check(_lib.lib().kfb_gemm_f64_i8(m, n, k, alpha, a.data_ptr(), k, b.data_ptr(), k,
                                          1.0 if C is not None else 0.0, c.data_ptr(), n, S,
                                          torch.cuda.current_stream().cuda_stream))
    return c.cpu().numpy()


def bound(A, B, S):
    k = A.shape[1]
    ma = np.abs(A).max(axis=1)[:, None]
    mb = np.abs(B).max(axis=1)[None, :]
    return (6 + 5 * S) * k * 2.0 ** (-7 * S) * ma * mb


@pytest.mark.parametrize("S", [2, 4, 6, 7])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 64, 64), (300, 150, 720), (77, 200, 130)])
def test_matches_fp64_within_the_slicing_bound(S, m, n, k):
    rng = np.random.default_rng(1000 * S + m + n + k)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((n, k))
    A[0] *= 1e-3                      # rows of very different scale
    if m > 3:
        A[3] = 0.0                    # a zero row
    if n > 2:
        B[2] *= 1e5
    got = gemm(A, B, S)
    want = A @ B.T
    err = np.abs(got - want)
    assert np.all(err <= bound(A, B, S)), (err / bound(A, B, S)).max()


def test_seven_planes_are_fp64_class():
    """With 7 planes the error is at FP64 level relative to |A_i||B_j| (and
    ~1e7 x below FP32's)."""
    rng = np.random.default_rng(7)
    A = rng.standard_normal((256, 720))
    B = rng.standard_normal((192, 720))
    got = gemm(A, B, 7)
    want = A @ B.T
    scale = np.linalg.norm(A, axis=1)[:, None] * np.linalg.norm(B, axis=1)[None, :]
    assert (np.abs(got - want) / scale).max() < 1e-13
    f32 = (A.astype(np.float32) @ B.T.astype(np.float32)).astype(np.float64)
    assert (np.abs(f32 - want) / scale).max() > 1e-9


def test_accumulate_and_alpha():
    rng = np.random.default_rng(3)
    A = rng.standard_normal((200, 96))
    B = rng.standard_normal((70, 96))
    C = rng.standard_normal((200, 70))
    got = gemm(A, B, 7, C=C, alpha=-0.5)
    want = C - 0.5 * (A @ B.T)
    np.testing.assert_allclose(got, want, rtol=0, atol=(0.5 * bound(A, B, 7)).max() + 1e-15)


def test_rejects_bad_arguments():
    from kernelforge_b200 import _lib
    lib = _lib.lib()
    p = ctypes.c_void_p(16)
    assert lib.kfb_gemm_f64_i8(4, 4, 4, 1.0, p, 4, p, 4, 0.0, p, 4, 8, None) == \
        _lib.KFB_ERR_INVALID_ARG
    assert lib.kfb_gemm_f64_i8(4, 4, 4, 1.0, p, 4, p, 4, 0.5, p, 4, 7, None) == \
        _lib.KFB_ERR_INVALID_ARG
    assert lib.kfb_gemm_f64_i8(4, 4, 4, 1.0, p, 2, p, 4, 0.0, p, 4, 7, None) == \
        _lib.KFB_ERR_INVALID_ARG
