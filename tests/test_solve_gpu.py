"""RFP Cholesky / solve on the GPU: FP64 cho_solve_rfp against the oracle and the
reference's golden solve; rfp_potrf / rfp_potrs (both UPLO, odd and even n)
against LAPACK's dpftrf; the mixed-precision solve reaches its tolerance."""
import numpy as np
import pytest
import scipy.linalg.lapack as lapack

from conftest import load_golden
from oracle import oracle as o

pytestmark = pytest.mark.gpu


def spd(n, seed, cond=1e3):
    rng = np.random.default_rng(seed)
    Qm, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.logspace(0, np.log10(cond), n)
    return (Qm * ev) @ Qm.T


@pytest.mark.parametrize("n", [1, 2, 7, 8, 65, 130])
def test_cho_solve_rfp_matches_oracle(n):
    from kernelforge_b200 import kernelmath as km
    A = spd(n, n)
    y = np.random.default_rng(1).standard_normal(n)
    arf = o.full_to_rfp(A)
    mine = arf.copy()
    alpha = km.cho_solve_rfp(mine, y, l2=1e-3)
    ref_arf = arf.copy()
    ref = o.cho_solve_rfp(ref_arf, y, 1e-3)
    np.testing.assert_allclose(alpha, ref, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(mine, ref_arf, rtol=1e-10, atol=1e-12)  # factor written back


def test_cho_solve_rfp_golden():
    from kernelforge_b200 import kernelmath as km
    g = load_golden("golden_fchl19.npz")
    alpha = km.cho_solve_rfp(g["kernel_gaussian_symm_rfp"].copy(), g["cho_y"], float(g["cho_l2"]))
    np.testing.assert_allclose(alpha, g["cho_alpha"], rtol=1e-7, atol=1e-9)


def test_cho_solve_rfp_not_pd():
    from kernelforge_b200 import kernelmath as km
    with pytest.raises(RuntimeError, match="info"):
        km.cho_solve_rfp(o.full_to_rfp(-np.eye(5)), np.ones(5))


def test_full_to_rfp_and_back_match_reference():
    from kernelforge_b200 import kernelmath as km
    g = load_golden("golden_fchl19.npz")
    K = o.rfp_to_full(g["kernel_gaussian_symm_rfp"], g["N"].shape[0])
    np.testing.assert_allclose(km.full_to_rfp(K, uplo="U"), g["full_to_rfp_U"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(km.full_to_rfp(K, uplo="L"), g["full_to_rfp_L"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(km.full_to_rfp(K, uplo="U", transr="T"), g["full_to_rfp_U_T"],
                               rtol=0, atol=1e-14)
    np.testing.assert_allclose(km.rfp_to_full(g["full_to_rfp_U"], K.shape[0], uplo="U"), K,
                               rtol=0, atol=1e-14)


@pytest.mark.parametrize("n", [5, 6, 63, 64, 257])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_rfp_potrf_potrs_match_lapack(n, uplo, dtype):
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    A = spd(n, n + 3, cond=50.0)
    arf, info = lapack.dtrttf(np.asfortranarray(A), transr="N", uplo=uplo)
    ref, info = lapack.dpftrf(n, (arf + 0.0).copy(), transr="N", uplo=uplo)
    tdt = getattr(torch, dtype)
    K = torch.tensor(arf, dtype=tdt, device="cuda")
    assert cgk.rfp_potrf(K, n, 0.0, uplo) == 0
    tol = 1e-11 if dtype == "float64" else 2e-4
    np.testing.assert_allclose(K.cpu().numpy(), ref, rtol=tol, atol=tol)
    b = np.random.default_rng(n).standard_normal(n)
    B = torch.tensor(b, dtype=tdt, device="cuda").reshape(n, 1).contiguous()
    cgk.rfp_potrs(K, B, uplo)
    np.testing.assert_allclose(A @ B.cpu().numpy().ravel(), b, rtol=50 * tol, atol=50 * tol)


def test_rfp_potrf_reports_info():
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    A = np.eye(6)
    A[3, 3] = -1.0
    K = torch.tensor(o.full_to_rfp(A, uplo_lower=True), dtype=torch.float32, device="cuda")
    assert cgk.rfp_potrf(K, 6, 0.0, "L") == 4


def test_mixed_solve_reaches_tolerance():
    """A real FCHL19 kernel matrix (FP32 RFP) at lambda = 1e-8: the FP64 residual
    of the returned alpha against the FP32-stored matrix is below 1e-10."""
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    from kernelforge_b200 import cuda_local_kernels as clk
    from kernelforge_b200 import synthetic
    mols = synthetic.make_molecules(300, 9, 21, seed=3)
    X, Q, N = synthetic.fchl19_batched(mols, dtype=np.float32)
    K = clk.kernel_gaussian_symm_rfp(torch.tensor(X, device="cuda"), Q, N, 2.0)
    y = mols.E - mols.E.mean()
    n = len(y)
    alpha, info = cgk.krr_solve_mixed(K, torch.tensor(y), l2=1e-8, uplo="L", tol=1e-10)
    assert info["converged"], info
    A32 = o.rfp_to_full(K.cpu().numpy().astype(np.float64), n, uplo_lower=True)
    r = y - (A32 + 1e-8 * np.eye(n)) @ alpha.cpu().numpy()
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(y)


def test_mixed_solve_matches_fp64_solution_when_well_conditioned():
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    n = 200
    A = spd(n, 9, cond=1e4)
    y = np.random.default_rng(4).standard_normal(n)
    K = torch.tensor(o.full_to_rfp(A, uplo_lower=True), dtype=torch.float32, device="cuda")
    A32 = o.rfp_to_full(K.cpu().numpy().astype(np.float64), n, uplo_lower=True)
    alpha, info = cgk.krr_solve_mixed(K, torch.tensor(y), l2=0.0, uplo="L", tol=1e-12)
    assert info["converged"], info
    np.testing.assert_allclose(alpha.cpu().numpy(), np.linalg.solve(A32, y), rtol=1e-9, atol=1e-11)


@pytest.mark.parametrize("factor", ["fp32", "fp64"])
def test_mixed_solve_factor_choice(factor):
    """Both factor precisions converge to the FP64 solution of the FP32-stored
    system; the FP64 factor needs at most two refinement steps."""
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    from kernelforge_b200 import cuda_local_kernels as clk
    from kernelforge_b200 import synthetic
    mols = synthetic.make_molecules(400, 9, 21, seed=5)
    X, Q, N = synthetic.fchl19_batched(mols, dtype=np.float32)
    K = clk.kernel_gaussian_symm_rfp(torch.tensor(X, device="cuda"), Q, N, 2.0)
    y = mols.E - mols.E.mean()
    n = len(y)
    alpha, info = cgk.krr_solve_mixed(K, torch.tensor(y), l2=1e-2, uplo="L", tol=1e-11,
                                      factor=factor)
    assert info["converged"], info
    A32 = o.rfp_to_full(K.cpu().numpy().astype(np.float64), n, uplo_lower=True)
    ref = np.linalg.solve(A32 + 1e-2 * np.eye(n), y)
    np.testing.assert_allclose(alpha.cpu().numpy(), ref, rtol=1e-7,
                               atol=1e-7 * np.abs(ref).max())
    if factor == "fp64":
        assert info["iterations"] <= 3, info


@pytest.mark.parametrize("factor", ["fp32", "fp64"])
def test_mixed_solve_many_row_blocks(factor):
    """Refinement at n = 9,700: for the FP64 factor, 152 row blocks of the
    blocked triangular solves, more than one per CTA on a 148-SM device, and a
    ragged last block."""
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    n = 9700
    rng = np.random.default_rng(21)
    B = rng.normal(size=(n, 48))
    A32 = (B @ B.T / 48.0 + 0.5 * np.eye(n)).astype(np.float32)
    y = rng.normal(size=n)
    K = torch.tensor(o.full_to_rfp(A32.astype(np.float64), uplo_lower=True).astype(np.float32),
                     device="cuda")
    alpha, info = cgk.krr_solve_mixed(K, torch.tensor(y), l2=1e-3, uplo="L", tol=1e-11,
                                      factor=factor)
    assert info["converged"], info
    if factor == "fp64":
        assert info["iterations"] <= 3, info
    ref = np.linalg.solve(A32.astype(np.float64) + 1e-3 * np.eye(n), y)
    np.testing.assert_allclose(alpha.cpu().numpy(), ref, rtol=1e-8,
                               atol=1e-8 * np.abs(ref).max())


@pytest.mark.parametrize("n", [5, 64, 65, 130])
def test_mixed_solve_fp64_factor_small_orders(n):
    """FP64-factor refinement at orders around the 64-row blocks of the
    triangular sweeps (one block, exactly one, one plus a ragged row, two plus a
    ragged block)."""
    import torch

    from kernelforge_b200 import cuda_global_kernels as cgk
    rng = np.random.default_rng(100 + n)
    B = rng.normal(size=(n, n))
    A32 = (B @ B.T / n + 0.3 * np.eye(n)).astype(np.float32)
    y = rng.normal(size=n)
    K = torch.tensor(o.full_to_rfp(A32.astype(np.float64), uplo_lower=True).astype(np.float32),
                     device="cuda")
    alpha, info = cgk.krr_solve_mixed(K, torch.tensor(y), l2=1e-3, uplo="L", tol=1e-11,
                                      factor="fp64")
    assert info["converged"], info
    ref = np.linalg.solve(A32.astype(np.float64) + 1e-3 * np.eye(n), y)
    np.testing.assert_allclose(alpha.cpu().numpy(), ref, rtol=1e-8,
                               atol=1e-8 * np.abs(ref).max())
