"""Jacobian / Hessian / full kernels on the GPU against the oracle and the
reference's golden outputs.  FP64: rtol 1e-10 (the reference's own tolerance
for these kernels); FP32: rtol 1e-4 relative to max|K|."""
import numpy as np
import pytest

from conftest import load_golden, make_set
from oracle import oracle as o

pytestmark = pytest.mark.gpu


def close(got, ref, precision):
    if precision == "fp64":
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * max(1.0, np.abs(ref).max()))
    else:
        np.testing.assert_allclose(got, ref, rtol=1e-3, atol=1e-4 * max(1.0, np.abs(ref).max()))


GOLDEN_CASES = [
    ("kernel_gaussian_jacobian", ("X1", "X2", "dX2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_jacobian_t", ("X1", "dX1", "X2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_hessian", ("X1", "dX1", "X2", "dX2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_hessian_symm", ("X1", "dX1", "Q1", "N1")),
    ("kernel_gaussian_hessian_symm_rfp", ("X1", "dX1", "Q1", "N1")),
    ("kernel_gaussian_full", ("X1", "dX1", "X2", "dX2", "Q1", "Q2", "N1", "N2")),
    ("kernel_gaussian_full_symm", ("X1", "dX1", "Q1", "N1")),
    ("kernel_gaussian_full_symm_rfp", ("X1", "dX1", "Q1", "N1")),
]


@pytest.mark.parametrize("name,args", GOLDEN_CASES)
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_golden_random(name, args, precision):
    from kernelforge_b200 import local_kernels as lk
    g = load_golden("golden_random.npz")
    got = getattr(lk, name)(*[g[a] for a in args], float(g["sigma"]), precision=precision)
    assert got.shape == g[name].shape
    close(got, g[name], precision)


def test_golden_fchl19():
    from kernelforge_b200 import local_kernels as lk
    g = load_golden("golden_fchl19.npz")
    X, dX, Q, N, s = g["X"], g["dX"], g["Q"], g["N"], float(g["sigma"])
    close(lk.kernel_gaussian_jacobian(X[:4], X[2:], dX[2:], Q[:4], Q[2:], N[:4], N[2:], s),
          g["kernel_gaussian_jacobian"], "fp64")
    close(lk.kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, s), g["kernel_gaussian_hessian_symm_rfp"],
          "fp64")
    close(lk.kernel_gaussian_full_symm_rfp(X, dX, Q, N, s), g["kernel_gaussian_full_symm_rfp"],
          "fp64")


@pytest.mark.parametrize("seed", [1, 2])
def test_larger_ragged_sets(seed):
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1 = make_set(9, 7, 33, 3, seed)
    X2, dX2, Q2, N2 = make_set(6, 5, 33, 3, seed + 10)
    X1 *= 0.4
    X2 *= 0.4
    s = 2.0
    close(lk.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s),
          o.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s), "fp64")
    close(lk.kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, s),
          o.kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, s), "fp64")
    close(lk.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s),
          o.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), "fp64")
    close(lk.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s),
          o.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), "fp64")


def test_jacobian_t_is_minus_jacobian_transposed():
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1 = make_set(5, 6, 10, 2, 3)
    X2, dX2, Q2, N2 = make_set(4, 6, 10, 2, 4)
    jt = lk.kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, 2.0)
    j = lk.kernel_gaussian_jacobian(X2, X1, dX1, Q2, Q1, N2, N1, 2.0)
    np.testing.assert_allclose(jt, -j.T, rtol=1e-12, atol=1e-12)


def test_full_symm_is_symmetric_and_matches_asym():
    from kernelforge_b200 import local_kernels as lk
    X, dX, Q, N = make_set(5, 5, 12, 2, 8)
    F = lk.kernel_gaussian_full_symm(X, dX, Q, N, 2.0)
    np.testing.assert_allclose(F, F.T, rtol=1e-12, atol=1e-12)
    Fa = lk.kernel_gaussian_full(X, dX, X, dX, Q, Q, N, N, 2.0)
    np.testing.assert_allclose(F, Fa, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("rep", [48, 720])
def test_tensor_core_contractions_match_oracle(rep):
    """precision='split_f16' runs the Jacobian and Hessian contraction GEMMs on
    the tcgen05 tensor cores (rep a multiple of 16): FP32-level agreement."""
    from kernelforge_b200 import local_kernels as lk
    X1, dX1, Q1, N1 = make_set(7, 6, rep, 3, 21)
    X2, dX2, Q2, N2 = make_set(5, 6, rep, 3, 22)
    sc = 1.0 / np.sqrt(rep)
    X1 *= 2 * sc
    X2 *= 2 * sc
    dX1 *= sc
    dX2 *= sc
    s = 2.0
    p = "split_f16"
    close(lk.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s), p)
    close(lk.kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1, N2, s), p)
    close(lk.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), p)
    close(lk.kernel_gaussian_hessian_symm_rfp(X1, dX1, Q1, N1, s, precision=p),
          o.kernel_gaussian_hessian_symm_rfp(X1, dX1, Q1, N1, s), p)
    close(lk.kernel_gaussian_full_symm_rfp(X1, dX1, Q1, N1, s, precision=p),
          o.kernel_gaussian_full_symm_rfp(X1, dX1, Q1, N1, s), p)
    close(lk.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), p)


@pytest.mark.parametrize("precision,rep", [("fp64", 33), ("fp32", 33), ("split_f16", 48)])
def test_jacobian_chunked_outer_molecules(precision, rep, monkeypatch):
    """A workspace of a few kB splits the outer molecules into chunks (each with
    its own dot-product block and label tiles).  Outer molecules lacking a label
    (zero rows of V), an outer label the inner set lacks, empty molecules and
    rep not a multiple of 4 (scalar row edges) on the CUDA-core paths."""
    from kernelforge_b200 import local_kernels as lk
    monkeypatch.setenv("KFB_WORKSPACE_GB", "0.00002")
    X1, dX1, Q1, N1 = make_set(9, 7, rep, 3, 31)
    X2, dX2, Q2, N2 = make_set(6, 5, rep, 3, 32)
    sc = 1.0 / np.sqrt(rep)
    X1 *= 2 * sc
    X2 *= 2 * sc
    dX1 *= sc
    dX2 *= sc
    Q1[2, :] = 1          # outer molecule with one label only
    Q1[4, :2] = 9         # an outer label the inner set lacks
    N1[6] = 0             # empty outer molecule
    s = 2.0
    if precision == "fp64":
        close(lk.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s),
              o.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s), "fp64")
        close(lk.kernel_gaussian_jacobian_t(X2, dX2, X1, Q2, Q1, N2, N1, s),
              o.kernel_gaussian_jacobian_t(X2, dX2, X1, Q2, Q1, N2, N1, s), "fp64")
    else:
        close(lk.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s, precision=precision),
              o.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s), precision)


@pytest.mark.parametrize("ma1,ma2", [(23, 5), (4, 23)])
def test_tensor_core_hessian_large_molecules(ma1, ma2):
    """Set-1 molecules of more than 21 atoms (more than 64 Jacobian rows) take
    the contraction with their Jacobian rows as M; smaller ones take the pairs'
    Y rows as M and 64-column tiles; 23-atom molecules b (69 columns of Y) are
    never merged into one problem.  Both sides, asymmetric and symmetric,
    against the oracle at the split-fp16 tolerance."""
    from kernelforge_b200 import local_kernels as lk
    rep = 48
    X1, dX1, Q1, N1 = make_set(4, ma1, rep, 3, 51, n_min=ma1 - 2)
    X2, dX2, Q2, N2 = make_set(3, ma2, rep, 3, 52, n_min=ma2 - 2)
    sc = 1.0 / np.sqrt(rep)
    X1 *= 2 * sc
    X2 *= 2 * sc
    dX1 *= sc
    dX2 *= sc
    s = 2.0
    p = "split_f16"
    close(lk.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), p)
    Xs, dXs, Qs, Ns = (X1, dX1, Q1, N1) if ma1 > ma2 else (X2, dX2, Q2, N2)
    close(lk.kernel_gaussian_hessian_symm_rfp(Xs, dXs, Qs, Ns, s, precision=p),
          o.kernel_gaussian_hessian_symm_rfp(Xs, dXs, Qs, Ns, s), p)


def test_tensor_core_hessian_disjoint_labels():
    """No atom of set 2 shares a label with set 1: every projection problem
    list is empty and the tensor-core Hessian is exactly zero."""
    from kernelforge_b200 import local_kernels as lk
    rep = 48
    X1, dX1, Q1, N1 = make_set(3, 6, rep, 1, 53, species=[1])
    X2, dX2, Q2, N2 = make_set(4, 6, rep, 1, 54, species=[2])
    H = lk.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, 2.0, precision="split_f16")
    assert H.shape == (int(3 * N1.sum()), int(3 * N2.sum()))
    assert not np.any(H)


@pytest.mark.parametrize("gb,ycore,path", [
    ("0.00005", None, ["hessian:rank-in-y", "hessian:y-cuda-core"]),
    ("0.0001", None, ["hessian:rank-kernel", "hessian:y-gemm"]),
    ("4", None, ["hessian:rank-kernel", "hessian:y-gemm"]),
    ("4", "cuda-core", ["hessian:rank-kernel", "hessian:y-cuda-core"])])
def test_hessian_tensor_core_batches(gb, ycore, path, monkeypatch):
    """Tensor-core Hessians with kernel 1 in GEMM form: a workspace of ~100 kB
    gives batches of a few molecule pairs spanning at most two molecules b (the
    projection buffer's capacity), the default one batch; symmetric RFP,
    asymmetric and full energy+force kernels against the oracle.  At ~54 kB the
    projection and rank buffers (18 kB each here) no longer fit half the
    workspace together, so the rank term stays inside Y (CUDA-core Y kernel);
    with the rank term outside, Y is a tensor-core GEMM per molecule b unless
    KFB_HESSIAN_Y=cuda-core keeps the CUDA-core kernel.  The path log shows
    which forms each call took."""
    from kernelforge_b200 import _lib
    from kernelforge_b200 import local_kernels as lk
    monkeypatch.setenv("KFB_WORKSPACE_GB", gb)
    if ycore:
        monkeypatch.setenv("KFB_HESSIAN_Y", ycore)
    rep = 48
    X1, dX1, Q1, N1 = make_set(7, 6, rep, 3, 41)
    X2, dX2, Q2, N2 = make_set(5, 6, rep, 3, 42)
    sc = 1.0 / np.sqrt(rep)
    X1 *= 2 * sc
    X2 *= 2 * sc
    dX1 *= sc
    dX2 *= sc
    Q2[1, :2] = 9   # a set-2 label set 1 lacks
    s = 2.0
    p = "split_f16"
    _lib.path_log_clear()
    close(lk.kernel_gaussian_hessian_symm_rfp(X1, dX1, Q1, N1, s, precision=p),
          o.kernel_gaussian_hessian_symm_rfp(X1, dX1, Q1, N1, s), p)
    assert _lib.path_log() == path
    _lib.path_log_clear()
    close(lk.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), p)
    assert _lib.path_log() == path
    close(lk.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s, precision=p),
          o.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s), p)
