"""FCHL19 descriptors and Jacobians on the GPU (kfb_fchl19_repr) against the
reference's own outputs (tests/golden/golden_repr.npz) and the torch restatement.
FP64: X at rtol 1e-10, Jacobians at 1e-9 of their largest entry (both sides are
analytic); float32 storage (cuda_fchl19_repr): 1e-5."""
import ast
import math

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def golden():
    g = load_golden("golden_repr.npz")
    return g, ast.literal_eval(str(g["nondefault"]))


def close_x(got, ref, rtol=1e-10):
    np.testing.assert_allclose(got, ref, rtol=rtol, atol=rtol * max(1e-3, np.abs(ref).max()))


def close_g(got, ref, tol=1e-9):
    np.testing.assert_allclose(got, ref, rtol=tol, atol=tol * max(1e-3, np.abs(ref).max()))


@pytest.mark.parametrize("c", range(6))
def test_golden_default(c):
    from kernelforge_b200 import fchl19_repr as fr
    g, _ = golden()
    R, Z = g[f"d{c}_R"], g[f"d{c}_Z"]
    X = fr.generate_fchl_acsf(R, Z)
    assert X.shape == g[f"d{c}_X"].shape and X.dtype == np.float64
    close_x(X, g[f"d{c}_X"])
    X2, J = fr.generate_fchl_acsf_and_gradients(R, Z)
    close_x(X2, g[f"d{c}_X"])
    assert J.shape == g[f"d{c}_G"].shape
    close_g(J, g[f"d{c}_G"])


@pytest.mark.parametrize("c", range(3))
def test_golden_nondefault(c):
    from kernelforge_b200 import fchl19_repr as fr
    g, nd = golden()
    X, J = fr.generate_fchl_acsf_and_gradients(g[f"n{c}_R"], g[f"n{c}_Z"], **nd)
    close_x(X, g[f"n{c}_X"])
    close_g(J, g[f"n{c}_G"])


def test_golden_nfourier2():
    from kernelforge_b200 import fchl19_repr as fr
    g, _ = golden()
    X = fr.generate_fchl_acsf(g["f_R"].reshape(-1), g["f_Z"], elements=[1, 6, 7, 8],
                              nFourier=2)
    close_x(X, g["f_X"])


def test_batched_padding_and_float32():
    """Several molecules in one launch, padded; float32 storage through the
    torch-facing module with element indices."""
    import torch
    from kernelforge_b200 import cuda_fchl19_repr as cr
    from kernelforge_b200 import fchl19_repr as fr
    g, _ = golden()
    mols = [(g[f"d{c}_R"], g[f"d{c}_Z"]) for c in (2, 3, 4, 5)]
    nm, ma = len(mols), max(len(z) for _, z in mols)
    C = np.zeros((nm, ma, 3))
    Zp = np.zeros((nm, ma), np.int32)
    N = np.array([len(z) for _, z in mols], np.int32)
    for m, (R, Z) in enumerate(mols):
        C[m, :len(Z)] = R
        Zp[m, :len(Z)] = Z
    X, dX = fr.generate_batched(C, Zp, N, gradients=True, dtype="float64")
    X, dX = X.cpu().numpy(), dX.cpu().numpy()
    for m, (R, Z) in enumerate(mols):
        n = len(Z)
        close_x(X[m, :n], g[f"d{[2, 3, 4, 5][m]}_X"])
        close_g(dX[m, :n, :, :3 * n], g[f"d{[2, 3, 4, 5][m]}_G"])
        assert not X[m, n:].any() and not dX[m, n:].any() and not dX[m, :, :, 3 * n:].any()
    lut = {e: k for k, e in enumerate((1, 6, 7, 8, 16))}
    Q = np.vectorize(lambda z: lut.get(int(z), 0))(Zp).astype(np.int32)
    ct = torch.tensor(C, dtype=torch.float32, device="cuda")
    rep, grad = cr.generate_fchl_acsf_and_gradients(
        ct, torch.tensor(Q, device="cuda"), torch.tensor(N, device="cuda"), 5)
    assert rep.dtype == torch.float32 and tuple(grad.shape) == (nm, ma, 720, ma, 3)
    # float32 coordinates: compare with the FP64 result on the same rounded coordinates
    X32, dX32 = fr.generate_batched(C.astype(np.float32).astype(np.float64), Zp, N,
                                    gradients=True, dtype="float64")
    close_x(rep.double().cpu().numpy(), X32.cpu().numpy(), 1e-5)
    close_g(grad.double().cpu().numpy().reshape(dX32.shape), dX32.cpu().numpy(), 1e-5)
    rep2 = cr.generate_fchl_acsf(ct, torch.tensor(Q, device="cuda"),
                                 torch.tensor(N, device="cuda"), 5)
    assert torch.equal(rep2, rep)


def test_against_restatement_and_finite_differences():
    """A 16-atom molecule: the torch restatement (autograd) and central finite
    differences of the GPU descriptor itself."""
    import torch
    from kernelforge_b200 import fchl19_repr as fr
    from kernelforge_b200 import synthetic
    mols = synthetic.make_molecules(1, 16, 16, seed=5)
    R, Z = mols.R[0], mols.Z[0]
    X, J = fr.generate_fchl_acsf_and_gradients(R, Z)
    zi = synthetic._zidx(Z)
    f = lambda r: synthetic._fchl19_one(r, zi)
    Rt = torch.tensor(R, dtype=torch.float64)
    close_x(X, f(Rt).numpy())
    close_g(J, torch.func.jacfwd(f)(Rt).numpy().reshape(J.shape))
    h = 1e-5
    for a, t in [(0, 0), (7, 1), (15, 2)]:
        Rp, Rm = R.copy(), R.copy()
        Rp[a, t] += h
        Rm[a, t] -= h
        fd = (fr.generate_fchl_acsf(Rp, Z) - fr.generate_fchl_acsf(Rm, Z)) / (2 * h)
        np.testing.assert_allclose(J[:, :, 3 * a + t], fd, rtol=1e-5,
                                   atol=1e-6 * np.abs(J).max())


def test_edge_cases_and_errors():
    from kernelforge_b200 import fchl19_repr as fr
    X, J = fr.generate_fchl_acsf_and_gradients(np.zeros((1, 3)), [6])
    assert X.shape == (1, 720) and not X.any() and J.shape == (1, 720, 3) and not J.any()
    with pytest.raises(RuntimeError):
        fr.generate_fchl_acsf(np.zeros((2, 3)) + [[0, 0, 0], [1, 0, 0]], [6, 9])
    with pytest.raises(ValueError):
        fr.generate_fchl_acsf(np.zeros((3, 2)), [1, 1, 1])
    with pytest.raises(ValueError):
        fr.generate_fchl_acsf(np.zeros((0, 3)), [])
    with pytest.raises(ValueError):
        fr.generate_fchl_acsf_and_gradients(np.eye(3), [1, 1, 1], nFourier=2)
    assert fr.compute_rep_size(5, 24, 20, 2) == 720
