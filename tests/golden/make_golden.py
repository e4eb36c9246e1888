"""Generate the golden fixtures of tests/golden/ from the reference itself.

Builds the reference's CPU FP64 modules (local_kernels, kernelmath, fchl19_repr)
from its sources with oracle/build_ref.sh, runs them on small seeded inputs and
stores inputs and outputs as compressed .npz files:

* golden_random.npz  -- random-normal descriptors (the shapes and value
  distribution the reference's unit tests use: a few molecules, few atoms,
  small rep, three species, ragged N), all eleven kernel functions;
* golden_fchl19.npz  -- synthetic molecules (H/C/N/O) with reference FCHL19
  descriptors and Jacobians (reduced basis: elements 1,6,7,8, nRs2=8, nRs3=6,
  rep 152), the kernels on them, RFP packings and a Cholesky solve;
* golden_fchl19_720.npz -- default 720-dim FCHL19 descriptors of a few
  molecules (no Jacobians) and the scalar kernels on them.

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT   (or KERNELFORGE_REFERENCE_ROOT set)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kernelforge_b200 import synthetic  # noqa: E402


def main(ref_root):
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh"), ref_root])
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import fchl19_repr as fr
    import kernelmath as km
    import local_kernels as lk

    sigma = 2.5
    # ------------------------------------------------------------ random
    rng = np.random.default_rng(20261203)
    nm1, nm2, ma, rep = 7, 5, 6, 9
    X1 = rng.standard_normal((nm1, ma, rep))
    X2 = rng.standard_normal((nm2, ma, rep))
    N1 = rng.integers(1, ma + 1, size=nm1).astype(np.int32)
    N2 = rng.integers(1, ma + 1, size=nm2).astype(np.int32)
    N1[2] = 0                      # an empty molecule
    Q1 = np.zeros((nm1, ma), np.int32)
    Q2 = np.zeros((nm2, ma), np.int32)
    for a in range(nm1):
        Q1[a, :N1[a]] = rng.choice([1, 2, 3], size=N1[a])
    for b in range(nm2):
        Q2[b, :N2[b]] = rng.choice([1, 2, 3], size=N2[b])
    dX1 = rng.standard_normal((nm1, ma, rep, 3 * ma))
    dX2 = rng.standard_normal((nm2, ma, rep, 3 * ma))
    out = dict(X1=X1, X2=X2, Q1=Q1, Q2=Q2, N1=N1, N2=N2, dX1=dX1, dX2=dX2, sigma=sigma)
    out["kernel_gaussian"] = lk.kernel_gaussian(X1, X2, Q1, Q2, N1, N2, sigma)
    out["kernel_gaussian_symm"] = lk.kernel_gaussian_symm(X1, Q1, N1, sigma)
    out["kernel_gaussian_symm_rfp"] = lk.kernel_gaussian_symm_rfp(X1, Q1, N1, sigma)
    out["kernel_gaussian_jacobian"] = lk.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2,
                                                                  sigma)
    out["kernel_gaussian_jacobian_t"] = lk.kernel_gaussian_jacobian_t(X1, dX1, X2, Q1, Q2, N1,
                                                                      N2, sigma)
    out["kernel_gaussian_hessian"] = lk.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2,
                                                                sigma)
    out["kernel_gaussian_hessian_symm"] = lk.kernel_gaussian_hessian_symm(X1, dX1, Q1, N1, sigma)
    out["kernel_gaussian_hessian_symm_rfp"] = lk.kernel_gaussian_hessian_symm_rfp(X1, dX1, Q1,
                                                                                  N1, sigma)
    out["kernel_gaussian_full"] = lk.kernel_gaussian_full(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma)
    out["kernel_gaussian_full_symm"] = lk.kernel_gaussian_full_symm(X1, dX1, Q1, N1, sigma)
    out["kernel_gaussian_full_symm_rfp"] = lk.kernel_gaussian_full_symm_rfp(X1, dX1, Q1, N1,
                                                                            sigma)
    np.savez_compressed(os.path.join(HERE, "golden_random.npz"), **out)

    # ------------------------------------------------------------ FCHL19 (reduced basis)
    mols = synthetic.make_molecules(6, 4, 8, seed=7)
    elements = [1, 6, 7, 8]
    ma = max(len(z) for z in mols.Z)
    reps, grads = [], []
    for m in range(mols.nm):
        r, g = fr.generate_fchl_acsf_and_gradients(mols.R[m], mols.Z[m], elements=elements,
                                                    nRs2=8, nRs3=6)
        reps.append(r)
        grads.append(g)
    rep = reps[0].shape[1]
    X = np.zeros((mols.nm, ma, rep))
    dX = np.zeros((mols.nm, ma, rep, 3 * ma))
    Q = np.zeros((mols.nm, ma), np.int32)
    N = np.zeros((mols.nm,), np.int32)
    for m in range(mols.nm):
        n = len(mols.Z[m])
        X[m, :n] = reps[m]
        dX[m, :n, :, :3 * n] = grads[m]
        Q[m, :n] = mols.Z[m]
        N[m] = n
    sig = 2.0
    g = dict(X=X, dX=dX, Q=Q, N=N, sigma=sig, E=mols.E,
             coords=np.concatenate(mols.R), Z=np.concatenate(mols.Z), natoms=N.copy())
    g["kernel_gaussian_symm_rfp"] = lk.kernel_gaussian_symm_rfp(X, Q, N, sig)
    g["kernel_gaussian"] = lk.kernel_gaussian(X[:4], X[2:], Q[:4], Q[2:], N[:4], N[2:], sig)
    g["kernel_gaussian_jacobian"] = lk.kernel_gaussian_jacobian(X[:4], X[2:], dX[2:], Q[:4],
                                                                Q[2:], N[:4], N[2:], sig)
    g["kernel_gaussian_hessian_symm_rfp"] = lk.kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, sig)
    g["kernel_gaussian_full_symm_rfp"] = lk.kernel_gaussian_full_symm_rfp(X, dX, Q, N, sig)
    K = lk.kernel_gaussian_symm(X, Q, N, sig)
    g["full_to_rfp_U"] = km.full_to_rfp(K, uplo="U")
    g["full_to_rfp_L"] = km.full_to_rfp(K, uplo="L")
    g["full_to_rfp_U_T"] = km.full_to_rfp(K, uplo="U", transr="T")
    y = mols.E - mols.E.mean()
    g["cho_y"] = y
    g["cho_l2"] = 1e-6
    g["cho_alpha"] = km.cho_solve_rfp(g["kernel_gaussian_symm_rfp"].copy(), y, l2=1e-6)
    np.savez_compressed(os.path.join(HERE, "golden_fchl19.npz"), **g)

    # ------------------------------------------------------------ FCHL19 720-dim
    mols = synthetic.make_molecules(5, 5, 9, seed=11)
    ma = max(len(z) for z in mols.Z)
    X = np.zeros((mols.nm, ma, 720))
    Q = np.zeros((mols.nm, ma), np.int32)
    N = np.zeros((mols.nm,), np.int32)
    for m in range(mols.nm):
        n = len(mols.Z[m])
        X[m, :n] = fr.generate_fchl_acsf(mols.R[m], mols.Z[m])
        Q[m, :n] = mols.Z[m]
        N[m] = n
    h = dict(X=X, Q=Q, N=N, sigma=2.0, coords=np.concatenate(mols.R),
             Z=np.concatenate(mols.Z), natoms=N.copy())
    h["kernel_gaussian_symm"] = lk.kernel_gaussian_symm(X, Q, N, 2.0)
    h["kernel_gaussian_symm_rfp"] = lk.kernel_gaussian_symm_rfp(X, Q, N, 2.0)
    np.savez_compressed(os.path.join(HERE, "golden_fchl19_720.npz"), **h)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, HERE)
    from _refroot import reference_root
    main(reference_root(sys.argv[1:]))
