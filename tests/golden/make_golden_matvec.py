"""Golden fixtures of the contracted energy/force prediction functions
(kernel_gaussian_local_compute_alpha_desc, _jacobian_t_matvec, _hessian_matvec,
_full_matvec; src/local_kernels.cpp:2821-3425), from the reference itself.

Builds the reference's CPU FP64 `local_kernels` module with oracle/build_ref.sh
and runs the four functions, plus kernel_gaussian_full (the uncontracted
kernel the predictions equal), on
* random-normal sets with ragged sizes, an empty molecule and three labels;
* the reduced-basis FCHL19 molecules of golden_fchl19.npz (real Jacobians).
Output: tests/golden/golden_matvec.npz.

Usage:  python tests/golden/make_golden_matvec.py REFERENCE_ROOT   (or KERNELFORGE_REFERENCE_ROOT set)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def run_case(lk, out, tag, X1, dX1, Q1, N1, X2, dX2, Q2, N2, sigma, rng):
    naq1, naq2 = int(3 * N1.sum()), int(3 * N2.sum())
    aE = rng.standard_normal(len(N2))
    aF = rng.standard_normal(naq2)
    ad = lk.kernel_gaussian_local_compute_alpha_desc(dX2, Q2, N2, aF)
    out.update({f"{tag}_X1": X1, f"{tag}_dX1": dX1, f"{tag}_Q1": Q1, f"{tag}_N1": N1,
                f"{tag}_X2": X2, f"{tag}_dX2": dX2, f"{tag}_Q2": Q2, f"{tag}_N2": N2,
                f"{tag}_sigma": sigma, f"{tag}_alpha_E": aE, f"{tag}_alpha_F": aF,
                f"{tag}_alpha_desc": ad})
    out[f"{tag}_jacobian_t_matvec"] = lk.kernel_gaussian_local_jacobian_t_matvec(
        X1, X2, ad, Q1, Q2, N1, N2, sigma)
    out[f"{tag}_hessian_matvec"] = lk.kernel_gaussian_local_hessian_matvec(
        X1, dX1, X2, ad, Q1, Q2, N1, N2, sigma)
    E, F = lk.kernel_gaussian_local_full_matvec(X1, dX1, X2, ad, aE, Q1, Q2, N1, N2, sigma)
    out[f"{tag}_full_matvec_E"], out[f"{tag}_full_matvec_F"] = E, F
    out[f"{tag}_kernel_gaussian_full"] = lk.kernel_gaussian_full(
        X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma)


def main(ref_root):
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh"), ref_root])
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import local_kernels as lk

    rng = np.random.default_rng(20261206)
    out = {}
    # random, ragged, three labels, an empty query molecule
    nm1, nm2, ma1, ma2, rep = 5, 6, 5, 6, 11
    X1 = rng.standard_normal((nm1, ma1, rep)) * 0.4
    X2 = rng.standard_normal((nm2, ma2, rep)) * 0.4
    N1 = rng.integers(1, ma1 + 1, nm1).astype(np.int32)
    N2 = rng.integers(1, ma2 + 1, nm2).astype(np.int32)
    N1[3] = 0
    Q1 = np.zeros((nm1, ma1), np.int32)
    Q2 = np.zeros((nm2, ma2), np.int32)
    for a in range(nm1):
        Q1[a, :N1[a]] = rng.choice([1, 6, 8], N1[a])
    for b in range(nm2):
        Q2[b, :N2[b]] = rng.choice([1, 6, 8], N2[b])
    dX1 = rng.standard_normal((nm1, ma1, rep, 3 * ma1)) * 0.3
    dX2 = rng.standard_normal((nm2, ma2, rep, 3 * ma2)) * 0.3
    run_case(lk, out, "r", X1, dX1, Q1, N1, X2, dX2, Q2, N2, 1.7, rng)
    # reduced-basis FCHL19 molecules
    g = np.load(os.path.join(HERE, "golden_fchl19.npz"))
    X, dX, Q, N = g["X"], g["dX"], g["Q"], g["N"]
    run_case(lk, out, "f", X[:3], dX[:3], Q[:3], N[:3], X[2:], dX[2:], Q[2:], N[2:],
             float(g["sigma"]), rng)
    np.savez_compressed(os.path.join(HERE, "golden_matvec.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_matvec.npz"))


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _refroot import reference_root
    main(reference_root(sys.argv[1:]))
