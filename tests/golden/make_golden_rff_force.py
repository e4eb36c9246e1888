"""Golden fixtures of the elemental random-Fourier-feature force path
(rff_gradient_elemental and rff_full_gramian_elemental_rfp,
src/rff_elemental.cpp:363-500, :799-935), from the reference itself.

Runs the reference's CPU FP64 `kitchen_sinks` module (oracle/build_ref.sh) on
* the reduced-basis FCHL19 molecules of golden_fchl19.npz (real Jacobians,
  elements H/C/N/O -> 0..3), D = 40;
* random-normal descriptors and Jacobians, ragged sizes, one empty molecule,
  three element types, rep 24, D = 32.
W ~ N(0, 1) / sigma, b ~ U(0, 2 pi).  Output: tests/golden/golden_rff_force.npz.

Usage:  python tests/golden/make_golden_rff_force.py REFERENCE_ROOT   (or KERNELFORGE_REFERENCE_ROOT set)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def case(ks, out, tag, X, dX, Qe, N, D, sigma, rng):
    nel = int(Qe.max()) + 1
    W = rng.standard_normal((nel, X.shape[2], D)) / sigma
    b = rng.uniform(0.0, 2.0 * np.pi, (nel, D))
    Y = rng.standard_normal(X.shape[0])
    F = rng.standard_normal(int(3 * N.sum()))
    Ql = [Qe[m, :N[m]].copy() for m in range(X.shape[0])]
    out.update({f"{tag}_X": X, f"{tag}_dX": dX, f"{tag}_Q": Qe, f"{tag}_N": N, f"{tag}_W": W,
                f"{tag}_b": b, f"{tag}_Y": Y, f"{tag}_F": F})
    dX5 = dX.reshape(dX.shape[0], dX.shape[1], dX.shape[2], dX.shape[1], 3)  # the module's 5-D form
    out[f"{tag}_G"] = ks.rff_gradient_elemental(X, dX5, Ql, W, b)         # (D, ngrads)
    ztz, zty = ks.rff_full_gramian_elemental_rfp(X, dX5, Ql, W, b, Y, F, 2, 2)
    out[f"{tag}_ZtZ_rfp"], out[f"{tag}_ZtY"] = ztz, zty


def main(ref_root):
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh"), ref_root])
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import kitchen_sinks as ks

    rng = np.random.default_rng(20261208)
    out = {}
    g = np.load(os.path.join(HERE, "golden_fchl19.npz"))
    X, dX, Qz, N = g["X"], g["dX"], g["Q"], g["N"].astype(np.int32)
    Qe = np.full(Qz.shape, -1, np.int32)
    for m in range(X.shape[0]):
        for j in range(N[m]):
            Qe[m, j] = [1, 6, 7, 8].index(int(Qz[m, j]))
    case(ks, out, "f", X, dX, Qe, N, 40, 2.0, rng)
    nm, ma, rep = 7, 6, 24
    N = rng.integers(1, ma + 1, size=nm).astype(np.int32)
    N[3] = 0
    Qe = np.full((nm, ma), -1, np.int32)
    for m in range(nm):
        Qe[m, :N[m]] = rng.integers(0, 3, size=N[m])
    X = rng.standard_normal((nm, ma, rep)) * 0.3
    dX = rng.standard_normal((nm, ma, rep, 3 * ma)) * 0.2
    X[Qe < 0] = 0.0
    case(ks, out, "r", X, dX, Qe, N, 32, 1.5, rng)
    np.savez_compressed(os.path.join(HERE, "golden_rff_force.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_rff_force.npz"))


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _refroot import reference_root
    main(reference_root(sys.argv[1:]))
