"""Golden fixtures of the elemental random-Fourier-feature comparator, from the
reference itself.

Builds the reference's CPU FP64 `kitchen_sinks` module (src/rff_features.cpp,
src/rff_elemental.cpp and their bindings) with oracle/build_ref.sh and runs
rff_features_elemental and rff_gramian_elemental_rfp on

* the default 720-dim FCHL19 descriptors of golden_fchl19_720.npz (elements
  H/C/N/O mapped to indices 0..3), D = 64;
* random-normal descriptors with ragged sizes, one empty molecule and three
  element types, rep 32, D = 48.

W ~ N(0, 1) / sigma and b ~ U(0, 2 pi) as in the reference's LocalRFFModel
(models/rff.py:110-112).  Output: tests/golden/golden_rff.npz.

Usage:  python tests/golden/make_golden_rff.py REFERENCE_ROOT   (or KERNELFORGE_REFERENCE_ROOT set)
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main(ref_root):
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh"), ref_root])
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import kitchen_sinks as ks

    out = {}
    sigma = 2.0
    # ------------------------------------------------------ FCHL19 720-dim
    g = np.load(os.path.join(HERE, "golden_fchl19_720.npz"))
    X, Qz, N = g["X"], g["Q"], g["N"]
    elements = [1, 6, 7, 8]
    Qe = np.full(Qz.shape, -1, np.int32)
    for m in range(X.shape[0]):
        for j in range(N[m]):
            Qe[m, j] = elements.index(int(Qz[m, j]))
    rng = np.random.default_rng(20261205)
    D = 64
    W = rng.standard_normal((len(elements), X.shape[2], D)) / sigma
    b = rng.uniform(0.0, 2.0 * np.pi, (len(elements), D))
    Y = rng.standard_normal(X.shape[0])
    Ql = [Qe[m, :N[m]].copy() for m in range(X.shape[0])]
    out.update(f_X=X, f_Q=Qe, f_N=N.astype(np.int32), f_W=W, f_b=b, f_Y=Y)
    out["f_Z"] = ks.rff_features_elemental(X, Ql, W, b)
    ztz, zty = ks.rff_gramian_elemental_rfp(X, Ql, W, b, Y, 2)
    out["f_ZtZ_rfp"], out["f_ZtY"] = ztz, zty
    # ------------------------------------------------------ random, ragged
    nm, ma, rep, D2 = 9, 7, 32, 48
    Xr = rng.standard_normal((nm, ma, rep)) * 0.3
    Nr = rng.integers(1, ma + 1, size=nm).astype(np.int32)
    Nr[4] = 0
    Qr = np.full((nm, ma), -1, np.int32)
    for m in range(nm):
        Qr[m, :Nr[m]] = rng.integers(0, 3, size=Nr[m])
    Xr[Qr < 0] = 0.0
    Wr = rng.standard_normal((3, rep, D2)) / sigma
    br = rng.uniform(0.0, 2.0 * np.pi, (3, D2))
    Yr = rng.standard_normal(nm)
    Qlr = [Qr[m, :Nr[m]].copy() for m in range(nm)]
    out.update(r_X=Xr, r_Q=Qr, r_N=Nr, r_W=Wr, r_b=br, r_Y=Yr)
    out["r_Z"] = ks.rff_features_elemental(Xr, Qlr, Wr, br)
    ztz, zty = ks.rff_gramian_elemental_rfp(Xr, Qlr, Wr, br, Yr, 3)
    out["r_ZtZ_rfp"], out["r_ZtY"] = ztz, zty
    np.savez_compressed(os.path.join(HERE, "golden_rff.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_rff.npz"))


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _refroot import reference_root
    main(reference_root(sys.argv[1:]))
