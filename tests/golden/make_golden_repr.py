"""Golden fixtures of the FCHL19 descriptor and its Jacobian
(fchl19_repr.generate_fchl_acsf / generate_fchl_acsf_and_gradients,
src/fchl19_repr.cpp:89-781), from the reference itself.

Builds the reference's CPU FP64 modules with oracle/build_ref.sh and evaluates
* default hyper-parameters (H/C/N/O/S, 720 dims) on molecules of 1-12 atoms,
  including one spread over 20 A so that pairs fall beyond both cut-offs;
* non-default hyper-parameters (3 elements, other basis sizes, cut-offs,
  widths, decays and weight);
* nFourier = 2 (descriptor only: the reference's gradient path has the first
  harmonic only).
Output: tests/golden/golden_repr.npz.

Usage:  python tests/golden/make_golden_repr.py REFERENCE_ROOT   (or KERNELFORGE_REFERENCE_ROOT set)
"""
import math
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

NONDEFAULT = dict(elements=[1, 6, 8], nRs2=10, nRs3=8, nFourier=1, eta2=0.5, eta3=2.0,
                  zeta=2.5, rcut=5.0, acut=4.5, two_body_decay=1.5, three_body_decay=0.8,
                  three_body_weight=10.0)


def molecule(rng, n, box, elements, p=None):
    R = []
    while len(R) < n:
        x = rng.uniform(0, box, 3)
        if all(np.linalg.norm(x - y) > 0.9 for y in R):
            R.append(x)
    return np.array(R), rng.choice(elements, size=n, p=p).astype(np.int32)


def main(ref_root):
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh"), ref_root])
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import fchl19_repr as fr

    rng = np.random.default_rng(20261207)
    out = {}
    cases = [(1, 6.0), (2, 6.0), (5, 5.0), (9, 6.0), (12, 6.0), (7, 20.0)]
    for c, (n, box) in enumerate(cases):
        R, Z = molecule(rng, n, box, [1, 6, 7, 8, 16], p=[0.4, 0.3, 0.1, 0.1, 0.1])
        X, G = fr.generate_fchl_acsf_and_gradients(R, Z)
        out[f"d{c}_R"], out[f"d{c}_Z"], out[f"d{c}_X"], out[f"d{c}_G"] = R, Z, X, G
        assert np.allclose(fr.generate_fchl_acsf(R, Z), X, rtol=1e-12, atol=1e-14)
    for c, n in enumerate([4, 8, 11]):
        R, Z = molecule(rng, n, 5.0, NONDEFAULT["elements"])
        X, G = fr.generate_fchl_acsf_and_gradients(R, Z, **NONDEFAULT)
        out[f"n{c}_R"], out[f"n{c}_Z"], out[f"n{c}_X"], out[f"n{c}_G"] = R, Z, X, G
    R, Z = molecule(rng, 8, 6.0, [1, 6, 7, 8])
    out["f_R"], out["f_Z"] = R, Z
    out["f_X"] = fr.generate_fchl_acsf(R, Z, elements=[1, 6, 7, 8], nFourier=2)
    out["nondefault"] = np.array(repr(NONDEFAULT))
    np.savez_compressed(os.path.join(HERE, "golden_repr.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_repr.npz"))


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _refroot import reference_root
    main(reference_root(sys.argv[1:]))
