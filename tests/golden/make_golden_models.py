"""Golden fixtures of the model-level API (LocalKRRModel fit / predict / save,
python/kernelforge/models/krr.py, base.py, representations.py), from the
reference itself.

The reference's model modules are imported from the reference checkout over
its own CPU FP64 extension modules built by oracle/build_ref.sh (the models
package's __init__, which needs the reference's CUDA extensions, is bypassed).
Seeded synthetic molecules (4-6 atoms, H/C/N/O, Morse labels) and a reduced
descriptor (nRs2=8, nRs3=6) keep the fixture small.  Stores, per training mode,
the test predictions and training scores, and the energy+force model as the
reference saved it (tests/golden/ref_local_krr_ef.npz, re-compressed).

Usage:  python tests/golden/make_golden_models.py REFERENCE_ROOT   (or KERNELFORGE_REFERENCE_ROOT set)
"""
import os
import subprocess
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

REPR = dict(nRs2=8, nRs3=6)
ELEMENTS = [1, 6, 7, 8]


def reference_models(ref_root):
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    import fchl19_repr
    import kernelmath
    import local_kernels
    kf = types.ModuleType("kernelforge")
    kf.__path__ = []
    kf.fchl19_repr, kf.kernelmath, kf.local_kernels = fchl19_repr, kernelmath, local_kernels
    kf.fchl18_repr = types.ModuleType("kernelforge.fchl18_repr")
    models = types.ModuleType("kernelforge.models")
    models.__path__ = [os.path.join(ref_root, "python", "kernelforge", "models")]
    sys.modules.update({"kernelforge": kf, "kernelforge.fchl19_repr": fchl19_repr,
                        "kernelforge.kernelmath": kernelmath,
                        "kernelforge.local_kernels": local_kernels,
                        "kernelforge.fchl18_repr": kf.fchl18_repr,
                        "kernelforge.models": models})
    from kernelforge.models import krr
    return krr


def main(ref_root):
    subprocess.check_call([os.path.join(ROOT, "oracle", "build_ref.sh"), ref_root])
    krr = reference_models(ref_root)
    from kernelforge_b200 import synthetic
    mols = synthetic.make_molecules(22, 4, 6, seed=31)
    R, Z = [np.asarray(r) for r in mols.R], [np.asarray(z, np.int32) for z in mols.Z]
    E, F = np.asarray(mols.E), [np.asarray(f) for f in mols.F]
    tr, te = slice(0, 16), slice(16, 22)
    N = np.array([len(z) for z in Z], np.int32)
    ma = int(N.max())
    Rp, Zp, Fp_ = np.zeros((len(Z), ma, 3)), np.zeros((len(Z), ma), np.int32), \
        np.zeros((len(Z), ma, 3))
    for m in range(len(Z)):
        Rp[m, :N[m]], Zp[m, :N[m]], Fp_[m, :N[m]] = R[m], Z[m], np.reshape(F[m], (-1, 3))
    out = {"R": Rp, "Z": Zp, "N": N, "E": E, "F": Fp_}
    for mode, kw in (("e", dict(energies=E[tr])), ("f", dict(forces=F[tr])),
                     ("ef", dict(energies=E[tr], forces=F[tr]))):
        m = krr.LocalKRRModel(sigma=2.5, l2=1e-8, elements=ELEMENTS, repr_params=REPR)
        m.fit(R[tr], Z[tr], **kw)
        Ep, Fp = m.predict(R[te], Z[te])
        out[f"{mode}_E"], out[f"{mode}_F"] = Ep, np.asarray(Fp)
        for k, s in m.train_score_.items():
            out[f"{mode}_train_{k}_mae"] = s.mae
        if mode == "ef":
            with tempfile.TemporaryDirectory() as d:
                m.save(os.path.join(d, "m.npz"))
                saved = dict(np.load(os.path.join(d, "m.npz"), allow_pickle=True))
            np.savez_compressed(os.path.join(HERE, "ref_local_krr_ef.npz"), **saved)
    np.savez_compressed(os.path.join(HERE, "golden_models.npz"), **out)
    print("wrote golden_models.npz and ref_local_krr_ef.npz")


if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    from _refroot import reference_root
    main(reference_root(sys.argv[1:]))
