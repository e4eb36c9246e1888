"""The FCHL19 descriptor restatement (kernelforge_b200.synthetic, torch FP64 with
autograd Jacobians) against the reference's own outputs (tests/golden/golden_repr.npz,
made by tests/golden/make_golden_repr.py), on the CPU."""
import ast
import os

import numpy as np
import pytest
import torch

from kernelforge_b200 import synthetic

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_repr.npz"))
NONDEFAULT = ast.literal_eval(str(G["nondefault"]))


def restated(R, Z, elements, **kw):
    zi = synthetic._zidx(Z, elements)
    Rt = torch.tensor(R, dtype=torch.float64)
    f = lambda r: synthetic._fchl19_one(r, zi, nelem=len(elements), **kw)
    X = f(Rt).numpy()
    J = torch.func.jacfwd(f)(Rt).numpy()      # (n, rep, n, 3)
    return X, J.reshape(J.shape[0], J.shape[1], -1)


def _kw(p):
    return {k: p[k] for k in ("nRs2", "nRs3", "eta2", "eta3", "zeta", "rcut", "acut",
                              "two_body_decay", "three_body_decay", "three_body_weight")}


@pytest.mark.parametrize("c", range(6))
def test_restatement_default(c):
    R, Z = G[f"d{c}_R"], G[f"d{c}_Z"]
    X, J = restated(R, Z, synthetic.ELEMENTS)
    np.testing.assert_allclose(X, G[f"d{c}_X"], rtol=1e-11, atol=1e-13)
    if len(Z) > 1:
        np.testing.assert_allclose(J, G[f"d{c}_G"], rtol=1e-8, atol=1e-10 * np.abs(J).max())


@pytest.mark.parametrize("c", range(3))
def test_restatement_nondefault(c):
    R, Z = G[f"n{c}_R"], G[f"n{c}_Z"]
    X, J = restated(R, Z, NONDEFAULT["elements"], **_kw(NONDEFAULT))
    np.testing.assert_allclose(X, G[f"n{c}_X"], rtol=1e-11, atol=1e-13)
    np.testing.assert_allclose(J, G[f"n{c}_G"], rtol=1e-8, atol=1e-10 * np.abs(J).max())


def test_golden_gradients_are_translation_invariant():
    """Every column block sums to zero over the atoms (the identity the GPU kernel
    uses for the centre atom's own columns)."""
    for c in range(1, 6):
        Gd = G[f"d{c}_G"]                       # (n, rep, 3n)
        n = Gd.shape[0]
        np.testing.assert_allclose(Gd.reshape(n, -1, n, 3).sum(axis=2), 0.0,
                                   atol=1e-9 * np.abs(Gd).max())
