"""The contracted-prediction oracle against the reference's own outputs
(tests/golden/golden_matvec.npz) and against the uncontracted kernel."""
import os

import numpy as np
import pytest

from oracle import matvec as om

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_matvec.npz"))


def _case(tag):
    return {k[len(tag) + 1:]: G[k] for k in G.files if k.startswith(tag + "_")}


@pytest.mark.parametrize("tag", ["r", "f"])
def test_oracle_alpha_desc(tag):
    c = _case(tag)
    ad = om.alpha_desc(c["dX2"], c["Q2"], c["N2"], c["alpha_F"])
    np.testing.assert_allclose(ad, c["alpha_desc"], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("tag", ["r", "f"])
def test_oracle_matvecs(tag):
    c = _case(tag)
    args = (c["Q1"], c["Q2"], c["N1"], c["N2"], float(c["sigma"]))
    E, _ = om.matvec(c["X1"], None, c["X2"], c["alpha_desc"], None, *args)
    np.testing.assert_allclose(E, c["jacobian_t_matvec"], rtol=1e-12, atol=1e-13)
    _, F = om.matvec(c["X1"], c["dX1"], c["X2"], c["alpha_desc"], None, *args)
    np.testing.assert_allclose(F, c["hessian_matvec"], rtol=1e-12, atol=1e-13)
    E, F = om.matvec(c["X1"], c["dX1"], c["X2"], c["alpha_desc"], c["alpha_E"], *args)
    np.testing.assert_allclose(E, c["full_matvec_E"], rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(F, c["full_matvec_F"], rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("tag", ["r", "f"])
def test_golden_matvec_equals_full_kernel_product(tag):
    """The reference's contracted outputs are rows of its full E+F kernel times
    [alpha_E; alpha_F] (the identity the GPU path is built on)."""
    c = _case(tag)
    K = c["kernel_gaussian_full"]
    nm1 = c["N1"].shape[0]
    v = np.concatenate([c["alpha_E"], c["alpha_F"]])
    np.testing.assert_allclose(K[:nm1] @ v, c["full_matvec_E"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(K[nm1:] @ v, c["full_matvec_F"], rtol=1e-10, atol=1e-12)
