"""The feature-map oracle (oracle/features.py) pinned on the CPU: the elemental
random Fourier features and their normal equations against the reference's own
kitchen_sinks module (golden_rff.npz, made by tests/golden/make_golden_rff.py),
and the cos-MLP pair-loss gradient against central finite differences."""
import numpy as np
import pytest

from conftest import load_golden
from oracle import features as of
from oracle import oracle as o


@pytest.mark.parametrize("case", ["f", "r"])
def test_rff_features_match_reference(case):
    g = load_golden("golden_rff.npz")
    Z = of.rff_features_elemental(g[case + "_X"], g[case + "_Q"], g[case + "_N"],
                                  g[case + "_W"], g[case + "_b"])
    np.testing.assert_allclose(Z, g[case + "_Z"], rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("case", ["f", "r"])
def test_rff_gramian_matches_reference_rfp(case):
    g = load_golden("golden_rff.npz")
    ztz, zty = of.rff_gramian(g[case + "_Z"], g[case + "_Y"])
    # the reference's CPU Gramian is RFP TRANSR='N', UPLO='U'
    np.testing.assert_allclose(o.full_to_rfp(ztz), g[case + "_ZtZ_rfp"], rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(zty, g[case + "_ZtY"], rtol=1e-11, atol=1e-11)


def test_rff_empty_molecule_is_zero():
    g = load_golden("golden_rff.npz")
    N = g["r_N"]
    Z = of.rff_features_elemental(g["r_X"], g["r_Q"], N, g["r_W"], g["r_b"])
    assert np.all(Z[N == 0] == 0.0)


def _small_net(rng, rep=12, H=16, D=24):
    W1 = rng.standard_normal((H, rep)) * 0.3
    b1 = rng.uniform(0, 2 * np.pi, H)
    W2 = rng.standard_normal((D, H)) * 0.5
    b2 = rng.uniform(0, 2 * np.pi, D)
    return [W1, b1, W2, b2]


def test_cosmlp_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    params = _small_net(rng)
    P, rep = 5, params[0].shape[1]
    xi = rng.standard_normal((P, rep))
    xj = rng.standard_normal((P, rep))
    t = rng.uniform(0, 1, P)
    _, grads = of.cosmlp_pair_loss_grad(xi, xj, t, *params)
    h = 1e-6
    for k, (p, gk) in enumerate(zip(params, grads)):
        flat = p.reshape(-1)
        for idx in rng.choice(flat.size, size=min(12, flat.size), replace=False):
            old = flat[idx]
            flat[idx] = old + h
            lp, _ = of.cosmlp_pair_loss_grad(xi, xj, t, *params)
            flat[idx] = old - h
            lm, _ = of.cosmlp_pair_loss_grad(xi, xj, t, *params)
            flat[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - gk.reshape(-1)[idx]) <= 1e-7 + 1e-6 * abs(fd), (k, idx)


def test_cosmlp_features_sum_per_molecule():
    rng = np.random.default_rng(3)
    params = [_small_net(rng) for _ in range(2)]
    nm, ma, rep = 4, 3, params[0][0].shape[1]
    X = rng.standard_normal((nm, ma, rep))
    Q = np.array([[0, 1, -1], [1, 1, 0], [-1, -1, -1], [0, 0, 0]], np.int32)
    N = np.array([2, 3, 0, 2], np.int32)
    Z = of.cosmlp_features_elemental(X, Q, N, params)
    want = np.zeros_like(Z)
    for m in range(nm):
        for j in range(N[m]):
            e = Q[m, j]
            phi, _ = of.cosmlp_forward(X[m, j][None], *params[e])
            want[m] += phi[0]
    np.testing.assert_allclose(Z, want, rtol=1e-13, atol=1e-13)
    assert np.all(Z[2] == 0)


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -2.5, 0.0], np.float32)
    got = of.to_bf16(x)
    np.testing.assert_array_equal(got, np.array([1.0, 1.0, 1.0 + 2.0 ** -6, -2.5, 0.0],
                                                np.float32))


@pytest.mark.parametrize("tag", ["f", "r"])
def test_oracle_rff_force_path_matches_reference(tag):
    """The force features and the energy+force normal equations of the oracle
    against the reference's kitchen_sinks (tests/golden/golden_rff_force.npz)."""
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_rff_force.npz"))
    a = {k[2:]: g[k] for k in g.files if k.startswith(tag + "_")}
    G = of.rff_gradient_elemental(a["X"], a["dX"], a["Q"], a["N"], a["W"], a["b"])
    np.testing.assert_allclose(G, a["G"].T, rtol=1e-11, atol=1e-12 * np.abs(G).max())
    Z = of.rff_features_elemental(a["X"], a["Q"], a["N"], a["W"], a["b"])
    A, rhs = of.rff_full_gramian(Z, G, a["Y"], a["F"])
    np.testing.assert_allclose(rhs, a["ZtY"], rtol=1e-11, atol=1e-12 * np.abs(rhs).max())
    np.testing.assert_allclose(o.full_to_rfp(A), a["ZtZ_rfp"], rtol=1e-11,
                               atol=1e-12 * np.abs(A).max())
