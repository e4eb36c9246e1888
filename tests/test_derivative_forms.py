"""The algebra behind the GPU derivative kernels, checked on the CPU against the oracle.

Jacobian: the GPU path (derivs.cu) contracts per-(outer molecule, inner atom) v rows with
the Jacobians instead of forming J_j^T (x_i - x_j) per atom pair (v_row_jacobian below).

Hessian: the tensor-core path never forms J_i^T (w I - w' d d^T) J_j per atom pair.  It uses
  * t'_ij = w'_ij (P_ij - PB_j), P_ij = (x_i - mu_l) . J_j and PB_j = (x_j - mu_l) . J_j
    (mu_l the set-1 mean of the label both atoms share, so the difference does not cancel);
  * w_ij = exp(c (n_i + n_j - 2 g_ij)) / sigma^2 with centred norms n and dot products g;
  * H_ab = sum_i J_i^T Y_i with Y_i = sum_j w_ij J_j, then minus the rank term
    sum_ij s_ij t'_ij^T, s_ij = PB1_i - Q_ij, PB1_i = (x_i - mu_l) . J_i,
    Q_ij = (x_j - mu_l) . J_i.
These tests restate those steps in numpy (FP64) on small ragged sets and compare them with
the oracle's Jacobian and Hessian (src/local_kernels.cpp, kernel_gaussian_jacobian and
kernel_gaussian_hessian), so a change of a decomposition that breaks its identity fails here
without a GPU."""
import numpy as np
import pytest

from conftest import make_set
from oracle import oracle as o


def gemm_form_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, sigma):
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    c2, is2 = -1.0 / (2 * sigma * sigma), 1.0 / (sigma * sigma)
    is4 = is2 * is2
    labels = sorted({int(q) for a in range(nm1) for q in Q1[a, :N1[a]]})
    mu = {l: np.mean([X1[a, i] for a in range(nm1) for i in range(N1[a]) if Q1[a, i] == l],
                     axis=0) for l in labels}
    off1 = np.concatenate([[0], np.cumsum(3 * N1)])
    off2 = np.concatenate([[0], np.cumsum(3 * N2)])
    H = np.zeros((off1[-1], off2[-1]))
    for a in range(nm1):
        na = N1[a]
        for b in range(nm2):
            nb = N2[b]
            Hab = np.zeros((3 * na, 3 * nb))
            for i in range(na):
                l = int(Q1[a, i])
                Ji = dX1[a, i][:, :3 * na]            # rep x 3 n_a
                xi = X1[a, i] - mu[l]
                pb1 = xi @ Ji                         # PB1_i
                Y = np.zeros((rep, 3 * nb))
                for j in range(nb):
                    if int(Q2[b, j]) != l:
                        continue
                    Jj = dX2[b, j][:, :3 * nb]        # rep x 3 n_b
                    xj = X2[b, j] - mu[l]
                    g = xi @ xj
                    e = np.exp(c2 * max(xi @ xi + xj @ xj - 2 * g, 0.0))
                    Y += e * is2 * Jj
                    t = e * is4 * (xi @ Jj - xj @ Jj)  # t'_ij = w' (P - PB)
                    s = pb1 - xj @ Ji                 # s_ij = PB1 - Q
                    Hab -= np.outer(s, t)
                Hab += Ji.T @ Y
            H[off1[a]:off1[a + 1], off2[b]:off2[b + 1]] = Hab
    return H


@pytest.mark.parametrize("seed", [0, 1])
def test_gemm_form_matches_oracle(seed):
    rep = 12
    X1, dX1, Q1, N1 = make_set(4, 5, rep, 3, 60 + seed)
    X2, dX2, Q2, N2 = make_set(3, 5, rep, 3, 70 + seed)
    X1 *= 0.4
    X2 *= 0.4
    Q2[1, :2] = 9   # a set-2 label set 1 lacks: no partners
    s = 2.0
    ref = o.kernel_gaussian_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s)
    got = gemm_form_hessian(X1, dX1, X2, dX2, Q1, Q2, N1, N2, s)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_gemm_form_symmetric_set():
    rep = 12
    X, dX, Q, N = make_set(4, 6, rep, 2, 80)
    X *= 0.4
    s = 1.5
    ref = o.kernel_gaussian_hessian(X, dX, X, dX, Q, Q, N, N, s)
    got = gemm_form_hessian(X, dX, X, dX, Q, Q, N, N, s)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    np.testing.assert_allclose(got, got.T, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def v_row_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, sigma):
    """The Jacobian as the GPU path forms it (derivs.cu): per outer molecule o and inner
    atom u the v row v_{o,u} = sum_{i in o, q_i = q_u} (e_iu / sigma^2) (x_i - x_u), with
    e from norms and dot products, then K[o, off_m + c] = sum_{u in m} v_{o,u} . J_u[:, c]."""
    nm1, _, rep = X1.shape
    nm2 = X2.shape[0]
    c2, is2 = -1.0 / (2 * sigma * sigma), 1.0 / (sigma * sigma)
    off2 = np.concatenate([[0], np.cumsum(3 * N2)])
    K = np.zeros((nm1, off2[-1]))
    for o_ in range(nm1):
        for m in range(nm2):
            for u in range(N2[m]):
                xu = X2[m, u]
                v = np.zeros(rep)
                for i in range(N1[o_]):
                    if Q1[o_, i] != Q2[m, u]:
                        continue
                    xi = X1[o_, i]
                    e = np.exp(c2 * max(xi @ xi + xu @ xu - 2 * (xi @ xu), 0.0))
                    v += e * is2 * (xi - xu)
                K[o_, off2[m]:off2[m + 1]] += v @ dX2[m, u][:, :3 * N2[m]]
    return K


@pytest.mark.parametrize("seed", [0, 1])
def test_v_row_jacobian_matches_oracle(seed):
    rep = 12
    X1, _, Q1, N1 = make_set(5, 5, rep, 3, 90 + seed)
    X2, dX2, Q2, N2 = make_set(4, 5, rep, 3, 95 + seed)
    X1 *= 0.4
    X2 *= 0.4
    Q1[1, :] = 1    # an outer molecule with one label
    s = 2.0
    ref = o.kernel_gaussian_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s)
    got = v_row_jacobian(X1, X2, dX2, Q1, Q2, N1, N2, s)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
