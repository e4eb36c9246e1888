"""CPU FP64 oracle of the contracted energy/force predictions (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/, never by the kernelforge_b200
package.

Restates kernel_gaussian_local_compute_alpha_desc / _jacobian_t_matvec /
_hessian_matvec / _full_matvec (src/local_kernels.cpp:2821-3425) from the
kernel definitions: with d = x_i - x_j, e = exp(-|d|^2 / 2 sigma^2),
w = e / sigma^2, w2 = e / sigma^4 over same-label pairs (i query, j training)
and the training atoms' Ad_j = J_j alpha_F,b (alpha_desc),

  E_a      = sum_{i in a, j} alpha_E[b] e + w (d . Ad_j)
  F_(a,c)  = sum_{i in a} J_i[:, c] . g_i,
  g_i      = sum_j w Ad_j + v_ij d,   v_ij = -w alpha_E[b] - w2 (d . Ad_j),

i.e. the rows of kernel_gaussian_full(query, training) times [alpha_E; alpha_F]
(the energy part without alpha_E is jacobian_t_matvec, the force part without
alpha_E is hessian_matvec).  Pinned against the reference's own outputs
(tests/golden/golden_matvec.npz, made by tests/golden/make_golden_matvec.py).
"""
from __future__ import annotations

import numpy as np


def _offsets(N, ma):
    n = np.clip(np.asarray(N), 0, ma)
    return np.concatenate([[0], np.cumsum(3 * n)]).astype(int), n


def alpha_desc(dX2, Q2, N2, alpha):
    dX2 = np.asarray(dX2, np.float64)
    nm2, ma2, rep, _ = dX2.shape
    off, n2 = _offsets(N2, ma2)
    out = np.zeros((nm2, ma2, rep))
    for b in range(nm2):
        nb = n2[b]
        if nb:
            out[b, :nb] = dX2[b, :nb, :, :3 * nb] @ np.asarray(alpha)[off[b]:off[b] + 3 * nb]
    return out


def matvec(X1, dX1, X2, ad, alpha_E, Q1, Q2, N1, N2, sigma):
    """(E, F): E (nm1,) if ad or alpha_E is given, F (naq1,) if dX1 is given."""
    X1 = np.asarray(X1, np.float64)
    X2 = np.asarray(X2, np.float64)
    nm1, ma1, rep = X1.shape
    nm2, ma2, _ = X2.shape
    off1, n1 = _offsets(N1, ma1)
    _, n2 = _offsets(N2, ma2)
    E = np.zeros(nm1)
    F = np.zeros(off1[-1]) if dX1 is not None else None
    is2, is4, c = 1.0 / sigma ** 2, 1.0 / sigma ** 4, -0.5 / sigma ** 2
    for a in range(nm1):
        for i in range(n1[a]):
            xi = X1[a, i]
            g = np.zeros(rep)
            for b in range(nm2):
                aE = 0.0 if alpha_E is None else float(alpha_E[b])
                for j in range(n2[b]):
                    if Q1[a, i] != Q2[b, j]:
                        continue
                    d = xi - X2[b, j]
                    e = np.exp(c * d @ d)
                    w, w2 = e * is2, e * is4
                    dad = 0.0 if ad is None else d @ ad[b, j]
                    E[a] += aE * e + w * dad
                    if ad is not None:
                        g += w * ad[b, j]
                    g += (-w * aE - w2 * dad) * d
            if F is not None:
                F[off1[a]:off1[a] + 3 * n1[a]] += g @ np.asarray(dX1, np.float64)[a, i, :, :3 * n1[a]]
    return E, F
