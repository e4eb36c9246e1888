"""CPU FP64 oracle of the per-molecule feature maps (numpy).

TEST INFRASTRUCTURE ONLY: imported by tests/ and the cpu_baseline leg of
bench.py, never by the kernelforge_b200 package.

* rff_features_elemental / rff_gramian: the reference's elemental random
  Fourier features, restated from src/rff_elemental.hpp:7-24 and the steps of
  src/rff_elemental.cpp:30-135 (gather the atoms of element e, Z_e = X_e W_e,
  cos(Z_e + b_e) sqrt(2/D), scatter-add per molecule) and the normal equations
  of src/rff_elemental.cpp:641-700 (Z^T Z, Z^T Y); the force features
  rff_gradient_elemental and the energy + force normal equations.  Pinned
  against the reference's own kitchen_sinks module (tests/golden/golden_rff.npz,
  golden_rff_force.npz).
* The learned cos-MLP map (no reference counterpart): forward pass, the pair
  loss and its analytic FP64 gradient, the per-molecule feature sums.  The
  gradient is pinned by central finite differences in the CPU tests.

Element indices in Q are 0-based with -1 for padding, as in the reference's
RFF functions (src/rff_elemental.hpp:14-15).
"""
from __future__ import annotations

import numpy as np


def rff_features_elemental(X, Q, N, W, b):
    """LZ[m] = sum over atoms j < N[m] with e = Q[m, j] >= 0 of
    sqrt(2/D) cos(X[m, j] @ W[e] + b[e])."""
    X = np.asarray(X, np.float64)
    W = np.asarray(W, np.float64)
    b = np.asarray(b, np.float64)
    nm, ma, _ = X.shape
    D = b.shape[1]
    norm = np.sqrt(2.0 / D)
    LZ = np.zeros((nm, D))
    for e in range(W.shape[0]):
        mols, atoms = [], []
        for m in range(nm):
            for j in range(min(max(int(N[m]), 0), ma)):
                if int(Q[m, j]) == e:
                    mols.append(m)
                    atoms.append(j)
        if not mols:
            continue
        Xe = X[mols, atoms]                       # (total_e, rep)
        Ze = np.cos(Xe @ W[e] + b[e]) * norm      # (total_e, D)
        np.add.at(LZ, np.asarray(mols), Ze)
    return LZ


def rff_gramian(Z, Y):
    """Dense Z^T Z and Z^T Y (the reference packs the first as RFP 'U')."""
    Z = np.asarray(Z, np.float64)
    return Z.T @ Z, Z.T @ np.asarray(Y, np.float64)


# ------------------------------------------------------------------ cos-MLP
def rff_gradient_elemental(X, dX, Q, N, W, b):
    """G (total_naq, D): row 3 off_m + 3 a + t (atom a of molecule m, axis t) is
    sqrt(2/D) sum_j sin(x_j W[e_j] + b[e_j]) * (W[e_j]^T dX[m, j, :, 3 a + t]),
    the force features with F = G w (src/rff_elemental.cpp:363-500, which stores
    the transpose (D, ngrads)).  dX is (nm, ma, rep, 3 ma)."""
    X = np.asarray(X, np.float64)
    dX = np.asarray(dX, np.float64)
    W = np.asarray(W, np.float64)
    b = np.asarray(b, np.float64)
    nm, ma, _ = X.shape
    D = b.shape[1]
    norm = np.sqrt(2.0 / D)
    n = np.clip(np.asarray(N), 0, ma)
    off = np.concatenate([[0], np.cumsum(3 * n)]).astype(int)
    G = np.zeros((off[-1], D))
    for m in range(nm):
        nc = 3 * n[m]
        for j in range(n[m]):
            e = int(Q[m, j])
            if e < 0:
                continue
            z = X[m, j] @ W[e] + b[e]
            G[off[m]:off[m] + nc] += norm * (dX[m, j, :, :nc].T @ W[e]) * np.sin(z)[None, :]
    return G


def rff_full_gramian(Z, G, Y, F):
    """Energy + force normal equations: [Z; G]^T [Z; G] and Z^T Y + G^T F
    (src/rff_elemental.cpp:799-935)."""
    A = np.concatenate([np.asarray(Z, np.float64), np.asarray(G, np.float64)])
    return A.T @ A, A.T @ np.concatenate([np.ravel(Y), np.ravel(F)])


def to_bf16(a):
    """Round to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def cosmlp_forward(x, W1, b1, W2, b2):
    """phi(x) = sqrt(2/D) cos(W2 cos(W1 x + b1) + b2) for the rows of x, with
    the intermediates (z1, h, z2)."""
    x = np.asarray(x, np.float64)
    z1 = x @ np.asarray(W1, np.float64).T + b1
    h = np.cos(z1)
    z2 = h @ np.asarray(W2, np.float64).T + b2
    s = np.sqrt(2.0 / z2.shape[1])
    return s * np.cos(z2), (z1, h, z2)


def cosmlp_pair_loss_grad(xi, xj, t, W1, b1, W2, b2):
    """loss = mean_p (phi(xi_p) . phi(xj_p) - t_p)^2 and its gradient with
    respect to (W1, b1, W2, b2), by the chain rule in FP64."""
    P = xi.shape[0]
    x = np.concatenate([np.asarray(xi, np.float64), np.asarray(xj, np.float64)])
    phi, (z1, h, z2) = cosmlp_forward(x, W1, b1, W2, b2)
    s = np.sqrt(2.0 / z2.shape[1])
    k = np.sum(phi[:P] * phi[P:], axis=1)
    r = k - np.asarray(t, np.float64)
    loss = np.mean(r * r)
    g = (2.0 / P) * r[:, None]
    dphi = np.concatenate([g * phi[P:], g * phi[:P]])
    dz2 = dphi * (-s * np.sin(z2))
    gW2 = dz2.T @ h
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ np.asarray(W2, np.float64)) * (-np.sin(z1))
    gW1 = dz1.T @ x
    gb1 = dz1.sum(axis=0)
    return loss, (gW1, gb1, gW2, gb2)


def cosmlp_features_elemental(X, Q, N, params):
    """Per-molecule sums of phi_e over the atoms of each element e;
    params[e] = (W1, b1, W2, b2)."""
    X = np.asarray(X, np.float64)
    nm, ma, _ = X.shape
    D = params[0][3].shape[0]
    LZ = np.zeros((nm, D))
    for e, (W1, b1, W2, b2) in enumerate(params):
        mols, atoms = [], []
        for m in range(nm):
            for j in range(min(max(int(N[m]), 0), ma)):
                if int(Q[m, j]) == e:
                    mols.append(m)
                    atoms.append(j)
        if not mols:
            continue
        phi, _ = cosmlp_forward(X[mols, atoms], W1, b1, W2, b2)
        np.add.at(LZ, np.asarray(mols), phi)
    return LZ


# ------------------------------------------ the GPU's arithmetic, restated
# The tensor-core path rounds to bfloat16 the GEMM operands: descriptors,
# weights, the hidden activations h and the back-propagated dZ2 / dZ1; it
# accumulates in FP32.  These variants apply the same roundings in FP64 so that
# a parity test can use a tolerance at the FP32-accumulation level.
def cosmlp_forward_bf16(x, W1, b1, W2, b2):
    xb = to_bf16(x).astype(np.float64)
    z1 = xb @ to_bf16(W1).astype(np.float64).T + b1
    h = to_bf16(np.cos(z1)).astype(np.float64)
    z2 = h @ to_bf16(W2).astype(np.float64).T + b2
    s = np.sqrt(2.0 / z2.shape[1])
    return s * np.cos(z2), (xb, z1, h, z2)


def cosmlp_pair_loss_grad_bf16(xi, xj, t, W1, b1, W2, b2):
    P = xi.shape[0]
    x = np.concatenate([np.asarray(xi, np.float64), np.asarray(xj, np.float64)])
    phi, (xb, z1, h, z2) = cosmlp_forward_bf16(x, W1, b1, W2, b2)
    D = z2.shape[1]
    s2 = 2.0 / D
    ci, cj = np.cos(z2[:P]), np.cos(z2[P:])
    r = s2 * np.sum(ci * cj, axis=1) - np.asarray(t, np.float64)
    loss = np.mean(r * r)
    g = ((2.0 / P) * r * s2)[:, None]
    dz2 = np.concatenate([-g * cj * np.sin(z2[:P]), -g * ci * np.sin(z2[P:])])
    dz2 = to_bf16(dz2).astype(np.float64)
    gW2 = dz2.T @ h
    gb2 = dz2.sum(axis=0)
    dz1 = to_bf16((dz2 @ to_bf16(W2).astype(np.float64)) * (-np.sin(z1))).astype(np.float64)
    gW1 = dz1.T @ xb
    gb1 = dz1.sum(axis=0)
    return loss, (gW1, gb1, gW2, gb2)


def cosmlp_features_elemental_bf16(X, Q, N, params):
    X = np.asarray(X, np.float64)
    nm, ma, _ = X.shape
    D = params[0][3].shape[0]
    LZ = np.zeros((nm, D))
    for e, (W1, b1, W2, b2) in enumerate(params):
        sel = [(m, j) for m in range(nm) for j in range(min(max(int(N[m]), 0), ma))
               if int(Q[m, j]) == e]
        if not sel:
            continue
        mols = np.array([m for m, _ in sel])
        phi, _ = cosmlp_forward_bf16(X[mols, [j for _, j in sel]], W1, b1, W2, b2)
        np.add.at(LZ, mols, phi)
    return LZ
