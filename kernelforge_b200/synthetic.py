"""Seeded synthetic molecules, Morse labels and FCHL19 descriptors.

The reference's benchmark datasets (rMD17, QM7b) are downloaded at run time
and are not available offline; this module generates stand-in data with the
same shapes and value distributions:

* molecules with ``n ~ U{nmin..nmax}`` atoms, elements H/C/N/O drawn with
  p = (0.5, 0.3, 0.1, 0.1), positions uniform in a 6 A box with a 0.9 A
  minimum pair distance (rejection sampling, atom by atom);
* labels from a pairwise Morse potential E = sum_{i<j} D (1 - exp(-a (r - r0)))^2
  (D=1, a=1.5, r0=1.2) and analytic forces F = -dE/dR;
* FCHL19 atomic descriptors with the reference's default hyper-parameters
  (elements [1,6,7,8,16], nRs2=24, nRs3=20, nFourier=1 -> 720 dims), restated
  from the published FCHL19 definition as implemented in the reference's
  generate_fchl_acsf (src/fchl19_repr.cpp:89-300, defaults in
  src/fchl19_repr_bindings.cpp:226-240), evaluated with torch in float64; the
  Jacobians dX/dR come from torch autograd.

Padded layouts follow the reference's models/representations.py:126-145:
X (nm, ma, rep), dX (nm, ma, rep, 3*ma), Q (nm, ma) int32, N (nm,) int32.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

ELEMENTS = (1, 6, 7, 8, 16)
P_ELEMENTS = {1: 0.5, 6: 0.3, 7: 0.1, 8: 0.1}


@dataclass
class Molecules:
    Z: list          # list of int arrays (n,)
    R: list          # list of float64 arrays (n, 3)
    E: np.ndarray    # (nm,) Morse energies
    F: list          # list of (n, 3) Morse forces

    @property
    def nm(self) -> int:
        return len(self.Z)


def make_molecules(nmol: int, nmin: int, nmax: int, seed: int, box: float = 6.0,
                   dmin: float = 0.9) -> Molecules:
    """Random molecules (see module docstring); deterministic for a given seed."""
    rng = np.random.default_rng(seed)
    elems = np.array(list(P_ELEMENTS.keys()))
    probs = np.array(list(P_ELEMENTS.values()))
    Zs, Rs = [], []
    for _ in range(nmol):
        n = int(rng.integers(nmin, nmax + 1))
        z = rng.choice(elems, size=n, p=probs).astype(np.int32)
        pos = np.zeros((n, 3))
        k = 0
        while k < n:
            p = rng.uniform(0.0, box, size=3)
            if k == 0 or np.min(np.linalg.norm(pos[:k] - p, axis=1)) >= dmin:
                pos[k] = p
                k += 1
        Zs.append(z)
        Rs.append(pos)
    E = np.zeros(nmol)
    Fs = []
    for m in range(nmol):
        e, f = morse(Rs[m])
        E[m] = e
        Fs.append(f)
    return Molecules(Zs, Rs, E, Fs)


def morse(R: np.ndarray, D: float = 1.0, a: float = 1.5, r0: float = 1.2):
    """Pairwise Morse energy and forces (F = -dE/dR)."""
    diff = R[:, None, :] - R[None, :, :]
    r = np.linalg.norm(diff, axis=-1)
    iu = np.triu_indices(len(R), 1)
    x = np.exp(-a * (r - r0))
    E = float(np.sum((D * (1.0 - x) ** 2)[iu]))
    with np.errstate(divide="ignore", invalid="ignore"):
        dEdr = 2.0 * D * a * (1.0 - x) * x
        g = np.where(r > 0, dEdr / r, 0.0)
    np.fill_diagonal(g, 0.0)
    grad = np.einsum("ij,ijk->ik", g, diff)
    return E, -grad


# ---------------------------------------------------------------------------
# FCHL19 descriptor (torch, float64)
# ---------------------------------------------------------------------------

def rep_size(nelem: int = 5, nRs2: int = 24, nRs3: int = 20, nFourier: int = 1) -> int:
    return nelem * nRs2 + nelem * (nelem + 1) // 2 * nRs3 * 2 * nFourier


def _fchl19_one(R: torch.Tensor, zidx: torch.Tensor, nelem: int = 5, nRs2: int = 24,
                nRs3: int = 20, eta2: float = 0.32, eta3: float = 2.7, zeta: float = math.pi,
                rcut: float = 8.0, acut: float = 8.0, two_body_decay: float = 1.8,
                three_body_decay: float = 0.57, three_body_weight: float = 13.4) -> torch.Tensor:
    """Descriptor of one molecule (n, rep) from coordinates R (n, 3) and element
    channel indices zidx (n,).  Differentiable in R."""
    n = R.shape[0]
    dt = R.dtype
    eps = 1e-12
    rep = rep_size(nelem, nRs2, nRs3)
    dev = R.device
    Rs2 = torch.arange(1, nRs2 + 1, dtype=dt, device=dev) * (rcut / nRs2)
    Rs3 = torch.arange(1, nRs3 + 1, dtype=dt, device=dev) * (acut / nRs3)
    diff = R[None, :, :] - R[:, None, :]                 # diff[i, j] = R_j - R_i
    eye = torch.eye(n, dtype=torch.bool, device=dev)
    r2 = (diff * diff).sum(-1)
    r = torch.sqrt(torch.where(eye, torch.ones_like(r2), r2))
    r = torch.where(eye, torch.zeros_like(r), r)

    # ---- two-body: log-normal radial basis on each neighbour's element channel
    rs = torch.where(eye, torch.ones_like(r), r)
    t = eta2 / torch.clamp(rs * rs, min=eps)
    log1pt = torch.log1p(t)
    sig = torch.sqrt(torch.clamp(log1pt, min=0.0))
    mu = torch.log(rs) - 0.5 * log1pt
    decay2 = 0.5 * (torch.cos(math.pi * rs / rcut) + 1.0)
    pref = decay2 / (sig * math.sqrt(2 * math.pi) * rs ** two_body_decay)
    dlog = torch.log(Rs2)[None, None, :] - mu[:, :, None]
    g = torch.exp(-0.5 * dlog * dlog / (sig * sig)[:, :, None]) / Rs2[None, None, :]
    val = pref[:, :, None] * g                           # (n, n, nRs2): centre i, neighbour j
    mask2 = (~eye) & (r <= rcut)
    val = val * mask2[:, :, None].to(dt)
    onehot = (zidx.long()[:, None] == torch.arange(nelem, device=dev)).to(dt)  # (n, nelem)
    two = torch.einsum("ijk,je->iek", val, onehot).reshape(n, nelem * nRs2)

    # ---- three-body: ATM-weighted angular/radial terms for neighbour pairs (j<k)
    decay3 = 0.5 * (torch.cos(math.pi * rs / acut) + 1.0)
    inv_r = torch.where(eye, torch.zeros_like(r), 1.0 / torch.clamp(rs, min=eps))
    e = diff * inv_r[:, :, None]                         # e[i, j] = (R_j - R_i)/r_ij
    cos_i = torch.einsum("ijx,ikx->ijk", e, e).clamp(-1.0, 1.0)      # angle at i
    cos_j = -torch.einsum("ijx,jkx->ijk", e, e)          # dot(-e_ij, e_jk)
    cos_k = torch.einsum("ikx,jkx->ijk", e, e)           # dot(e_ik, e_jk)
    rij = r[:, :, None].expand(n, n, n)
    rik = r[:, None, :].expand(n, n, n)
    rjk = r[None, :, :].expand(n, n, n)
    prod = torch.clamp(rik * rij * rjk, min=eps)
    # the three-body weight is normalised by sqrt(eta3/pi), as the reference's
    # binding does (src/fchl19_repr_bindings.cpp:83-84)
    w3 = math.sqrt(eta3 / math.pi) * three_body_weight
    ksi3 = (1.0 + 3.0 * cos_i * cos_j * cos_k) * (w3 / prod ** three_body_decay)
    sin_i = torch.sqrt(torch.clamp(1.0 - cos_i * cos_i, min=1e-30))
    w = 2.0 * math.exp(-0.5 * zeta * zeta)
    ang = torch.stack([w * cos_i, w * sin_i], dim=-1)    # (n, n, n, 2)
    rbar = 0.5 * (rij + rik)
    radial = torch.exp(-eta3 * (rbar[..., None] - Rs3) ** 2) * \
        (decay3[:, :, None] * decay3[:, None, :])[..., None]          # (n, n, n, nRs3)
    idx = torch.arange(n, device=dev)
    valid = (idx[None, :, None] < idx[None, None, :]) & (idx[:, None, None] != idx[None, :, None]) \
        & (idx[:, None, None] != idx[None, None, :])
    valid = valid & (r[:, :, None] <= acut) & (r[:, None, :] <= acut)
    coef = (ksi3 * valid.to(dt))[..., None, None] * radial[..., :, None] * ang[..., None, :]
    # element pair channel of (elem_j, elem_k)
    npair = nelem * (nelem + 1) // 2
    p = torch.minimum(zidx[:, None], zidx[None, :]).long()
    q = torch.maximum(zidx[:, None], zidx[None, :]).long()
    pair = -p * (p + 1) // 2 + q + nelem * p            # (n, n) over (j, k)
    pair_oh = (pair[..., None] == torch.arange(npair, device=dev)).to(dt)  # (n, n, npair)
    three = torch.einsum("ijkla,jkp->ipla", coef, pair_oh).reshape(n, npair * nRs3 * 2)
    out = torch.cat([two, three], dim=1)
    assert out.shape[1] == rep
    return out


def _zidx(z: np.ndarray, elements=ELEMENTS) -> torch.Tensor:
    lut = {e: i for i, e in enumerate(elements)}
    return torch.tensor([lut[int(v)] for v in z], dtype=torch.long)


def fchl19(mols: Molecules, gradients: bool = False, max_atoms: int | None = None,
           dtype=np.float64, elements=ELEMENTS, nRs2: int = 24, nRs3: int = 20):
    """Padded FCHL19 arrays: X (nm, ma, rep) [, dX (nm, ma, rep, 3*ma)], Q, N
    (rep = 720 for the default elements and basis sizes)."""
    nm = mols.nm
    ma = max_atoms or max(len(z) for z in mols.Z)
    nel = len(elements)
    rep = rep_size(nel, nRs2, nRs3)
    kw = dict(nelem=nel, nRs2=nRs2, nRs3=nRs3)
    X = np.zeros((nm, ma, rep), dtype=dtype)
    dX = np.zeros((nm, ma, rep, 3 * ma), dtype=dtype) if gradients else None
    Q = np.zeros((nm, ma), dtype=np.int32)
    N = np.zeros((nm,), dtype=np.int32)
    with torch.no_grad() if not gradients else torch.enable_grad():
        for m in range(nm):
            z = mols.Z[m]
            n = len(z)
            R = torch.tensor(mols.R[m], dtype=torch.float64)
            zi = _zidx(z, elements)
            if gradients:
                J = torch.func.jacfwd(lambda rr: _fchl19_one(rr, zi, **kw))(R)   # (n, rep, n, 3)
                rep_m = _fchl19_one(R, zi, **kw).detach().numpy()
                dX[m, :n, :, : 3 * n] = J.reshape(n, rep, 3 * n).numpy()
            else:
                rep_m = _fchl19_one(R, zi, **kw).numpy()
            X[m, :n] = rep_m
            Q[m, :n] = z
            N[m] = n
    return (X, dX, Q, N) if gradients else (X, Q, N)


def fchl19_batched(mols: Molecules, max_atoms: int | None = None, dtype=np.float32,
                   device: str = "cpu", chunk: int = 256):
    """Descriptors only (no Jacobians), vectorised over molecules of equal size;
    used for the large scalar-kernel workloads."""
    nm = mols.nm
    ma = max_atoms or max(len(z) for z in mols.Z)
    rep = rep_size()
    X = np.zeros((nm, ma, rep), dtype=dtype)
    Q = np.zeros((nm, ma), dtype=np.int32)
    N = np.zeros((nm,), dtype=np.int32)
    sizes = np.array([len(z) for z in mols.Z])
    f = torch.vmap(_fchl19_one)
    for n in np.unique(sizes):
        ids = np.nonzero(sizes == n)[0]
        for s in range(0, len(ids), chunk):
            sel = ids[s:s + chunk]
            R = torch.tensor(np.stack([mols.R[m] for m in sel]), dtype=torch.float64, device=device)
            zi = torch.stack([_zidx(mols.Z[m]) for m in sel]).to(device)
            with torch.no_grad():
                out = f(R, zi).cpu().numpy()
            X[sel, :n] = out.astype(dtype)
            for j, m in enumerate(sel):
                Q[m, :n] = mols.Z[m]
            N[sel] = n
    return X, Q, N


def fchl19_batched_grad(mols: Molecules, max_atoms: int | None = None, dtype=np.float32,
                        device: str = "cuda", chunk: int = 8):
    """Descriptors and Jacobians (X, dX, Q, N), vectorised over molecules of
    equal size with torch.func (vmap of jacfwd); used for the derivative-kernel
    workloads.  dX is (nm, ma, 720, 3*ma)."""
    nm = mols.nm
    ma = max_atoms or max(len(z) for z in mols.Z)
    rep = rep_size()
    X = np.zeros((nm, ma, rep), dtype=dtype)
    dX = np.zeros((nm, ma, rep, 3 * ma), dtype=dtype)
    Q = np.zeros((nm, ma), dtype=np.int32)
    N = np.zeros((nm,), dtype=np.int32)
    sizes = np.array([len(z) for z in mols.Z])
    f = torch.vmap(_fchl19_one)
    jf = torch.vmap(torch.func.jacfwd(_fchl19_one, argnums=0))
    for n in np.unique(sizes):
        ids = np.nonzero(sizes == n)[0]
        for s in range(0, len(ids), chunk):
            sel = ids[s:s + chunk]
            R = torch.tensor(np.stack([mols.R[m] for m in sel]), dtype=torch.float64,
                             device=device)
            zi = torch.stack([_zidx(mols.Z[m]) for m in sel]).to(device)
            with torch.no_grad():
                out = f(R, zi)
            J = jf(R, zi)                                   # (b, n, rep, n, 3)
            X[sel, :n] = out.cpu().numpy().astype(dtype)
            dX[sel, :n, :, : 3 * n] = J.reshape(len(sel), n, rep, 3 * n).detach().cpu().numpy() \
                .astype(dtype)
            for m in sel:
                Q[m, :n] = mols.Z[m]
            N[sel] = n
    return X, dX, Q, N
