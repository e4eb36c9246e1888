"""Model-level drop-in for the reference's ``kernelforge.models`` FCHL19 kernel
ridge models, ``LocalKRRModel`` (python/kernelforge/models/krr.py:22-324) and
``CudaLocalKRRModel`` (models/cuda_local_krr.py:435-1180), with what a user sees
of their base class (models/base.py:56-430): ``fit`` / ``predict`` / ``score`` /
``save`` / ``load``, the training mode inferred from the labels given, the
per-element energy baseline, ``train_score_``, the ``.npz`` keys (saved models
move between the two libraries) and the same exception types and texts.

Design.  A fitted model keeps its descriptors, Jacobians and coefficients on the
GPU as torch tensors, so neither fit nor predict copies X or dX through the
host; ``save`` makes the only NumPy copies.  The pieces:

* ``_Molecules``        one call's geometry, padded for the GPU; element counts
                        and the flat force layout (3 per atom, molecule order);
* ``_Labels``           the labels a fit got: the KRR target vector built from
                        them, and training predictions split back into
                        energies / forces with the target's sign convention
                        (force rows of the energy+force target are -F);
* ``_ElementBaseline``  per-element energies, least squares on element counts
                        without intercept (models/base.py:401-418);
* ``_DeviceSet``        FCHL19 descriptors (+ Jacobians) resident on the GPU;
* ``_FP64Solver``       FP64 kernel matrices (RFP) and the FP64-class
                        tensor-core Cholesky solve with iterative refinement;
* ``_MixedSolver``      tensor-core kernel matrices (split fp16, FP32 RFP) and
                        the FP32-factor / FP64-refinement solve;
* ``_contract``         energies and forces at query molecules from the
                        contracted matvec (no query x training matrix).

``LocalKRRModel`` computes in FP64 (predictions agree with the reference's CPU
model to ~1e-10); ``CudaLocalKRRModel`` builds energy and energy+force kernels
on the tensor cores and solves them with the mixed solver.
"""
from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib
from ._device import require_cuda, stream_handle

__all__ = ["ModelScore", "BaseModel", "LocalKRRModel", "CudaLocalKRRModel", "compute_fchl19"]

_DEFAULT_ELEMENTS = [1, 6, 7, 8, 16]


# --------------------------------------------------------------------------
# scores
# --------------------------------------------------------------------------

@dataclass
class ModelScore:
    """MAE, Pearson r and the least-squares line pred = slope * ref + intercept."""

    mae: float
    pearson_r: float
    slope: float
    intercept: float

    def __str__(self) -> str:
        return (f"MAE={self.mae:.4f}  r={self.pearson_r:.6f}  "
                f"slope={self.slope:.6f}  intercept={self.intercept:.4f}")

    @classmethod
    def of(cls, ref, pred) -> "ModelScore":
        ref = np.asarray(ref, np.float64).ravel()
        pred = np.asarray(pred, np.float64).ravel()
        slope, intercept = np.polyfit(ref, pred, 1)
        return cls(mae=float(np.abs(pred - ref).mean()),
                   pearson_r=float(np.corrcoef(ref, pred)[0, 1]),
                   slope=float(slope), intercept=float(intercept))


# --------------------------------------------------------------------------
# geometry, labels and the energy baseline (host side, small)
# --------------------------------------------------------------------------

class _Molecules:
    """A batch of molecules padded to the largest one: ``coords`` (nm, ma, 3),
    ``z`` (nm, ma) int32 (0 in the padding) and ``n`` (nm,) atom counts."""

    def __init__(self, coords_list, z_list):
        if len(coords_list) != len(z_list):
            raise ValueError(f"coords_list and z_list must have the same length, "
                             f"got {len(coords_list)} and {len(z_list)}")
        zs = [np.asarray(z, dtype=np.int32).ravel() for z in z_list]
        self.n = np.array([len(z) for z in zs], dtype=np.int32)
        ma = int(self.n.max(initial=1))
        self.coords = np.zeros((len(zs), ma, 3))
        self.z = np.zeros((len(zs), ma), dtype=np.int32)
        for i, (r, z) in enumerate(zip(coords_list, zs)):
            self.coords[i, :len(z)] = np.asarray(r, dtype=np.float64).reshape(len(z), 3)
            self.z[i, :len(z)] = z

    def __len__(self) -> int:
        return len(self.n)

    @property
    def naq(self) -> int:
        return int(3 * self.n.sum())

    def element_counts(self, elements) -> np.ndarray:
        """(nm, len(elements)) numbers of atoms of each element (padding has z = 0,
        which no element equals)."""
        el = np.asarray(elements, dtype=np.int32)
        return (self.z[:, :, None] == el[None, None, :]).sum(axis=1).astype(np.float64)

    def flat_forces(self, forces) -> np.ndarray:
        """Forces in the kernels' row order (molecule, atom, xyz) as one vector,
        from an (nm, n_atoms, 3) / (nm, 3 n_atoms) array or a list of per-molecule
        arrays (models/base.py:363-381 accepts the same forms)."""
        if isinstance(forces, np.ndarray):
            f = np.asarray(forces, dtype=np.float64)
            if f.ndim not in (2, 3):
                raise ValueError(f"forces ndarray must be 2D or 3D, got {f.ndim}D")
            f = f.reshape(len(f), -1)
            if f.shape[1] != 3 * self.n.max(initial=0) or np.any(self.n != self.n[0]):
                return np.concatenate([f[i, :3 * k] for i, k in enumerate(self.n)])
            return f.ravel()
        return np.concatenate([np.asarray(fi, dtype=np.float64).ravel() for fi in forces])


class _Labels:
    """The labels a fit was given.  ``target()`` is the right-hand side of the
    KRR system; ``pairs(mode, y, y_fit, nm)`` splits a target and fitted values
    of it into (reference, prediction) pairs per label kind."""

    def __init__(self, mols: _Molecules, energies, forces):
        if energies is None and forces is None:
            raise ValueError("At least one of `energies` or `forces` must be provided.")
        if forces is None:
            self.mode = "energy_only"
        else:
            self.mode = "force_only" if energies is None else "energy_and_force"
        self.nm = len(mols)
        self.E = None if energies is None else np.asarray(energies, np.float64).ravel().copy()
        self.F = None if forces is None else mols.flat_forces(forces)

    def target(self) -> np.ndarray:
        if self.mode == "energy_only":
            return self.E
        if self.mode == "force_only":
            return self.F
        return np.concatenate([self.E, -self.F])

    @staticmethod
    def pairs(mode, y, y_fit, nm):
        if mode == "energy_only":
            return {"energy": (y, y_fit)}
        if mode == "force_only":
            return {"force": (y, y_fit)}
        return {"energy": (y[:nm], y_fit[:nm]), "force": (-y[nm:], -y_fit[nm:])}


class _ElementBaseline:
    """E_mol ~ sum over atoms of e[element]: fitted once on the training
    energies and subtracted from them (added back to predictions)."""

    def __init__(self, elements=None, energies=None):
        self.elements = np.asarray([] if elements is None else elements, dtype=np.int32)
        self.energies = np.asarray([] if energies is None else energies, dtype=np.float64)

    @classmethod
    def fit(cls, mols: _Molecules, E) -> "_ElementBaseline":
        present = np.unique(mols.z[mols.z > 0]) if mols.z.size else np.array([], np.int32)
        coef, *_ = np.linalg.lstsq(mols.element_counts(present), E, rcond=None)
        return cls(present, coef)

    def __call__(self, mols: _Molecules) -> np.ndarray:
        if self.elements.size == 0:
            return np.zeros(len(mols))
        return mols.element_counts(self.elements) @ self.energies


# --------------------------------------------------------------------------
# descriptors on the device
# --------------------------------------------------------------------------

class _DeviceSet:
    """FCHL19 descriptors X (nm, ma, rep) and Jacobians dX (nm, ma, rep, 3 ma)
    as CUDA tensors, with the nuclear charges Q (nm, ma) and atom counts N."""

    def __init__(self, X, dX, Q, N):
        self.X, self.dX = X, dX
        self.Q = np.ascontiguousarray(Q, dtype=np.int32)
        self.N = np.ascontiguousarray(N, dtype=np.int32)

    @classmethod
    def compute(cls, mols: _Molecules, elements, repr_params, dtype) -> "_DeviceSet":
        from . import fchl19_repr as fr
        require_cuda()
        X, dX = fr.generate_batched(mols.coords, mols.z, mols.n, elements=elements,
                                    gradients=True, dtype=dtype, **(repr_params or {}))
        return cls(X, dX, mols.z, mols.n)

    @classmethod
    def from_host(cls, X, dX, Q, N, dtype) -> "_DeviceSet":
        import torch
        tdt = torch.float64 if dtype == "float64" else torch.float32
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a)).to("cuda", tdt)  # noqa: E731
        return cls(dev(X), None if dX is None else dev(dX), Q, N)

    @property
    def f64(self) -> bool:
        import torch
        return self.X.dtype == torch.float64

    @property
    def naq(self) -> int:
        return int(3 * np.clip(self.N, 0, self.X.shape[1]).sum())

    def host(self, what):
        t = {"X": self.X, "dX": self.dX}[what]
        return None if t is None else t.cpu().numpy()


def compute_fchl19(coords_list, z_list, elements, with_gradients, repr_params, dtype="float64"):
    """(X, dX or None, Q, Q_elem, N) as NumPy arrays, like the reference's helper
    (models/representations.py:57-150), computed on the GPU; Q holds nuclear
    charges, Q_elem element indices into ``elements``."""
    mols = _Molecules(coords_list, z_list)
    ds = _DeviceSet.compute(mols, elements, repr_params, dtype)
    lut = {e: i for i, e in enumerate(elements)}
    q_elem = [np.array([lut[int(v)] for v in mols.z[m, :k]], dtype=np.int32)
              for m, k in enumerate(mols.n)]
    X = ds.host("X").astype(np.float64, copy=False)
    dX = ds.host("dX").astype(np.float64, copy=False) if with_gradients else None
    return X, dX, mols.z, q_elem, mols.n


# --------------------------------------------------------------------------
# kernel matrices, solves and the contracted prediction (device tensors)
# --------------------------------------------------------------------------

def _dt(ds: _DeviceSet) -> int:
    return _lib.KFB_F64 if ds.f64 else _lib.KFB_F32


def _alpha_desc(ds: _DeviceSet, alpha_F):
    """J^T alpha_F per training atom, (nm, ma, rep) float64 on the device."""
    import torch
    nm, ma, rep = ds.X.shape
    out = torch.empty((nm, ma, rep), dtype=torch.float64, device="cuda")
    af = alpha_F.reshape(-1).to(torch.float64).contiguous()
    _lib.check(_lib.lib().kfb_local_alpha_desc(
        ds.dX.data_ptr(), ds.Q.ctypes.data, ds.N.ctypes.data, nm, ma, rep, _dt(ds),
        af.data_ptr(), out.data_ptr(), stream_handle()))
    return out


def _contract(query: _DeviceSet, train: _DeviceSet, alpha_E, alpha_desc, sigma):
    """(E, Fr) = full(query, train) [alpha_E; alpha_F] with alpha_desc = J^T alpha_F,
    as float64 NumPy arrays, without forming the matrix."""
    import torch
    nm1, ma1, rep = query.X.shape
    nm2, ma2 = train.X.shape[:2]
    e = torch.empty(nm1, dtype=torch.float64, device="cuda")
    f = torch.empty(max(query.naq, 1), dtype=torch.float64, device="cuda")
    xt = train.X if train.X.dtype == query.X.dtype else train.X.to(query.X.dtype)
    _lib.check(_lib.lib().kfb_local_matvec(
        query.X.data_ptr(), query.dX.data_ptr(), xt.data_ptr(), alpha_desc.data_ptr(),
        alpha_E.data_ptr(), query.Q.ctypes.data, train.Q.ctypes.data, query.N.ctypes.data,
        train.N.ctypes.data, nm1, nm2, ma1, ma2, rep, float(sigma), _dt(query), e.data_ptr(),
        f.data_ptr(), stream_handle()))
    return e.cpu().numpy(), f[:query.naq].cpu().numpy()


class _FP64Solver:
    """FP64 kernel matrices in RFP and kfb_cho_solve_rfp on the device (the
    FP64-class tensor-core Cholesky plus two refinement steps against K)."""

    lambda_floor = False

    def __init__(self, sigma, l2):
        self.sigma, self.l2 = sigma, l2

    def matrix(self, ds: _DeviceSet, mode):
        import torch
        nm, ma, rep = ds.X.shape
        naq = ds.naq
        n = {"energy_only": nm, "force_only": naq, "energy_and_force": nm + naq}[mode]
        out = torch.empty((n * (n + 1) // 2,), dtype=torch.float64, device="cuda")
        lib, s, prec = _lib.lib(), stream_handle(), _lib.PREC["fp64"]
        if mode == "energy_only":
            st = lib.kfb_kernel_gaussian_symm(ds.X.data_ptr(), ds.Q.ctypes.data,
                                              ds.N.ctypes.data, nm, ma, rep, float(self.sigma),
                                              _dt(ds), prec, _lib.KFB_RFP_L, _lib.KFB_F64,
                                              out.data_ptr(), s)
        elif mode == "force_only":
            st = lib.kfb_kernel_gaussian_hessian_symm(ds.X.data_ptr(), ds.dX.data_ptr(),
                                                      ds.Q.ctypes.data, ds.N.ctypes.data, nm,
                                                      ma, rep, naq, float(self.sigma), _dt(ds),
                                                      prec, _lib.KFB_RFP_L, out.data_ptr(), s)
        else:
            st = lib.kfb_kernel_gaussian_full_symm(ds.X.data_ptr(), ds.dX.data_ptr(),
                                                   ds.Q.ctypes.data, ds.N.ctypes.data, nm, ma,
                                                   rep, naq, float(self.sigma), _dt(ds), prec,
                                                   _lib.KFB_RFP_L, out.data_ptr(), s)
        _lib.check(st)
        return out, n

    def solve(self, ds: _DeviceSet, mode, y):
        import torch
        K, n = self.matrix(ds, mode)
        yd = torch.as_tensor(y, dtype=torch.float64).to("cuda")
        alpha = torch.empty(n, dtype=torch.float64, device="cuda")
        info = ctypes.c_int(0)
        st = _lib.lib().kfb_cho_solve_rfp(K.data_ptr(), yd.data_ptr(), n, float(self.l2),
                                          _lib.KFB_RFP_L, alpha.data_ptr(), ctypes.byref(info),
                                          stream_handle())
        if st == _lib.KFB_ERR_NOT_PD:
            raise RuntimeError(f"DPFTRF failed, info={info.value}")
        _lib.check(st)
        # (K + l2 I) alpha = y, so the fitted values K alpha are y - l2 alpha
        return alpha, np.asarray(y, np.float64) - self.l2 * alpha.cpu().numpy(), self.l2, {}


def _truncated_eigensolve(A, b, rtol, atol, max_rank):
    """x = sum over kept eigenpairs of v (v . b) / lambda, keeping eigenvalues
    above max(atol, rtol lambda_max) (the largest max_rank of them, if set)."""
    import torch
    lam, V = torch.linalg.eigh(A)
    lam_max = float(lam[-1])
    tau = max(float(atol), float(rtol) * lam_max)
    idx = torch.nonzero(lam > tau).flatten()
    if max_rank is not None:
        idx = idx[max(0, idx.numel() - int(max_rank)):]
    if idx.numel() == 0:
        raise RuntimeError(f"Truncated eigensolve kept no eigenpairs. lambda_max={lam_max:.3e}, "
                           f"tau={tau:.3e}.")
    Vk = V[:, idx]
    x = Vk @ ((Vk.T @ b) / lam[idx])
    return x, {"rank": int(idx.numel()), "n": int(A.shape[0]), "lam_min": float(lam[0]),
               "lam_max": lam_max, "tau": tau, "dropped": int(A.shape[0] - idx.numel())}


def _jacobi_cg(A, b, rtol, atol, max_iter, restart=50):
    """Conjugate gradients with the inverse diagonal as preconditioner; every
    `restart` steps the residual is recomputed from x and the direction reset."""
    import torch
    d = A.diagonal()
    minv = torch.where(d > torch.finfo(A.dtype).eps, 1.0 / d, torch.ones_like(d))
    x = torch.zeros_like(b)
    r = b.clone()
    tol = max(float(atol), float(rtol) * float(torch.linalg.vector_norm(b)))
    limit = 10 * A.shape[0] if max_iter is None else int(max_iter)
    res = float(torch.linalg.vector_norm(r))
    it = 0
    z = minv * r
    p = z.clone()
    rz = torch.dot(r, z)
    while res > tol:
        if it >= limit:
            raise RuntimeError(f"CG did not converge within the iteration budget. "
                               f"residual={res:.3e}, tol={tol:.3e}, max_iter={limit}.")
        it += 1
        Ap = A @ p
        curv = float(torch.dot(p, Ap))
        if not (curv > 0.0) or not np.isfinite(curv):
            raise RuntimeError(f"CG breakdown: non-positive search-direction curvature at "
                               f"iteration {it} (p^T K p={curv:.3e}).")
        step = rz / curv
        x = x + step * p
        r = b - A @ x if it % restart == 0 else r - step * Ap
        res = float(torch.linalg.vector_norm(r))
        z = minv * r
        rz_new = torch.dot(r, z)
        p = z.clone() if it % restart == 0 else z + (rz_new / rz) * p
        rz = rz_new
    return x, {"iterations": it, "max_iter": limit, "residual_norm": res, "tol": tol,
               "n": int(A.shape[0]), "restart_period": restart}


class _MixedSolver(_FP64Solver):
    """Energy and energy+force kernel matrices on the tensor cores (split fp16,
    FP32 RFP).  ``method``:
      "cholesky"  the mixed solve (FP32-class factor, FP64 refinement; lambda
                  raised, and reported, when the FP32-stored matrix is
                  indefinite at l2);
      "eigh"      a truncated eigensolve of K + l2 I (models/cuda_local_krr.py:176-211);
      "cg"        Jacobi-preconditioned conjugate gradients (:214-290);
    the last two in FP64 on the dense matrix, with ``scaling`` "diagonal_scale"
    solving D (K + l2 I) D z = D y, alpha = D z, D = diag(K + l2 I)^(-1/2)
    (:293-315), or "none".  Force-only matrices stay on the FP64 path."""

    def __init__(self, sigma, l2, method="cholesky", scaling="diagonal_scale",
                 spectral=(3e-6, 0.0, None), cg=(2e-2, 0.0, None)):
        super().__init__(sigma, l2)
        if method not in ("cholesky", "eigh", "cg"):
            raise ValueError(f"Unsupported solver '{method}'. Expected 'cholesky', 'eigh', "
                             f"or 'cg'.")
        if scaling not in ("none", "diagonal_scale"):
            raise ValueError(f"Unsupported preprocessing '{scaling}'. Expected 'none' or "
                             f"'diagonal_scale'.")
        self.method, self.scaling, self.spectral, self.cg = method, scaling, spectral, cg

    def solve(self, ds: _DeviceSet, mode, y):
        import torch

        from . import cuda_global_kernels as cgk
        from . import cuda_local_kernels as clk
        if mode == "force_only":
            f64 = _DeviceSet(ds.X.double(), ds.dX.double(), ds.Q, ds.N)
            return _FP64Solver.solve(self, f64, mode, y)
        if mode == "energy_only":
            K = clk.kernel_gaussian_symm_rfp(ds.X, ds.Q, ds.N, self.sigma)
        else:
            K = clk.kernel_gaussian_full_symm_rfp(ds.X, ds.dX, ds.Q, ds.N, self.sigma)
        yd = torch.as_tensor(y, dtype=torch.float64).to("cuda")
        if self.method == "cholesky":
            alpha, info = cgk.krr_solve_mixed(K, yd, l2=self.l2, uplo="L", lambda_floor=True)
            lam = float(info.get("lambda_eff", self.l2))
            return alpha, np.asarray(y, np.float64) - lam * alpha.cpu().numpy(), lam, info
        n = yd.numel()
        dense = torch.empty((n, n), dtype=torch.float32, device="cuda")
        _lib.check(_lib.lib().kfb_rfp_to_full(K.data_ptr(), n, _lib.KFB_RFP_L, _lib.KFB_F32,
                                              dense.data_ptr(), stream_handle()))
        del K
        Kd = dense.double()
        del dense
        A = Kd.clone()
        A.diagonal().add_(float(self.l2))
        dsc = None
        b = yd
        if self.scaling == "diagonal_scale":
            dsc = torch.rsqrt(torch.clamp(A.diagonal(), min=torch.finfo(A.dtype).eps))
            A.mul_(dsc[:, None]).mul_(dsc[None, :])
            b = dsc * yd
        if self.method == "eigh":
            z, info = _truncated_eigensolve(A, b, *self.spectral)
        else:
            z, info = _jacobi_cg(A, b, *self.cg)
        del A
        alpha = z if dsc is None else dsc * z
        info = dict(info, solver=self.method, preprocessing=self.scaling)
        return alpha, (Kd @ alpha).cpu().numpy(), float(self.l2), info


# --------------------------------------------------------------------------
# the models
# --------------------------------------------------------------------------

class BaseModel:
    """fit / predict / score / save / load of the FCHL19 KRR models.  A subclass
    provides ``_solver()`` (kernel matrices and solve), ``_dtype`` (descriptor
    precision on the device) and its ``.npz`` layout (``_to_npz`` / ``_from_npz``)."""

    _dtype = "float64"

    # ---- public API -------------------------------------------------------
    def fit(self, coords_list, z_list, energies=None, forces=None):
        mols = _Molecules(coords_list, z_list)
        labels = _Labels(mols, energies, forces)
        self.training_mode_ = labels.mode
        if labels.E is not None:
            base = _ElementBaseline.fit(mols, labels.E)
            labels.E -= base(mols)
        else:
            base = _ElementBaseline()
        self.baseline_elements_, self.element_energies_ = base.elements, base.energies
        self._train = _DeviceSet.compute(mols, self.elements, self.repr_params, self._dtype)
        self._n_train = len(mols)
        y = labels.target()
        alpha, y_fit, l2_eff, info = self._solver().solve(self._train, labels.mode, y)
        self._set_coefficients(alpha, y, y_fit, l2_eff, info)
        self.train_score_ = {k: ModelScore.of(ref, pred) for k, (ref, pred) in
                             _Labels.pairs(self.training_mode_, y, y_fit,
                                           self._n_train).items()}
        self.is_fitted_ = True
        return self

    def predict(self, coords_list, z_list, compute_energy=True):
        """(energies (nm,), forces (3 sum n,)) with physical forces F = -dE/dR."""
        if not getattr(self, "is_fitted_", False):
            raise RuntimeError(f"{type(self).__name__} is not fitted yet. Call fit() first.")
        mols = _Molecules(coords_list, z_list)
        query = _DeviceSet.compute(mols, self.elements, self.repr_params, self._dtype)
        E, F = self._forward(query)
        if compute_energy:
            E = E + _ElementBaseline(self.baseline_elements_, self.element_energies_)(mols)
        return E, F

    def score(self, coords_list, z_list, energies=None, forces=None):
        if energies is None and forces is None:
            raise ValueError("At least one of `energies` or `forces` must be provided to "
                             "score().")
        if forces is not None and self.training_mode_ == "energy_only":
            raise ValueError("Cannot score forces: model was trained in energy_only mode "
                             "and does not predict forces.")
        E, F = self.predict(coords_list, z_list)
        out = {}
        if energies is not None:
            out["energy"] = ModelScore.of(energies, E)
        if forces is not None:
            out["force"] = ModelScore.of(_Molecules(coords_list, z_list).flat_forces(forces), F)
        return out

    def save(self, path) -> None:
        if not getattr(self, "is_fitted_", False):
            raise RuntimeError(f"{type(self).__name__} is not fitted yet. Call fit() first.")
        path = Path(path)
        np.savez(path if path.suffix == ".npz" else path.with_suffix(".npz"), **self._to_npz())

    @classmethod
    def load(cls, path):
        with np.load(Path(path), allow_pickle=True) as data:
            model = cls.__new__(cls)
            model._from_npz({k: data[k] for k in data.files})
        model.is_fitted_ = True
        return model

    # ---- shared internals ---------------------------------------------------
    def _set_coefficients(self, alpha, y, y_fit, l2_eff, info):
        """Keep the coefficients (device FP64) and J^T alpha_F of the force rows."""
        self._alpha = alpha
        self._y_train = np.asarray(y, np.float64)
        self._y_fit = np.asarray(y_fit, np.float64)
        self._l2_eff = l2_eff
        self.solve_info_ = info
        nm = self._n_train
        mode = self.training_mode_
        self._adesc = (_alpha_desc(self._train, alpha[nm:] if mode == "energy_and_force"
                                   else alpha) if mode != "energy_only" else None)

    def _alpha_host(self) -> np.ndarray:
        return self._alpha.cpu().numpy()

    def _forward(self, query: _DeviceSet):
        """Energies and physical forces at the query molecules: the contracted
        product with [alpha_E; alpha_F] of the full kernel, whose energy and
        force rows carry the sign conventions of the three training targets."""
        import torch
        nm, mode = self._n_train, self.training_mode_
        zeros_desc = lambda: torch.zeros(self._train.X.shape, dtype=torch.float64,  # noqa: E731
                                         device="cuda")
        if mode == "energy_only":
            E, Fr = _contract(query, self._train, self._alpha, zeros_desc(), self.sigma)
            return E, -Fr
        if mode == "force_only":
            aE = torch.zeros(nm, dtype=torch.float64, device="cuda")
            E, Fr = _contract(query, self._train, aE, self._adesc, self.sigma)
            return -E, Fr
        E, Fr = _contract(query, self._train, self._alpha[:nm].contiguous(), self._adesc,
                          self.sigma)
        return E, -Fr


class LocalKRRModel(BaseModel):
    """FCHL19 local KRR in FP64 on the GPU: energy_only, force_only or
    energy_and_force training (inferred from the labels), RFP kernel matrices
    and the Cholesky solve; predictions by the contracted matvecs."""

    def __init__(self, sigma=2.0, l2=1e-9, elements=None, repr_params=None):
        self.sigma = sigma
        self.l2 = l2
        self.elements = sorted(elements) if elements is not None else list(_DEFAULT_ELEMENTS)
        self.repr_params = repr_params if repr_params is not None else {}
        self.is_fitted_ = False

    def _solver(self):
        return _FP64Solver(self.sigma, self.l2)

    def _to_npz(self):
        out = {"model_class": "LocalKRRModel", "training_mode": self.training_mode_,
               "sigma": self.sigma, "l2": self.l2,
               "elements": np.array(self.elements, dtype=np.int32),
               "repr_params": json.dumps(self.repr_params),
               "baseline_elements": self.baseline_elements_,
               "element_energies": self.element_energies_, "alpha": self._alpha_host(),
               "y_train": self._y_train, "X_tr": self._train.host("X"),
               "Q_tr": self._train.Q, "N_tr": self._train.N}
        if self._train.dX is not None:
            out["dX_tr"] = self._train.host("dX")
        if self._adesc is not None:
            out["alpha_desc"] = self._adesc.cpu().numpy()
        return out

    def _from_npz(self, d):
        import torch
        self.sigma, self.l2 = float(d["sigma"]), float(d["l2"])
        self.elements = [int(e) for e in d["elements"]]
        self.repr_params = json.loads(str(d["repr_params"]))
        self.training_mode_ = str(d["training_mode"])
        self.baseline_elements_ = d["baseline_elements"].astype(np.int32)
        self.element_energies_ = d["element_energies"].astype(np.float64)
        self._train = _DeviceSet.from_host(d["X_tr"], d.get("dX_tr"), d["Q_tr"], d["N_tr"],
                                           "float64")
        self._n_train = len(self._train.N)
        self._alpha = torch.as_tensor(d["alpha"], dtype=torch.float64).to("cuda")
        self._y_train = d.get("y_train", np.zeros(0))
        self._y_fit = self._y_train - self.l2 * d["alpha"] if self._y_train.size else self._y_train
        self._l2_eff = self.l2
        ad = d.get("alpha_desc")
        self._adesc = None if ad is None else torch.as_tensor(ad, dtype=torch.float64).to("cuda")
        if self._adesc is None and self.training_mode_ != "energy_only":
            nm = self._n_train
            aF = self._alpha[nm:] if self.training_mode_ == "energy_and_force" else self._alpha
            self._adesc = _alpha_desc(self._train, aF)


class CudaLocalKRRModel(BaseModel):
    """FCHL19 local KRR with the kernel matrix on the tensor cores (split fp16,
    FP32 RFP); descriptors float32 on the device.  ``solver``: "eigh" (the
    reference's default: truncated eigensolve), "cg" (Jacobi-preconditioned
    CG) or "cholesky" (the FP32-factor / FP64-refinement solve, the fast one),
    with ``preprocessing`` "diagonal_scale" or "none"; unknown names raise
    ValueError when fit runs, as in the reference.  force_only training runs
    the FP64 path.  Energy-only models predict zero forces, as the reference's
    CUDA model does."""

    _dtype = "float32"

    def __init__(self, sigma=2.0, l2=1e-4, elements=None, repr_params=None, solver="eigh",
                 preprocessing="diagonal_scale", spectral_rtol=3e-6, spectral_atol=0.0,
                 spectral_max_rank=None, cg_rtol=2e-2, cg_atol=0.0, cg_max_iter=None):
        self.sigma, self.l2 = sigma, l2
        self.elements = sorted(elements) if elements is not None else list(_DEFAULT_ELEMENTS)
        self.repr_params = repr_params if repr_params is not None else {}
        self.solver, self.preprocessing = solver, preprocessing
        self.spectral_rtol, self.spectral_atol = spectral_rtol, spectral_atol
        self.spectral_max_rank = spectral_max_rank
        self.cg_rtol, self.cg_atol, self.cg_max_iter = cg_rtol, cg_atol, cg_max_iter
        self.is_fitted_ = False

    def _solver(self):
        return _MixedSolver(self.sigma, self.l2, self.solver, self.preprocessing,
                            (self.spectral_rtol, self.spectral_atol, self.spectral_max_rank),
                            (self.cg_rtol, self.cg_atol, self.cg_max_iter))

    def _forward(self, query):
        E, F = super()._forward(query)
        if self.training_mode_ == "energy_only":
            F = np.zeros_like(F)
        return E, F

    # the reference's file stores -1 for "no limit"
    _OPTIONAL_INTS = ("spectral_max_rank", "cg_max_iter")

    def _to_npz(self):
        nm = self._n_train
        alpha = self._alpha_host()
        aE = alpha[:nm] if self.training_mode_ != "force_only" else np.zeros(nm)
        adesc = (np.zeros(self._train.X.shape, np.float32) if self._adesc is None
                 else self._adesc.cpu().numpy())
        out = {"model_class": "CudaLocalKRRModel", "training_mode": self.training_mode_,
               "sigma": self.sigma, "l2": self.l2, "solver": self.solver,
               "preprocessing": self.preprocessing, "spectral_rtol": self.spectral_rtol,
               "spectral_atol": self.spectral_atol, "cg_rtol": self.cg_rtol,
               "cg_atol": self.cg_atol, "elements": np.array(self.elements, dtype=np.int32),
               "repr_params": json.dumps(self.repr_params), "n_train": nm,
               "max_atoms": int(self._train.X.shape[1]), "rep_size": int(self._train.X.shape[2]),
               "naq_train": self._train.naq, "baseline_elements": self.baseline_elements_,
               "element_energies": self.element_energies_, "alpha": alpha,
               "y_train": self._y_train, "y_pred_train": self._y_fit,
               "X_train": self._train.host("X").astype(np.float32),
               "dX_train": self._train.host("dX").astype(np.float32),
               "Q_train": self._train.Q, "N_train": self._train.N,
               "alpha_E": aE.astype(np.float32), "alpha_desc_F": adesc.astype(np.float32)}
        for k in self._OPTIONAL_INTS:
            v = getattr(self, k)
            out[k] = -1 if v is None else v
        return out

    def _from_npz(self, d):
        import torch
        self.sigma, self.l2 = float(d["sigma"]), float(d["l2"])
        self.solver = str(d.get("solver", "eigh"))
        self.preprocessing = str(d.get("preprocessing", "diagonal_scale"))
        self.spectral_rtol = float(d.get("spectral_rtol", 3e-6))
        self.spectral_atol = float(d.get("spectral_atol", 0.0))
        self.cg_rtol, self.cg_atol = float(d.get("cg_rtol", 2e-2)), float(d.get("cg_atol", 0.0))
        for k in self._OPTIONAL_INTS:
            v = int(d.get(k, -1))
            setattr(self, k, None if v < 0 else v)
        self.elements = [int(e) for e in d["elements"]]
        self.repr_params = json.loads(str(d["repr_params"]))
        self.training_mode_ = str(d["training_mode"])
        self.baseline_elements_ = d["baseline_elements"].astype(np.int32)
        self.element_energies_ = d["element_energies"].astype(np.float64)
        self._train = _DeviceSet.from_host(d["X_train"], d["dX_train"], d["Q_train"],
                                           d["N_train"], "float32")
        self._n_train = int(d["n_train"])
        self._alpha = torch.as_tensor(d["alpha"], dtype=torch.float64).to("cuda")
        self._y_train = d.get("y_train", np.zeros(0)).astype(np.float64)
        self._y_fit = d.get("y_pred_train", self._y_train - self.l2 * d["alpha"])
        self._l2_eff = self.l2
        # J^T alpha_F in FP64 from the stored Jacobians and the FP64 coefficients
        # (the file's alpha_desc_F is a float32 copy)
        nm = self._n_train
        self._adesc = None
        if self.training_mode_ == "energy_and_force":
            self._adesc = _alpha_desc(self._train, self._alpha[nm:])
        elif self.training_mode_ == "force_only":
            self._adesc = _alpha_desc(self._train, self._alpha)
