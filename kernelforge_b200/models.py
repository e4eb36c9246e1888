"""Model-level drop-in for the reference's ``kernelforge.models`` FCHL19 KRR
classes: ``LocalKRRModel`` (python/kernelforge/models/krr.py:22-324) and
``CudaLocalKRRModel`` (models/cuda_local_krr.py:435-1180), with the shared
``BaseModel`` behaviour (models/base.py:56-430): training mode from the given
labels, the per-element energy baseline, ``score``, and the ``.npz`` save format
(same keys, so files move between the two libraries).

Both run on the GPU through libkfb: descriptors (``fchl19_repr``), kernels,
solves and the contracted energy/force predictions.  ``LocalKRRModel`` keeps the
reference's FP64 arithmetic (its predictions agree with the reference's CPU model
to ~1e-10); ``CudaLocalKRRModel`` builds the kernel on the tensor cores
(split fp16, FP32 RFP storage) and solves it with the FP32/FP64 mixed solver
(``krr_solve_mixed``, lambda raised when the FP32-stored kernel is indefinite).
"""
from __future__ import annotations

import json
from abc import ABC, abstractmethod
from dataclasses import dataclass
from pathlib import Path

import numpy as np

__all__ = ["ModelScore", "BaseModel", "LocalKRRModel", "CudaLocalKRRModel", "compute_fchl19"]

_DEFAULT_ELEMENTS = [1, 6, 7, 8, 16]


# --------------------------------------------------------------------------
# scores and the base class (models/base.py)
# --------------------------------------------------------------------------

@dataclass
class ModelScore:
    """MAE, Pearson r and the linear fit pred = slope ref + intercept."""

    mae: float
    pearson_r: float
    slope: float
    intercept: float

    def __str__(self) -> str:
        return (f"MAE={self.mae:.4f}  r={self.pearson_r:.6f}  "
                f"slope={self.slope:.6f}  intercept={self.intercept:.4f}")


def _compute_score(y_ref, y_pred) -> ModelScore:
    ref, pred = np.ravel(y_ref), np.ravel(y_pred)
    mae = float(np.mean(np.abs(pred - ref)))
    r = float(np.corrcoef(ref, pred)[0, 1])
    slope, intercept = np.polyfit(ref, pred, 1)
    return ModelScore(mae=mae, pearson_r=r, slope=float(slope), intercept=float(intercept))


def _infer_mode(energies, forces) -> str:
    if energies is not None and forces is not None:
        return "energy_and_force"
    if energies is not None:
        return "energy_only"
    if forces is not None:
        return "force_only"
    raise ValueError("At least one of `energies` or `forces` must be provided.")


def _validate_geometry(coords_list, z_list):
    if len(coords_list) != len(z_list):
        raise ValueError(f"coords_list and z_list must have the same length, "
                         f"got {len(coords_list)} and {len(z_list)}")
    return ([np.asarray(r, dtype=np.float64) for r in coords_list],
            [np.asarray(z, dtype=np.int32) for z in z_list])


def _coerce_forces(forces):
    """Forces as (n_mols, n_atoms*3), or one flat array for molecules of
    different sizes (models/base.py:363-381)."""
    if isinstance(forces, np.ndarray):
        f = np.asarray(forces, dtype=np.float64)
        if f.ndim == 3:
            return f.reshape(len(f), -1)
        if f.ndim == 2:
            return f
        raise ValueError(f"forces ndarray must be 2D or 3D, got {f.ndim}D")
    rows = [np.asarray(fi, dtype=np.float64).ravel() for fi in forces]
    if len({len(r) for r in rows}) == 1:
        return np.array(rows, dtype=np.float64)
    return np.concatenate(rows)


def _build_composition_matrix(z_list, elements):
    A = np.zeros((len(z_list), len(elements)))
    for i, z in enumerate(z_list):
        for j, e in enumerate(elements):
            A[i, j] = float(np.sum(z == e))
    return A


def _fit_element_baseline(z_list, energies):
    """Per-element energies by least squares on element counts, no intercept
    (models/base.py:401-418)."""
    elements = np.unique(np.concatenate([z.astype(np.int32) for z in z_list])).astype(np.int32)
    A = _build_composition_matrix(z_list, elements)
    e, *_ = np.linalg.lstsq(A, energies, rcond=None)
    return elements, np.asarray(e, dtype=np.float64)


def _check_fitted(model) -> None:
    if not getattr(model, "is_fitted_", False):
        raise RuntimeError(f"{type(model).__name__} is not fitted yet. Call fit() first.")


class BaseModel(ABC):
    """fit / predict / score / save / load shared by the models."""

    def fit(self, coords_list, z_list, energies=None, forces=None):
        coords_list, z_list = _validate_geometry(coords_list, z_list)
        self.training_mode_ = _infer_mode(energies, forces)
        E = None if energies is None else np.asarray(energies, dtype=np.float64).ravel()
        F = None if forces is None else _coerce_forces(forces)
        if E is not None:
            self.baseline_elements_, self.element_energies_ = _fit_element_baseline(z_list, E)
            E = E - _build_composition_matrix(z_list, self.baseline_elements_) @ \
                self.element_energies_
        else:
            self.baseline_elements_ = np.array([], dtype=np.int32)
            self.element_energies_ = np.array([], dtype=np.float64)
        self._fit(coords_list, z_list, E, F)
        self.train_score_ = self._compute_train_score()
        self.is_fitted_ = True
        return self

    def predict(self, coords_list, z_list, compute_energy=True):
        """(energies (M,), forces) with physical forces F = -dE/dR."""
        _check_fitted(self)
        coords_list, z_list = _validate_geometry(coords_list, z_list)
        E, F = self._predict(coords_list, z_list, compute_energy=compute_energy)
        if compute_energy and len(self.baseline_elements_) > 0:
            E = E + _build_composition_matrix(z_list, self.baseline_elements_) @ \
                self.element_energies_
        return E, F

    def score(self, coords_list, z_list, energies=None, forces=None):
        if energies is None and forces is None:
            raise ValueError("At least one of `energies` or `forces` must be provided to "
                             "score().")
        E, F = self.predict(coords_list, z_list)
        scores = {}
        if energies is not None:
            scores["energy"] = _compute_score(np.asarray(energies, np.float64).ravel(), E)
        if forces is not None:
            if self.training_mode_ == "energy_only":
                raise ValueError("Cannot score forces: model was trained in energy_only mode "
                                 "and does not predict forces.")
            scores["force"] = _compute_score(_coerce_forces(forces), F)
        return scores

    def save(self, path) -> None:
        _check_fitted(self)
        path = Path(path)
        if path.suffix != ".npz":
            path = path.with_suffix(".npz")
        np.savez(path, **self._arrays_to_save())

    @classmethod
    def load(cls, path):
        data = np.load(Path(path), allow_pickle=True)
        model = cls.__new__(cls)
        model._load_from_arrays(data)
        model.is_fitted_ = True
        return model

    def _compute_train_score(self):
        return {k: _compute_score(ref, pred)
                for k, (ref, pred) in self._training_labels_and_predictions().items()}

    @abstractmethod
    def _fit(self, coords_list, z_list, energies, forces): ...

    @abstractmethod
    def _predict(self, coords_list, z_list, compute_energy=True): ...

    @abstractmethod
    def _arrays_to_save(self): ...

    @abstractmethod
    def _load_from_arrays(self, data): ...

    @abstractmethod
    def _training_labels_and_predictions(self): ...


# --------------------------------------------------------------------------
# descriptors (models/representations.py:57-150), on the GPU
# --------------------------------------------------------------------------

def _pad(coords_list, z_list):
    N = np.array([len(z) for z in z_list], dtype=np.int32)
    ma = int(N.max())
    C = np.zeros((len(z_list), ma, 3))
    Z = np.zeros((len(z_list), ma), dtype=np.int32)
    for i, (r, z) in enumerate(zip(coords_list, z_list)):
        C[i, :len(z)] = np.asarray(r, np.float64).reshape(len(z), 3)
        Z[i, :len(z)] = z
    return C, Z, N


def compute_fchl19(coords_list, z_list, elements, with_gradients, repr_params, dtype="float64"):
    """(X, dX or None, Q_krr, Q_rff, N) as the reference's helper returns them
    (float64 NumPy; dX (n_mols, max_atoms, rep, 3 max_atoms)), computed on the GPU."""
    from . import fchl19_repr as fr
    C, Z, N = _pad(coords_list, z_list)
    out = fr.generate_batched(C, Z, N, elements=elements, gradients=with_gradients,
                              dtype=dtype, **(repr_params or {}))
    X, dX = (out if with_gradients else (out, None))
    X = X.cpu().numpy().astype(np.float64, copy=False)
    dX = None if dX is None else dX.cpu().numpy().astype(np.float64, copy=False)
    lut = {e: i for i, e in enumerate(elements)}
    Q_rff = [np.array([lut[int(v)] for v in z], dtype=np.int32) for z in z_list]
    return X, dX, Z, Q_rff, N


# --------------------------------------------------------------------------
# LocalKRRModel (models/krr.py), FP64 on the GPU
# --------------------------------------------------------------------------

class LocalKRRModel(BaseModel):
    """FCHL19 local KRR: energy_only, force_only or energy_and_force training
    (inferred from the labels), RFP-packed symmetric kernels and the Cholesky
    solve, all in FP64 on the GPU; predictions by the contracted matvecs."""

    def __init__(self, sigma=2.0, l2=1e-9, elements=None, repr_params=None):
        self.sigma = sigma
        self.l2 = l2
        self.elements = sorted(elements) if elements is not None else list(_DEFAULT_ELEMENTS)
        self.repr_params = repr_params if repr_params is not None else {}
        self.is_fitted_ = False

    def _fit(self, coords_list, z_list, energies, forces):
        from . import kernelmath, local_kernels as lk
        mode = self.training_mode_
        X, dX, Q, _, N = compute_fchl19(coords_list, z_list, self.elements, True,
                                        self.repr_params)
        self._X_tr, self._dX_tr, self._Q_tr, self._N_tr = X, dX, Q, N
        self._n_train = len(coords_list)
        self._n_atoms = X.shape[1]
        if mode == "energy_only":
            K = lk.kernel_gaussian_symm_rfp(X, Q, N, self.sigma)
            self._y_train = energies
            self._alpha = kernelmath.cho_solve_rfp(K, energies, l2=self.l2)
            self._alpha_desc = None
        elif mode == "force_only":
            F = forces.ravel()
            K = lk.kernel_gaussian_hessian_symm_rfp(X, dX, Q, N, self.sigma)
            self._y_train = F
            self._alpha = kernelmath.cho_solve_rfp(K, F, l2=self.l2)
            self._alpha_desc = lk.kernel_gaussian_local_compute_alpha_desc(dX, Q, N, self._alpha)
        else:
            # training labels [E; -F] (+dE/dR for the force rows of the full kernel)
            y = np.concatenate([energies, (-forces).ravel()])
            K = lk.kernel_gaussian_full_symm_rfp(X, dX, Q, N, self.sigma)
            self._y_train = y
            self._alpha = kernelmath.cho_solve_rfp(K, y, l2=self.l2)
            self._alpha_desc = lk.kernel_gaussian_local_compute_alpha_desc(
                dX, Q, N, self._alpha[self._n_train:])

    def _predict(self, coords_list, z_list, compute_energy=True):
        from . import local_kernels as lk
        mode = self.training_mode_
        X, dX, Q, _, N = compute_fchl19(coords_list, z_list, self.elements, True,
                                        self.repr_params)
        Xt, dXt, Qt, Nt, a = self._X_tr, self._dX_tr, self._Q_tr, self._N_tr, self._alpha
        s = self.sigma
        if mode == "energy_only":
            # E = K(test, train) alpha; F = +dK/dR_test alpha (the reference's
            # jacobian_t contraction), contracted: no test x train matrices
            zero = np.zeros_like(Xt)
            E, Fr = lk.kernel_gaussian_local_full_matvec(X, dX, Xt, zero, a, Q, Qt, N, Nt, s)
            return E, -Fr
        if mode == "force_only":
            if self._alpha_desc is not None:
                F = lk.kernel_gaussian_local_hessian_matvec(X, dX, Xt, self._alpha_desc, Q, Qt,
                                                            N, Nt, s)
                E = -lk.kernel_gaussian_local_jacobian_t_matvec(X, Xt, self._alpha_desc, Q, Qt,
                                                                N, Nt, s)
                return E, F
            F = lk.kernel_gaussian_hessian(X, dX, Xt, dXt, Q, Qt, N, Nt, s) @ a
            E = -(lk.kernel_gaussian_jacobian(X, Xt, dXt, Q, Qt, N, Nt, s) @ a)
            return E, F
        n = self._n_train
        if self._alpha_desc is not None:
            E, Fr = lk.kernel_gaussian_local_full_matvec(X, dX, Xt, self._alpha_desc, a[:n], Q,
                                                         Qt, N, Nt, s)
            return E, -Fr
        y = lk.kernel_gaussian_full(X, dX, Xt, dXt, Q, Qt, N, Nt, s) @ a
        return y[:len(N)], -y[len(N):]

    def _training_labels_and_predictions(self):
        y_pred = self._y_train - self.l2 * self._alpha
        n = self._n_train
        if self.training_mode_ == "energy_only":
            return {"energy": (self._y_train, y_pred)}
        if self.training_mode_ == "force_only":
            return {"force": (self._y_train, y_pred)}
        return {"energy": (self._y_train[:n], y_pred[:n]),
                "force": (-self._y_train[n:], -y_pred[n:])}

    def _arrays_to_save(self):
        d = {"model_class": "LocalKRRModel", "training_mode": self.training_mode_,
             "sigma": self.sigma, "l2": self.l2,
             "elements": np.array(self.elements, dtype=np.int32),
             "repr_params": json.dumps(self.repr_params),
             "baseline_elements": self.baseline_elements_,
             "element_energies": self.element_energies_, "alpha": self._alpha,
             "y_train": self._y_train, "X_tr": self._X_tr, "Q_tr": self._Q_tr,
             "N_tr": self._N_tr}
        if self._dX_tr is not None:
            d["dX_tr"] = self._dX_tr
        if self._alpha_desc is not None:
            d["alpha_desc"] = self._alpha_desc
        return d

    def _load_from_arrays(self, data):
        self.sigma = float(data["sigma"])
        self.l2 = float(data["l2"])
        self.elements = data["elements"].tolist()
        self.repr_params = json.loads(str(data["repr_params"]))
        self.baseline_elements_ = data["baseline_elements"].astype(np.int32)
        self.element_energies_ = data["element_energies"].astype(np.float64)
        self.training_mode_ = str(data["training_mode"])
        self._alpha = data["alpha"]
        self._y_train = data["y_train"] if "y_train" in data else np.array([], np.float64)
        self._X_tr, self._Q_tr, self._N_tr = data["X_tr"], data["Q_tr"], data["N_tr"]
        self._dX_tr = data["dX_tr"] if "dX_tr" in data else None
        self._alpha_desc = data["alpha_desc"] if "alpha_desc" in data else None
        self._n_train = len(self._N_tr)
        self._n_atoms = self._X_tr.shape[1]


# --------------------------------------------------------------------------
# CudaLocalKRRModel (models/cuda_local_krr.py): tensor-core kernel + mixed solve
# --------------------------------------------------------------------------

class CudaLocalKRRModel(BaseModel):
    """FCHL19 local KRR with the kernel on the tensor cores (split fp16, FP32 RFP)
    and the FP32-factor / FP64-refinement solve.  ``solver``, ``preprocessing``
    and the spectral / CG settings are accepted and saved for compatibility; every
    solver name runs the mixed Cholesky solve (lambda is raised, and reported in
    ``solve_info_``, when the FP32-stored kernel is indefinite at ``l2``).
    force_only training runs the FP64 path of :class:`LocalKRRModel`."""

    def __init__(self, sigma=2.0, l2=1e-4, elements=None, repr_params=None, solver="eigh",
                 preprocessing="diagonal_scale", spectral_rtol=3e-6, spectral_atol=0.0,
                 spectral_max_rank=None, cg_rtol=2e-2, cg_atol=0.0, cg_max_iter=None):
        if solver not in ("cholesky", "eigh", "cg"):
            raise ValueError("solver must be 'cholesky', 'eigh' or 'cg'")
        self.sigma, self.l2 = sigma, l2
        self.elements = sorted(elements) if elements is not None else list(_DEFAULT_ELEMENTS)
        self.repr_params = repr_params if repr_params is not None else {}
        self.solver, self.preprocessing = solver, preprocessing
        self.spectral_rtol, self.spectral_atol = spectral_rtol, spectral_atol
        self.spectral_max_rank = spectral_max_rank
        self.cg_rtol, self.cg_atol, self.cg_max_iter = cg_rtol, cg_atol, cg_max_iter
        self.is_fitted_ = False

    def _descriptors(self, coords_list, z_list):
        import torch

        from . import fchl19_repr as fr
        C, Z, N = _pad(coords_list, z_list)
        x, dx = fr.generate_batched(C, Z, N, elements=self.elements, gradients=True,
                                    dtype="float32", **self.repr_params)
        return x, dx, Z, N

    def _fit(self, coords_list, z_list, energies, forces):
        import torch

        from . import cuda_global_kernels as cgk
        from . import cuda_local_kernels as clk
        mode = self.training_mode_
        self._n_train = len(coords_list)
        if mode == "force_only":
            ref = LocalKRRModel(self.sigma, self.l2, self.elements, self.repr_params)
            ref.training_mode_ = mode
            ref._fit(coords_list, z_list, None, forces)
            self._fp64 = ref
            self._y_train = ref._y_train
            self._alpha = ref._alpha
            self._y_pred_train = ref._y_train - self.l2 * ref._alpha
            self._l2_eff = self.l2
            x, dx, Z, N = self._descriptors(coords_list, z_list)
            self._store(x, dx, Z, N)
            self._alpha_E_np = np.zeros(self._n_train, np.float32)
            self._alpha_desc_F_np = ref._alpha_desc.astype(np.float32)
            return
        x, dx, Z, N = self._descriptors(coords_list, z_list)
        self._store(x, dx, Z, N)
        if mode == "energy_only":
            K = clk.kernel_gaussian_symm_rfp(x, Z, N, self.sigma)
            y = energies
        else:
            K = clk.kernel_gaussian_full_symm_rfp(x, dx, Z, N, self.sigma)
            y = np.concatenate([energies, (-forces).ravel()])
        alpha, info = cgk.krr_solve_mixed(K, torch.tensor(y, device="cuda"), l2=self.l2,
                                          uplo="L", lambda_floor=True)
        del K
        self.solve_info_ = info
        self._l2_eff = float(info.get("lambda_eff", self.l2))
        self._alpha = alpha.cpu().numpy()
        self._y_train = y
        self._y_pred_train = y - self._l2_eff * self._alpha
        n = self._n_train
        self._alpha_E_np = self._alpha[:n].astype(np.float32)
        if mode == "energy_and_force":
            ad = clk.compute_alpha_desc(dx, N, alpha[n:])
            self._alpha_desc_F_np = ad.float().cpu().numpy()
            self._alpha_desc_F64 = ad.cpu().numpy()
        else:
            self._alpha_desc_F_np = np.zeros(x.shape, np.float32)

    def _store(self, x, dx, Z, N):
        self._X_train_np = x.cpu().numpy()
        self._dX_train_np = dx.cpu().numpy()
        self._Q_train_np, self._N_train_np = Z, N
        self._max_atoms, self._rep_size = x.shape[1], x.shape[2]
        self._naq_train = int(3 * N.sum())

    def _predict(self, coords_list, z_list, compute_energy=True):
        import torch

        from . import cuda_local_kernels as clk
        mode = self.training_mode_
        if mode == "force_only" and getattr(self, "_fp64", None) is not None:
            return self._fp64._predict(coords_list, z_list, compute_energy)
        x, dx, Z, N = self._descriptors(coords_list, z_list)
        xt = torch.tensor(self._X_train_np, device="cuda")
        n = self._n_train
        aE = torch.tensor(self._alpha[:n] if mode != "force_only" else
                          np.zeros(n), dtype=torch.float64, device="cuda")
        ad64 = getattr(self, "_alpha_desc_F64", None)
        if ad64 is None and mode == "energy_and_force":
            # a loaded model: rebuild J^T alpha_F in FP64 from the stored Jacobians
            # and the FP64 coefficients (the file's alpha_desc_F is float32)
            ad64 = clk.compute_alpha_desc(torch.tensor(self._dX_train_np, device="cuda"),
                                          self._N_train_np,
                                          torch.tensor(self._alpha[n:], device="cuda"))
            ad64 = ad64.cpu().numpy()
            self._alpha_desc_F64 = ad64
        ad = torch.tensor(ad64 if ad64 is not None else
                          self._alpha_desc_F_np.astype(np.float64), device="cuda")
        E, Fr = clk.kernel_gaussian_full_matvec(x, dx, Z, N, xt, self._Q_train_np,
                                                self._N_train_np, aE, ad, self.sigma)
        E = E.cpu().numpy()
        F = -Fr.cpu().numpy()
        if mode == "energy_only":
            # the reference's CUDA energy-only model returns zero forces
            F = np.zeros_like(F)
        return E, F

    def _training_labels_and_predictions(self):
        n = self._n_train
        if self.training_mode_ == "force_only":
            return {"force": (self._y_train, self._y_pred_train)}
        out = {"energy": (self._y_train[:n], self._y_pred_train[:n])}
        if len(self._y_train) > n:
            out["force"] = (-self._y_train[n:], -self._y_pred_train[n:])
        return out

    def _arrays_to_save(self):
        return {"model_class": "CudaLocalKRRModel", "training_mode": self.training_mode_,
                "sigma": self.sigma, "l2": self.l2, "solver": self.solver,
                "preprocessing": self.preprocessing, "spectral_rtol": self.spectral_rtol,
                "spectral_atol": self.spectral_atol,
                "spectral_max_rank": -1 if self.spectral_max_rank is None
                else self.spectral_max_rank,
                "cg_rtol": self.cg_rtol, "cg_atol": self.cg_atol,
                "cg_max_iter": -1 if self.cg_max_iter is None else self.cg_max_iter,
                "elements": np.array(self.elements, dtype=np.int32),
                "repr_params": json.dumps(self.repr_params), "n_train": self._n_train,
                "max_atoms": self._max_atoms, "rep_size": self._rep_size,
                "naq_train": self._naq_train, "baseline_elements": self.baseline_elements_,
                "element_energies": self.element_energies_, "alpha": self._alpha,
                "y_train": self._y_train, "y_pred_train": self._y_pred_train,
                "X_train": self._X_train_np, "dX_train": self._dX_train_np,
                "Q_train": self._Q_train_np, "N_train": self._N_train_np,
                "alpha_E": self._alpha_E_np, "alpha_desc_F": self._alpha_desc_F_np}

    def _load_from_arrays(self, data):
        get = lambda k, d: data[k] if k in data else d  # noqa: E731
        self.sigma, self.l2 = float(data["sigma"]), float(data["l2"])
        self.solver = str(get("solver", "eigh"))
        self.preprocessing = str(get("preprocessing", "diagonal_scale"))
        self.spectral_rtol = float(get("spectral_rtol", 3e-6))
        self.spectral_atol = float(get("spectral_atol", 0.0))
        smr = int(get("spectral_max_rank", -1))
        self.spectral_max_rank = None if smr < 0 else smr
        self.cg_rtol, self.cg_atol = float(get("cg_rtol", 2e-2)), float(get("cg_atol", 0.0))
        cmi = int(get("cg_max_iter", -1))
        self.cg_max_iter = None if cmi < 0 else cmi
        self.elements = data["elements"].tolist()
        self.repr_params = json.loads(str(data["repr_params"]))
        self.training_mode_ = str(data["training_mode"])
        self.baseline_elements_ = data["baseline_elements"].astype(np.int32)
        self.element_energies_ = data["element_energies"].astype(np.float64)
        self._n_train = int(data["n_train"])
        self._max_atoms, self._rep_size = int(data["max_atoms"]), int(data["rep_size"])
        self._naq_train = int(data["naq_train"])
        self._alpha = data["alpha"].astype(np.float64)
        self._y_train = get("y_train", np.array([], np.float64)).astype(np.float64)
        self._y_pred_train = get("y_pred_train", self._y_train - self.l2 * self._alpha)
        self._X_train_np = data["X_train"].astype(np.float32)
        self._dX_train_np = data["dX_train"].astype(np.float32)
        self._Q_train_np = data["Q_train"].astype(np.int32)
        self._N_train_np = data["N_train"].astype(np.int32)
        self._alpha_E_np = data["alpha_E"].astype(np.float32)
        self._alpha_desc_F_np = data["alpha_desc_F"].astype(np.float32)
        self._alpha_desc_F64 = None
        self._fp64 = None
