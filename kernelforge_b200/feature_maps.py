"""Learned cos-MLP feature map and the linear ridge model on per-molecule
features (no counterpart in the reference: it stands in for the random
Fourier features of ``kernelforge.cuda_rff_features``, models/rff.py).

Per element e the map is

    phi_e(x) = sqrt(2/D) cos(W2_e cos(W1_e x + b1_e) + b2_e)      (720 -> H -> D)

with BF16 weights and activations on the tensor cores and FP32 accumulation.
It is trained on same-element atom pairs so that phi(x_i) . phi(x_j) matches
the exact local Gaussian kernel value exp(-|x_i - x_j|^2 / (2 sigma^2)), the
pair term of the scalar kernel.  The initial weights make the untrained map a
random-Fourier-like map of the same sigma: with W1 small and b1 = pi/2 the
hidden layer is nearly linear, h ~ -W1 x, and W2 W1 has N(0, 1/sigma^2)
entries, so phi(x) . phi(y) ~ exp(-|x - y|^2 / (2 sigma^2)) before training.

Training, the forward pass and the per-molecule sums run in libkfb
(kfb_cosmlp_*); this module samples the pairs, drives the batches and keeps
checkpoints.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._device import host_i32, require_cuda, stream_handle

__all__ = ["CosMLPFeatureMap", "sample_pairs", "pair_targets", "fit_ridge", "predict_linear",
           "judge_feature_model", "element_baseline"]


def _x_dt(X):
    import torch
    if X.dtype == torch.float32:
        return _lib.KFB_F32
    if X.dtype == torch.float64:
        return _lib.KFB_F64
    raise RuntimeError("X must be float32 (or float64)")


def sample_pairs(Q, N, nelem, n_pairs, seed, molecules=None):
    """Seeded same-element atom pairs drawn uniformly over the atoms of the
    given molecules (default: all).  Returns one (pi, pj) pair of int32 arrays
    per element; indices are flat padded rows m * max_atoms + j, and each
    element gets pairs in proportion to its atom count."""
    q = host_i32(Q)
    n = host_i32(N).reshape(-1)
    nm, ma = q.shape
    mols = np.arange(nm) if molecules is None else np.asarray(molecules)
    rows, elem = [], []
    for m in mols:
        na = min(max(int(n[m]), 0), ma)
        e = q[m, :na]
        ok = e >= 0
        rows.append(m * ma + np.nonzero(ok)[0])
        elem.append(e[ok])
    rows = np.concatenate(rows) if rows else np.zeros(0, np.int64)
    elem = np.concatenate(elem) if elem else np.zeros(0, np.int32)
    rng = np.random.default_rng(seed)
    out = []
    total = max(len(rows), 1)
    for e in range(nelem):
        r = rows[elem == e]
        k = int(round(n_pairs * len(r) / total))
        if len(r) == 0 or k == 0:
            out.append((np.zeros(0, np.int32), np.zeros(0, np.int32)))
            continue
        out.append((r[rng.integers(0, len(r), k)].astype(np.int32),
                    r[rng.integers(0, len(r), k)].astype(np.int32)))
    return out


def pair_targets(X, pi, pj, sigma):
    """exp(-|x_i - x_j|^2 / (2 sigma^2)) for rows pi, pj of X (any shape whose
    last axis is the descriptor), computed on the device (float32)."""
    require_cuda()
    import torch
    Xr = X.reshape(-1, X.shape[-1]).contiguous()
    pi_d = torch.as_tensor(pi, dtype=torch.int32).to(Xr.device)
    pj_d = torch.as_tensor(pj, dtype=torch.int32).to(Xr.device)
    out = torch.empty((pi_d.numel(),), dtype=torch.float32, device=Xr.device)
    _lib.check(_lib.lib().kfb_pair_gaussian(Xr.data_ptr(), Xr.shape[0], pi_d.data_ptr(),
                                            pj_d.data_ptr(), pi_d.numel(), Xr.shape[1],
                                            float(sigma), _x_dt(Xr), out.data_ptr(),
                                            stream_handle()))
    return out


class CosMLPFeatureMap:
    """Per-element cos-MLP feature map rep -> hidden -> d (default 720 -> 512 ->
    4096) on one CUDA device."""

    def __init__(self, nelem, rep=720, hidden=512, d=4096, sigma=2.0, seed=0, max_pairs=4096,
                 init_scale=0.05):
        require_cuda()
        self.nelem, self.rep, self.hidden, self.d = int(nelem), int(rep), int(hidden), int(d)
        self.sigma, self.seed, self.max_pairs = float(sigma), int(seed), int(max_pairs)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().kfb_cosmlp_create(self.nelem, self.rep, self.hidden, self.d,
                                                self.max_pairs, ctypes.byref(h)))
        self._h = h
        self.init_parameters(init_scale)

    # -------------------------------------------------------------- memory
    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.lib().kfb_cosmlp_destroy(h)
            except Exception:
                pass
            self._h = None

    def _views(self, fn, shapes):
        """Tensors aliasing libkfb-owned device arrays (valid while the map lives)."""
        ptrs = [ctypes.c_void_p() for _ in range(4)]
        _lib.check(fn(self._h, *[ctypes.byref(p) for p in ptrs]))
        return [_device_view(p.value, shp) for p, shp in zip(ptrs, shapes)]

    def _shapes(self, per_element=False):
        E, H, D, R = self.nelem, self.hidden, self.d, self.rep
        if per_element:
            return [(H, R), (H,), (D, H), (D,)]
        return [(E, H, R), (E, H), (E, D, H), (E, D)]

    def parameters(self):
        """Device tensors (views) of the FP32 parameters W1, b1, W2, b2."""
        return self._views(_lib.lib().kfb_cosmlp_params, self._shapes())

    def grads(self):
        """Device tensors (views) of the last step's gradients (one element)."""
        return self._views(_lib.lib().kfb_cosmlp_grads, self._shapes(True))

    def sync(self, reset_optimizer=False):
        """Refresh the BF16 weight copies after writing the FP32 parameters."""
        _lib.check(_lib.lib().kfb_cosmlp_sync(self._h, int(bool(reset_optimizer)),
                                              stream_handle()))

    def init_parameters(self, init_scale=0.05):
        """Seeded initialisation (see the module docstring); zeroes Adam."""
        import torch
        rng = np.random.default_rng(self.seed)
        E, H, D, R = self.nelem, self.hidden, self.d, self.rep
        eps = float(init_scale)
        W1 = rng.standard_normal((E, H, R)) * eps
        b1 = np.full((E, H), math.pi / 2)
        W2 = rng.standard_normal((E, D, H)) / (self.sigma * eps * math.sqrt(H))
        b2 = rng.uniform(0.0, 2.0 * math.pi, (E, D))
        self.set_parameters([W1, b1, W2, b2], reset_optimizer=True)
        torch.cuda.current_stream().synchronize()

    def set_parameters(self, values, reset_optimizer=False):
        import torch
        for dst, v in zip(self.parameters(), values):
            dst.copy_(torch.as_tensor(np.asarray(v), dtype=torch.float32))
        self.sync(reset_optimizer)

    # ------------------------------------------------------------ training
    def step(self, elem, X, pi, pj, target, lr=1e-3, update=True):
        """One Adam step of element `elem` on a batch of pairs (device int32
        rows pi, pj of X viewed as (rows, rep); device float32 targets).
        Returns the batch loss."""
        Xr = X.reshape(-1, X.shape[-1])
        if not Xr.is_contiguous():
            raise RuntimeError("X must be contiguous")
        loss = ctypes.c_double(0.0)
        _lib.check(_lib.lib().kfb_cosmlp_pair_step(
            self._h, int(elem), Xr.data_ptr(), Xr.shape[0], _x_dt(Xr), pi.data_ptr(), pj.data_ptr(),
            target.data_ptr(), int(pi.numel()), float(lr), int(bool(update)), ctypes.byref(loss),
            stream_handle()))
        return loss.value

    def train(self, X, pairs, targets, epochs=1, lr=1e-3, batch=None, seed=0, lr_decay=1.0,
              log=None):
        """Adam over the pair sets of all elements for `epochs` passes.
        pairs[e] = (pi, pj) host arrays, targets[e] device float32; batches are
        interleaved across elements in proportion to their sizes.  Returns the
        mean loss of each epoch."""
        import torch
        batch = int(batch or self.max_pairs)
        dev = X.device
        pairs_d = [(torch.as_tensor(pi, dtype=torch.int32).to(dev),
                    torch.as_tensor(pj, dtype=torch.int32).to(dev)) for pi, pj in pairs]
        rng = np.random.default_rng(seed)
        history = []
        lr_e = float(lr)
        for ep in range(int(epochs)):
            sched = []
            perms = []
            for e, (pi, _) in enumerate(pairs_d):
                n = pi.numel()
                perms.append(torch.as_tensor(rng.permutation(n), device=dev) if n else None)
                sched += [(e, s) for s in range(0, n, batch)]
            order = rng.permutation(len(sched))
            tot, cnt = 0.0, 0
            for k in order:
                e, s0 = sched[k]
                pi, pj = pairs_d[e]
                sel = perms[e][s0:s0 + batch]
                bi = pi[sel].contiguous()
                bj = pj[sel].contiguous()
                bt = targets[e][sel].contiguous()
                loss = self.step(e, X, bi, bj, bt, lr=lr_e)
                tot += loss * bi.numel()
                cnt += bi.numel()
            history.append(tot / max(cnt, 1))
            if log:
                log(ep, history[-1])
            lr_e *= lr_decay
        return history

    # ----------------------------------------------------------- inference
    def features_elemental(self, X, Q, N):
        """Per-molecule sums of phi over the atoms of each element: (nmol, d)
        float32; Q holds element indices (-1 = padding) like the RFF path."""
        import torch
        if not X.is_cuda or X.dim() != 3:
            raise RuntimeError("X must be a 3D CUDA tensor (nmol, max_atoms, rep)")
        X = X.contiguous()
        nm, ma, rep = X.shape
        q = host_i32(Q).reshape(nm, ma)
        n = host_i32(N).reshape(nm)
        Z = torch.empty((nm, self.d), dtype=torch.float32, device=X.device)
        _lib.check(_lib.lib().kfb_cosmlp_features_elemental(
            self._h, X.data_ptr(), q.ctypes.data, n.ctypes.data, nm, ma, rep, _x_dt(X),
            Z.data_ptr(), stream_handle()))
        return Z

    # ---------------------------------------------------------- checkpoints
    def state_dict(self):
        """Host copies of the parameters and the Adam state."""
        import torch
        torch.cuda.current_stream().synchronize()
        names = ("W1", "b1", "W2", "b2")
        sd = {n: t.detach().cpu().numpy().copy() for n, t in zip(names, self.parameters())}
        m = (ctypes.c_void_p * 4)()
        v = (ctypes.c_void_p * 4)()
        steps = (ctypes.c_int * self.nelem)()
        _lib.check(_lib.lib().kfb_cosmlp_optimizer_state(self._h, m, v, steps))
        for k, (n, shp) in enumerate(zip(names, self._shapes())):
            sd["adam_m_" + n] = _device_view(m[k], shp).cpu().numpy().copy()
            sd["adam_v_" + n] = _device_view(v[k], shp).cpu().numpy().copy()
        sd["adam_steps"] = np.array(list(steps), np.int32)
        sd["config"] = np.array([self.nelem, self.rep, self.hidden, self.d], np.int64)
        sd["sigma"] = np.array(self.sigma)
        return sd

    def load_state_dict(self, sd):
        import torch
        cfg = [int(c) for c in sd["config"]]
        if cfg != [self.nelem, self.rep, self.hidden, self.d]:
            raise ValueError(f"checkpoint shape {cfg} does not match this map")
        names = ("W1", "b1", "W2", "b2")
        self.set_parameters([sd[n] for n in names], reset_optimizer=False)
        m = (ctypes.c_void_p * 4)()
        v = (ctypes.c_void_p * 4)()
        _lib.check(_lib.lib().kfb_cosmlp_optimizer_state(self._h, m, v, None))
        for k, (n, shp) in enumerate(zip(names, self._shapes())):
            _device_view(m[k], shp).copy_(torch.as_tensor(sd["adam_m_" + n]))
            _device_view(v[k], shp).copy_(torch.as_tensor(sd["adam_v_" + n]))
        steps = (ctypes.c_int * self.nelem)(*[int(s) for s in sd["adam_steps"]])
        _lib.check(_lib.lib().kfb_cosmlp_set_steps(self._h, steps))
        torch.cuda.current_stream().synchronize()

    def save(self, path):
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path, max_pairs=4096):
        sd = dict(np.load(path))
        nelem, rep, hidden, d = (int(c) for c in sd["config"])
        obj = cls(nelem, rep, hidden, d, sigma=float(sd["sigma"]), max_pairs=max_pairs)
        obj.load_state_dict(sd)
        return obj


def _device_view(ptr, shape):
    """A torch float32 CUDA tensor aliasing device memory owned by libkfb."""
    import torch
    n = int(np.prod(shape))

    class _Cuda:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (int(ptr), False),
                                    "version": 3, "strides": None}

    return torch.as_tensor(_Cuda(), device="cuda").view(*shape)


# ------------------------------------------------------------------ ridge
def fit_ridge(Z, y, l2, tol=1e-10, maxit=500, lambda_floor=True, factor="fp64"):
    """Weights of the linear ridge model (Z^T Z + l2 I) w = Z^T y (libkfb's
    kfb_ridge_solve_mixed: FP32 factor, FP64 refinement against Z itself).
    Returns (w float64 (d,), solve info dict)."""
    require_cuda()
    import torch
    if Z.dtype != torch.float32 or not Z.is_cuda or Z.dim() != 2:
        raise RuntimeError("Z must be a 2D float32 CUDA tensor")
    Z = Z.contiguous()
    nm, d = Z.shape
    yd = y.to(device=Z.device, dtype=torch.float64).contiguous()
    if yd.numel() != nm:
        raise RuntimeError("y must have one value per row of Z")
    w = torch.empty((d,), dtype=torch.float64, device=Z.device)
    info = _lib.SolveInfo()
    if factor not in ("fp32", "fp64"):
        raise ValueError("factor must be 'fp32' or 'fp64'")
    flags = (_lib.KFB_SOLVE_LAMBDA_FLOOR if lambda_floor else 0) | \
        (_lib.KFB_SOLVE_FP64_FACTOR if factor == "fp64" else 0)
    st = _lib.lib().kfb_ridge_solve_mixed(Z.data_ptr(), yd.data_ptr(), nm, d, float(l2),
                                          float(tol), int(maxit), flags, w.data_ptr(),
                                          ctypes.byref(info), stream_handle())
    res = {"iterations": info.iterations, "factor_info": info.factor_info, "shift": info.shift,
           "rel_residual": info.rel_residual, "used_cg": bool(info.used_cg),
           "lambda_eff": info.lambda_eff}
    if st == _lib.KFB_ERR_NOT_PD:
        raise RuntimeError(_lib.lib().kfb_last_error().decode())
    if st != _lib.KFB_OK and st != _lib.KFB_ERR_NO_CONVERGENCE:
        _lib.check(st)
    res["converged"] = st == _lib.KFB_OK
    return w, res


def predict_linear(Z, w):
    """Z @ w in float64."""
    import torch
    return Z.to(torch.float64) @ w.to(device=Z.device, dtype=torch.float64)


def element_baseline(Q, N, y, nelem, molecules=None):
    """Per-element energy baseline as the reference's models fit it
    (models/base.py:401-418): least squares of the energies on the element
    counts of each molecule, no intercept.  Q holds element indices (-1 =
    padding).  Returns (coef (nelem,), counts (nmol, nelem)); the baseline of
    molecule m is counts[m] @ coef."""
    q = host_i32(Q)
    n = host_i32(N).reshape(-1)
    nm, ma = q.shape
    counts = np.zeros((nm, nelem))
    valid = np.arange(ma)[None, :] < np.clip(n, 0, ma)[:, None]
    for e in range(nelem):
        counts[:, e] = np.sum((q == e) & valid, axis=1)
    idx = np.arange(nm) if molecules is None else np.asarray(molecules)
    coef, *_ = np.linalg.lstsq(counts[idx], np.asarray(y, np.float64)[idx], rcond=None)
    return coef, counts


def judge_feature_model(mae_feature, mae_exact, bound=1.01):
    """The feature model is used when its held-out MAE is within `bound` times
    the exact Gaussian KRR's; otherwise the exact model is the fallback."""
    ok = bool(np.isfinite(mae_feature)) and mae_feature <= bound * mae_exact
    return {"use": "feature" if ok else "exact", "mae_feature": float(mae_feature),
            "mae_exact": float(mae_exact), "bound": float(bound),
            "ratio": float(mae_feature / mae_exact) if mae_exact > 0 else float("inf")}
