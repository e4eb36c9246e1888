"""Feature maps on the GPU through libkfb, against the oracle and the
reference's golden outputs.

* RFF features: split-fp16 tensor-core products, FP32-class accuracy against
  the reference's FP64 output: relative Frobenius error <= 2e-6.
* Normal equations: FP32 SYRK, relative error <= 1e-5 against Z^T Z in FP64.
* cos-MLP forward and gradients: BF16 operands, FP32 accumulation; compared
  with the oracle that applies the same BF16 roundings in FP64, relative
  Frobenius error <= 2e-3 (a few operands round to the other side of a BF16
  tie when the FP32 and FP64 pre-activations differ in the last bits).
"""
import numpy as np
import pytest

from conftest import load_golden
from oracle import features as of
from oracle import oracle as o

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def cuda(a, dtype=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a))
    return t.to(device="cuda", dtype=dtype or t.dtype)


@pytest.mark.parametrize("case", ["f", "r"])
@pytest.mark.parametrize("xdtype", ["float32", "float64"])
def test_rff_features_match_reference(case, xdtype):
    import torch
    from kernelforge_b200 import cuda_rff_features as crf
    g = load_golden("golden_rff.npz")
    X = cuda(g[case + "_X"], getattr(torch, xdtype))
    Z = crf.rff_features_elemental(X, g[case + "_Q"], g[case + "_N"],
                                   cuda(g[case + "_W"], torch.float32),
                                   cuda(g[case + "_b"], torch.float32))
    ref = of.rff_features_elemental(np.asarray(X.cpu(), np.float64), g[case + "_Q"],
                                    g[case + "_N"], g[case + "_W"].astype(np.float32),
                                    g[case + "_b"].astype(np.float32))
    assert Z.shape == g[case + "_Z"].shape and Z.dtype == torch.float32
    assert rel(Z.cpu().numpy(), ref) <= 2e-6
    # and against the reference's own FP64 output (W, b in FP64 there)
    assert rel(Z.cpu().numpy(), g[case + "_Z"]) <= 2e-5
    N = g[case + "_N"]
    assert np.all(Z.cpu().numpy()[N == 0] == 0.0)


@pytest.mark.parametrize("case", ["f", "r"])
def test_rff_gramian_matches_reference(case):
    import torch
    from kernelforge_b200 import cuda_rff_features as crf
    g = load_golden("golden_rff.npz")
    ztz, zty = crf.rff_gramian_elemental_rfp(
        cuda(g[case + "_X"], torch.float32), g[case + "_Q"], g[case + "_N"],
        cuda(g[case + "_W"], torch.float32), cuda(g[case + "_b"], torch.float32),
        cuda(g[case + "_Y"], torch.float64))
    D = g[case + "_b"].shape[1]
    got = o.rfp_to_full(ztz.cpu().numpy().astype(np.float64), D, uplo_lower=True)
    ref = o.rfp_to_full(g[case + "_ZtZ_rfp"], D, uplo_lower=False)
    assert rel(got, ref) <= 1e-5
    assert rel(zty.cpu().numpy(), g[case + "_ZtY"]) <= 1e-5


def test_feature_gramian_layouts_agree():
    import torch
    from kernelforge_b200 import cuda_rff_features as crf
    rng = np.random.default_rng(11)
    Zh = rng.standard_normal((333, 72)).astype(np.float32)
    y = rng.standard_normal(333)
    Z = cuda(Zh)
    full, zty = crf.feature_gramian(Z, cuda(y), "full")
    ref = Zh.astype(np.float64).T @ Zh.astype(np.float64)
    assert rel(full.cpu().numpy(), ref) <= 1e-6
    np.testing.assert_allclose(full.cpu().numpy(), full.cpu().numpy().T, rtol=0, atol=0)
    assert rel(zty.cpu().numpy(), Zh.astype(np.float64).T @ y) <= 1e-12
    for lay, low in (("L", True), ("U", False)):
        rfp, none = crf.feature_gramian(Z, None, lay)
        assert none is None
        back = o.rfp_to_full(rfp.cpu().numpy().astype(np.float64), 72, uplo_lower=low)
        np.testing.assert_array_equal(back, full.cpu().numpy().astype(np.float64))


def test_pair_gaussian_matches_oracle():
    import torch
    from kernelforge_b200.feature_maps import pair_targets
    g = load_golden("golden_fchl19_720.npz")
    X = g["X"]
    rows = X.reshape(-1, X.shape[-1])
    rng = np.random.default_rng(5)
    pi = rng.integers(0, rows.shape[0], 300).astype(np.int32)
    pj = rng.integers(0, rows.shape[0], 300).astype(np.int32)
    for dt in (torch.float32, torch.float64):
        Xd = cuda(X, dt)
        t = pair_targets(Xd, pi, pj, 2.0).cpu().numpy()
        xr = np.asarray(Xd.cpu(), np.float64).reshape(-1, X.shape[-1])
        ref = np.exp(-np.sum((xr[pi] - xr[pj]) ** 2, axis=1) / 8.0)
        np.testing.assert_allclose(t, ref, rtol=2e-7, atol=1e-7)


def _elem_q(Qz, N, elements=(1, 6, 7, 8)):
    Qe = np.full(Qz.shape, -1, np.int32)
    for m in range(Qz.shape[0]):
        for j in range(N[m]):
            Qe[m, j] = elements.index(int(Qz[m, j]))
    return Qe


def _net_params(fm):
    W1, b1, W2, b2 = [t.detach().cpu().numpy().astype(np.float64) for t in fm.parameters()]
    return [(W1[e], b1[e], W2[e], b2[e]) for e in range(fm.nelem)]


def test_cosmlp_features_match_oracle():
    import torch
    from kernelforge_b200.feature_maps import CosMLPFeatureMap
    g = load_golden("golden_fchl19_720.npz")
    X, N = g["X"], g["N"]
    Qe = _elem_q(g["Q"], N)
    fm = CosMLPFeatureMap(4, rep=720, hidden=64, d=160, sigma=2.0, seed=3, max_pairs=64)
    Z = fm.features_elemental(cuda(X, torch.float32), Qe, N).cpu().numpy()
    ref = of.cosmlp_features_elemental_bf16(X.astype(np.float32), Qe, N, _net_params(fm))
    assert rel(Z, ref) <= 2e-3
    # the FP64 map without BF16 roundings is within BF16 accuracy
    exact = of.cosmlp_features_elemental(X, Qe, N, _net_params(fm))
    assert rel(Z, exact) <= 3e-2


@pytest.mark.parametrize("npairs", [40, 8, 203, 2048])
def test_cosmlp_gradients_match_oracle(npairs):
    import torch
    from kernelforge_b200.feature_maps import CosMLPFeatureMap
    rng = np.random.default_rng(npairs)
    rows = (rng.standard_normal((120, 48)) * 0.7).astype(np.float32)
    fm = CosMLPFeatureMap(2, rep=48, hidden=32, d=144, sigma=2.0, seed=9, max_pairs=2048,
                          init_scale=0.3)
    pi = rng.integers(0, 120, npairs).astype(np.int32)
    pj = rng.integers(0, 120, npairs).astype(np.int32)
    t = rng.uniform(0.0, 1.0, npairs).astype(np.float32)
    elem = 1
    Xd = cuda(rows)
    loss = fm.step(elem, Xd, cuda(pi), cuda(pj), cuda(t), update=False)
    gpu = [a.detach().cpu().numpy() for a in fm.grads()]
    W1, b1, W2, b2 = _net_params(fm)[elem]
    ref_loss, ref = of.cosmlp_pair_loss_grad_bf16(rows[pi], rows[pj], t, W1, b1, W2, b2)
    assert abs(loss - ref_loss) <= 1e-4 * ref_loss
    for name, a, b in zip(("W1", "b1", "W2", "b2"), gpu, ref):
        assert rel(a, b) <= 2e-3, name
    # and the unrounded FP64 gradient, within BF16 accuracy
    _, exact = of.cosmlp_pair_loss_grad(rows[pi], rows[pj], t, W1, b1, W2, b2)
    for name, a, b in zip(("W1", "b1", "W2", "b2"), gpu, exact):
        assert rel(a, b) <= 5e-2, name


def test_cosmlp_adam_first_step():
    """At step 1 Adam moves each parameter by lr * g / (|g| + eps)."""
    import torch
    from kernelforge_b200.feature_maps import CosMLPFeatureMap
    rng = np.random.default_rng(2)
    rows = (rng.standard_normal((64, 32)) * 0.5).astype(np.float32)
    fm = CosMLPFeatureMap(2, rep=32, hidden=16, d=64, sigma=2.0, seed=1, max_pairs=64,
                          init_scale=0.3)
    pi = rng.integers(0, 64, 48).astype(np.int32)
    pj = rng.integers(0, 64, 48).astype(np.int32)
    t = rng.uniform(0.0, 1.0, 48).astype(np.float32)
    before = [p.detach().cpu().numpy().copy() for p in fm.parameters()]
    lr = 1e-3
    fm.step(0, cuda(rows), cuda(pi), cuda(pj), cuda(t), lr=lr, update=True)
    grads = [gr.detach().cpu().numpy() for gr in fm.grads()]
    after = [p.detach().cpu().numpy() for p in fm.parameters()]
    for k in range(4):
        want = before[k][0] - lr * grads[k] / (np.abs(grads[k]) + 1e-8)
        np.testing.assert_allclose(after[k][0], want, rtol=1e-5, atol=1e-7)
        np.testing.assert_array_equal(after[k][1], before[k][1])  # element 1 untouched


def test_cosmlp_checkpoint_resume(tmp_path):
    import torch
    from kernelforge_b200.feature_maps import CosMLPFeatureMap
    rng = np.random.default_rng(4)
    rows = (rng.standard_normal((80, 32)) * 0.5).astype(np.float32)
    pi = cuda(rng.integers(0, 80, 64).astype(np.int32))
    pj = cuda(rng.integers(0, 80, 64).astype(np.int32))
    t = cuda(rng.uniform(0.0, 1.0, 64).astype(np.float32))
    Xd = cuda(rows)
    a = CosMLPFeatureMap(1, rep=32, hidden=16, d=64, seed=6, max_pairs=64, init_scale=0.3)
    for _ in range(3):
        a.step(0, Xd, pi, pj, t, lr=1e-2)
    path = tmp_path / "cosmlp.npz"
    a.save(path)
    b = CosMLPFeatureMap.load(path, max_pairs=64)
    la = [a.step(0, Xd, pi, pj, t, lr=1e-2) for _ in range(3)]
    lb = [b.step(0, Xd, pi, pj, t, lr=1e-2) for _ in range(3)]
    np.testing.assert_allclose(la, lb, rtol=1e-5)
    for p, q in zip(a.parameters(), b.parameters()):
        np.testing.assert_allclose(p.cpu().numpy(), q.cpu().numpy(), rtol=1e-5, atol=1e-6)


def test_cosmlp_rejects_bad_arguments():
    import torch
    from kernelforge_b200 import _lib
    from kernelforge_b200.feature_maps import CosMLPFeatureMap
    fm = CosMLPFeatureMap(1, rep=32, hidden=16, d=64, seed=6, max_pairs=16)
    x = cuda(np.zeros((4, 32), np.float32))
    idx = cuda(np.zeros(20, np.int32))
    t = cuda(np.zeros(20, np.float32))
    with pytest.raises(ValueError, match="npairs"):
        fm.step(0, x, idx, idx, t)
    with pytest.raises(ValueError, match="element"):
        fm.step(3, x, idx[:4], idx[:4], t[:4])
    with pytest.raises(ValueError):
        fm.features_elemental(cuda(np.zeros((2, 3, 48), np.float32)), np.zeros((2, 3)),
                              np.array([3, 3]))
    with pytest.raises((ValueError, _lib.KfbError)):
        CosMLPFeatureMap(1, rep=30, hidden=16, d=64)


def test_ridge_on_features_matches_fp64_solve():
    import torch
    from kernelforge_b200.feature_maps import fit_ridge, predict_linear
    rng = np.random.default_rng(8)
    Zh = rng.standard_normal((500, 96)).astype(np.float32)
    y = Zh.astype(np.float64) @ rng.standard_normal(96) + 0.01 * rng.standard_normal(500)
    w, info = fit_ridge(cuda(Zh), cuda(y), l2=1e-3, tol=1e-12)
    Zd = Zh.astype(np.float64)
    ref = np.linalg.solve(Zd.T @ Zd + 1e-3 * np.eye(96), Zd.T @ y)
    assert info["converged"] and info["lambda_eff"] == 1e-3
    # the refinement runs against Z itself: the exact normal equations
    assert rel(w.cpu().numpy(), ref) <= 1e-9
    assert rel(predict_linear(cuda(Zh), w).cpu().numpy(), Zd @ ref) <= 1e-9


def test_ridge_with_dominant_mode_below_fp32_resolution():
    """Per-molecule feature sums share one dominant direction; with the small
    eigenvalues below FP32 resolution of Z^T Z the solve still returns the FP64
    normal-equation solution at the requested l2 (no lambda floor needed)."""
    import torch
    from kernelforge_b200.feature_maps import fit_ridge
    rng = np.random.default_rng(12)
    nm, d = 3000, 160
    common = rng.uniform(0.5, 1.5, d)
    counts = rng.integers(9, 31, nm)
    Zh = (counts[:, None] * common[None, :] +
          0.01 * rng.standard_normal((nm, d))).astype(np.float32)
    y = Zh.astype(np.float64) @ (rng.standard_normal(d) * 0.1) + rng.standard_normal(nm)
    Zd = Zh.astype(np.float64)
    A = Zd.T @ Zd
    ev = np.linalg.eigvalsh(A)
    assert ev[-1] / ev[0] > 1e9          # far beyond FP32
    l2 = 1e-3
    # the FP64 residual floor of this system is ~1e-12 relative (|A| |w| >> |Z^T y|)
    w, info = fit_ridge(cuda(Zh), cuda(y), l2=l2, tol=1e-11, maxit=2000)
    ref = np.linalg.solve(A + l2 * np.eye(d), Zd.T @ y)
    assert info["converged"] and info["lambda_eff"] == l2, info
    assert rel(w.cpu().numpy(), ref) <= 1e-6


def test_training_gains_over_the_untrained_map():
    """What the trained network gains over the method without it: on held-out
    same-element pairs of FCHL19 atoms, the trained map's pair-kernel error is
    several times below that of the untrained map (a random-Fourier-like map of
    the same sigma) and below RFF at equal D."""
    import torch
    from kernelforge_b200 import cuda_rff_features as crf
    from kernelforge_b200 import synthetic
    from kernelforge_b200.feature_maps import CosMLPFeatureMap, pair_targets, sample_pairs
    mols = synthetic.make_molecules(400, 9, 21, seed=31)
    X, Qz, N = synthetic.fchl19_batched(mols, dtype=np.float32, device="cuda", chunk=128)
    Qe = _elem_q(Qz, N)
    Xd = cuda(X)
    ma, D = X.shape[1], 1024
    train = np.arange(300)
    test = np.arange(300, 400)
    pairs = sample_pairs(Qe, N, 4, 120000, seed=1, molecules=train)
    targets = [pair_targets(Xd, pi, pj, 2.0) for pi, pj in pairs]
    held = sample_pairs(Qe, N, 4, 8000, seed=2, molecules=test)
    W = torch.randn((4, 720, D), generator=torch.Generator().manual_seed(3)).cuda() / 2.0
    b = (torch.rand((4, D), generator=torch.Generator().manual_seed(4)) * 2 * np.pi).cuda()

    def rmse(feat):
        err = []
        for e, (pi, pj) in enumerate(held):
            if len(pi) == 0:
                continue
            def at(rows):
                xa = Xd.reshape(-1, 1, 720)[torch.tensor(rows, device="cuda").long()].contiguous()
                return feat(xa, np.full((len(rows), 1), e, np.int32), np.ones(len(rows), np.int32))
            k = (at(pi) * at(pj)).sum(1)
            err.append(((k - pair_targets(Xd, pi, pj, 2.0)) ** 2).double().cpu().numpy())
        return float(np.sqrt(np.concatenate(err).mean()))

    fm = CosMLPFeatureMap(4, 720, 256, D, sigma=2.0, seed=5, max_pairs=4096)
    untrained = rmse(fm.features_elemental)
    hist = fm.train(Xd, pairs, targets, epochs=4, lr=1e-3, batch=2048, seed=6)
    trained = rmse(fm.features_elemental)
    rff = rmse(lambda xa, q, n: crf.rff_features_elemental(xa, q, n, W, b))
    assert hist[-1] < hist[0]
    assert trained < untrained / 3, (trained, untrained)
    assert trained < rff, (trained, rff)


@pytest.mark.parametrize("case", ["f", "r"])
@pytest.mark.parametrize("xdtype", ["float32", "float64"])
def test_rff_force_features_match_reference(case, xdtype):
    """Force features G and the energy + force normal equations against the reference's
    kitchen_sinks (tests/golden/golden_rff_force.npz) and the oracle on the same
    float32 weights: split-fp16 products, FP32 accumulation."""
    import torch
    from kernelforge_b200 import cuda_rff_features as crf
    g = load_golden("golden_rff_force.npz")
    a = {k[2:]: g[k] for k in g if k.startswith(case + "_")}
    dt = getattr(torch, xdtype)
    X, dX = cuda(a["X"], dt), cuda(a["dX"], dt)
    W, b = cuda(a["W"], torch.float32), cuda(a["b"], torch.float32)
    G = crf.rff_gradient_elemental(X, dX, a["Q"], a["N"], W, b)
    assert G.dtype == torch.float32 and tuple(G.shape) == a["G"].T.shape
    ref32 = of.rff_gradient_elemental(np.asarray(X.cpu(), np.float64),
                                      np.asarray(dX.cpu(), np.float64), a["Q"], a["N"],
                                      a["W"].astype(np.float32), a["b"].astype(np.float32))
    assert rel(G.cpu().numpy(), ref32) <= 2e-5
    assert rel(G.cpu().numpy(), a["G"].T) <= 1e-4
    # energy + force normal equations (RFP 'L' here, 'U' in the reference's CPU code)
    ztz, zty = crf.rff_full_gramian_elemental_rfp(X, dX, a["Q"], a["N"], W, b,
                                                  cuda(a["Y"], torch.float64),
                                                  cuda(a["F"], torch.float64))
    D = a["b"].shape[1]
    got = o.rfp_to_full(ztz.cpu().numpy().astype(np.float64), D, uplo_lower=True)
    ref = o.rfp_to_full(a["ZtZ_rfp"], D, uplo_lower=False)
    assert rel(got, ref) <= 2e-4
    assert rel(zty.cpu().numpy(), a["ZtY"]) <= 2e-4
    # force predictions are G @ w
    w = torch.tensor(np.random.default_rng(3).standard_normal(D), device="cuda")
    Fp = crf.rff_predict_force_elemental(X, dX, a["Q"], a["N"], W, b, w)
    # each call recomputes G, whose per-molecule sums are accumulated atomically
    # in FP32: entries may differ between calls in the last bits, so the bound is
    # FP32-level against sum |G| |w| (and max |G| for the transposed copy)
    Gd, wn = G.double().cpu().numpy(), w.cpu().numpy()
    np.testing.assert_allclose(Fp.cpu().numpy(), Gd @ wn, rtol=0,
                               atol=1e-6 * (np.abs(Gd) @ np.abs(wn)).max())
    Gt = crf.rff_gradient_elemental_col_major(X, dX, a["Q"], a["N"], W, b)
    np.testing.assert_allclose(Gt.cpu().numpy(), G.cpu().numpy().T, rtol=0,
                               atol=1e-6 * np.abs(Gd).max())
