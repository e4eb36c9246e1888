"""Model-level API on the GPU against the reference's own LocalKRRModel
(tests/golden/golden_models.npz and the model it saved, ref_local_krr_ef.npz,
made by tests/golden/make_golden_models.py).  FP64 path: predictions at rtol
1e-6 (lambda 1e-8 amplifies the kernels' last-bit differences); a model loaded
from the reference's file predicts its values to 1e-9."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

KW = dict(sigma=2.5, l2=1e-8, elements=[1, 6, 7, 8], repr_params=dict(nRs2=8, nRs3=6))


def data():
    g = load_golden("golden_models.npz")
    N = g["N"]
    R = [g["R"][m, :N[m]] for m in range(len(N))]
    Z = [g["Z"][m, :N[m]] for m in range(len(N))]
    F = [g["F"][m, :N[m]] for m in range(len(N))]
    return g, R, Z, g["E"], F


def close(got, ref, rtol):
    ref = np.asarray(ref)
    np.testing.assert_allclose(got, ref, rtol=rtol, atol=rtol * np.abs(ref).max())


@pytest.mark.parametrize("mode", ["e", "f", "ef"])
def test_local_krr_matches_reference(mode):
    from kernelforge_b200.models import LocalKRRModel
    g, R, Z, E, F = data()
    kw = {"e": dict(energies=E[:16]), "f": dict(forces=F[:16]),
          "ef": dict(energies=E[:16], forces=F[:16])}[mode]
    m = LocalKRRModel(**KW).fit(R[:16], Z[:16], **kw)
    Ep, Fp = m.predict(R[16:], Z[16:])
    close(Ep, g[f"{mode}_E"], 1e-6)
    close(Fp, g[f"{mode}_F"], 1e-6)
    for k, s in m.train_score_.items():
        np.testing.assert_allclose(s.mae, g[f"{mode}_train_{k}_mae"], rtol=1e-4, atol=1e-9)


def test_load_reference_saved_model(tmp_path):
    """The reference's .npz loads into the GPU model, predicts the reference's values,
    and survives a save / load round trip."""
    from kernelforge_b200.models import LocalKRRModel
    g, R, Z, E, F = data()
    m = LocalKRRModel.load(os.path.join(GOLDEN, "ref_local_krr_ef.npz"))
    assert m.training_mode_ == "energy_and_force" and m.elements == [1, 6, 7, 8]
    Ep, Fp = m.predict(R[16:], Z[16:])
    close(Ep, g["ef_E"], 1e-9)
    close(Fp, g["ef_F"], 1e-9)
    m.save(tmp_path / "ours")
    m2 = LocalKRRModel.load(tmp_path / "ours.npz")
    Ep2, Fp2 = m2.predict(R[16:], Z[16:])
    # same model; the per-molecule energy and force sums are atomic adds of
    # terms of both signs, so repeated predictions agree to ~1e-12 relative
    np.testing.assert_allclose(Ep2, Ep, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(Fp2, Fp, rtol=1e-10, atol=1e-12 * np.abs(Fp).max())
    sc = m2.score(R[16:], Z[16:], energies=E[16:], forces=F[16:])
    assert set(sc) == {"energy", "force"} and sc["energy"].mae >= 0


@pytest.mark.parametrize("solver,kw,forces,l2", [
    ("cholesky", {}, True, 1e-4),
    ("eigh", dict(spectral_rtol=1e-13), True, 1e-4),     # nothing truncated: the exact solve
    # Jacobi CG converges on a well-conditioned system: energies, lambda 1e-2
    ("cg", dict(cg_rtol=1e-10, preprocessing="none"), False, 1e-2),
    ("cg", dict(cg_rtol=1e-10), False, 1e-2),           # with diagonal scaling
])
def test_cuda_local_krr(tmp_path, solver, kw, forces, l2):
    """Tensor-core kernel + each solver: close to the FP64 model at the same
    lambda, and a save / load round trip predicts the same values."""
    from kernelforge_b200.models import CudaLocalKRRModel, LocalKRRModel
    g, R, Z, E, F = data()
    lab = dict(energies=E[:16], forces=F[:16] if forces else None)
    ref = LocalKRRModel(sigma=2.5, l2=l2, elements=[1, 6, 7, 8],
                        repr_params=dict(nRs2=8, nRs3=6)).fit(R[:16], Z[:16], **lab)
    Er, Fr = ref.predict(R[16:], Z[16:])
    m = CudaLocalKRRModel(sigma=2.5, l2=l2, elements=[1, 6, 7, 8],
                          repr_params=dict(nRs2=8, nRs3=6), solver=solver,
                          **kw).fit(R[:16], Z[:16], **lab)
    if solver != "cholesky":
        assert m.solve_info_["solver"] == solver
        assert all(np.isfinite(s.mae) for s in m.train_score_.values())
    Ec, Fc = m.predict(R[16:], Z[16:])
    assert np.abs(Ec - Er).max() < 1e-2 * np.abs(Er).max() + 1e-3
    if forces:
        assert np.linalg.norm(Fc - Fr) < 1e-2 * np.linalg.norm(Fr) + 1e-3
    else:
        assert not np.any(Fc)   # the energy-only CUDA model predicts zero forces
    m.save(tmp_path / "c.npz")
    m2 = CudaLocalKRRModel.load(tmp_path / "c.npz")
    Ec2, Fc2 = m2.predict(R[16:], Z[16:])
    np.testing.assert_allclose(Ec2, Ec, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(Fc2, Fc, rtol=1e-5, atol=1e-5 * np.abs(Fc).max())


def test_cuda_model_truncated_eigensolve_and_errors():
    """The reference's default solver (truncated eigh) drops the eigenpairs below
    spectral_rtol * lambda_max; unknown solver / preprocessing names raise
    ValueError when fit runs (models/cuda_local_krr.py:314, :426)."""
    from kernelforge_b200.models import CudaLocalKRRModel
    g, R, Z, E, F = data()
    kw = dict(sigma=2.5, l2=1e-8, elements=[1, 6, 7, 8], repr_params=dict(nRs2=8, nRs3=6))
    m = CudaLocalKRRModel(**kw, spectral_rtol=1e-3).fit(R[:16], Z[:16], energies=E[:16])
    info = m.solve_info_
    assert info["solver"] == "eigh" and 0 < info["rank"] < 16 and info["dropped"] > 0
    assert info["tau"] == pytest.approx(1e-3 * info["lam_max"])
    Ep, _ = m.predict(R[16:], Z[16:])
    assert np.all(np.isfinite(Ep))
    with pytest.raises(ValueError, match="Unsupported solver"):
        CudaLocalKRRModel(**kw, solver="lu").fit(R[:4], Z[:4], energies=E[:4])
    with pytest.raises(ValueError, match="Unsupported preprocessing"):
        CudaLocalKRRModel(**kw, preprocessing="zca").fit(R[:4], Z[:4], energies=E[:4])


def test_model_errors():
    from kernelforge_b200.models import LocalKRRModel
    g, R, Z, E, F = data()
    with pytest.raises(RuntimeError):
        LocalKRRModel(**KW).predict(R[:2], Z[:2])
    with pytest.raises(ValueError):
        LocalKRRModel(**KW).fit(R[:3], Z[:2], energies=E[:3])
    with pytest.raises(ValueError):
        LocalKRRModel(**KW).fit(R[:3], Z[:3])
    m = LocalKRRModel(**KW).fit(R[:8], Z[:8], energies=E[:8])
    with pytest.raises(ValueError):
        m.score(R[8:10], Z[8:10], forces=F[8:10])
