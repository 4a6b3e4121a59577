"""H-matrix apply to several right-hand sides at once (spx_hmat_apply_multi) against the
single-vector apply, and ensembles whose samples share one geometry (one H-matrix applied to
all of them) against the samples run on their own."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import mesh as omesh

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def spx():
    import spinfemx_b200 as spx
    return spx


@pytest.mark.parametrize("precision", ["f64", "f32", "bf16"])
def test_matmat_equals_matvecs(spx, precision):
    X, T = omesh.kuhn_box(20, 14, 3, 2.0)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=16),
                                  precision=precision)
    rng = np.random.default_rng(5)
    for R in (1, 3, 8, 11):
        Xs = torch.as_tensor(rng.normal(size=(R, geom.Nb)), device="cuda")
        Y = H.matmat(Xs)
        for r in range(R):
            y = H.matvec(Xs[r].contiguous())
            err = float(torch.linalg.norm(Y[r] - y) / torch.linalg.norm(y))
            assert err < 1e-13, (R, r, err)
        Y2 = H.matmat(Xs)  # a second call reuses the work buffers
        assert torch.equal(Y, Y2)


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_ensemble_shared_geometry_equals_per_sample(spx, precision):
    boxes = [(12, 10, 2), (9, 7, 3), (12, 10, 2), (12, 10, 2)]  # three samples share one geometry
    ms = [omesh.kuhn_box(nx, ny, nz, 2.0) for nx, ny, nz in boxes]
    X, T, off = spx.ensemble_mesh(ms)
    kw = dict(precision=precision, ksp_rtol_u1=1e-12, ksp_rtol_u2=1e-12, ksp_atol=0.0, ksp_maxit_u1=20000,
              ksp_maxit_u2=20000, hmatrix_epsilon=1e-7, hmatrix_leaf_size=16)
    d = spx.DemagFieldLindholmGPU(X, T, 8e5, boundary_backend="ensemble", sample_offsets=off, dense_max_nb=100,
                                  **kw)
    rng = np.random.default_rng(7)
    m = rng.normal(size=(X.shape[0], 3))
    m = (m / np.linalg.norm(m, axis=1)[:, None]).ravel()
    H = torch.empty(3 * X.shape[0], dtype=torch.float64, device="cuda")
    d.compute_vec(torch.as_tensor(m, device="cuda"), H)
    H = H.cpu().numpy()
    for k, (Xs, Ts) in enumerate(ms):
        ds = spx.DemagFieldLindholmGPU(Xs, Ts, 8e5, boundary_backend="hmatrix", **kw)
        Hs = torch.empty(3 * Xs.shape[0], dtype=torch.float64, device="cuda")
        ds.compute_vec(torch.as_tensor(m[3 * off[k]:3 * off[k + 1]], device="cuda"), Hs)
        Hs = Hs.cpu().numpy()
        err = np.linalg.norm(H[3 * off[k]:3 * off[k + 1]] - Hs) / np.linalg.norm(Hs)
        assert err < (1e-9 if precision == "f64" else 2e-6), (k, err)
