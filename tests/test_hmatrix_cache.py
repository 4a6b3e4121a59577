"""H-matrix npz cache: the reference's HMatrixCPUData schema (storage.py:72-209) read and
written by the device H-matrix, and build_or_load_hmatrix's cache validation
(builder.py:814-927).

``tests/golden/hcache_film14.npz`` was written by the reference's own
``HMatrixCPUData.save`` (see tests/golden/make_golden.py); the expected products are
computed here from the file's arrays with the formula of ``HMatrixCPUData.matvec_cpu``
(storage.py:175-190).
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sps

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
from oracle import mesh as omesh  # noqa: E402

pytestmark = pytest.mark.gpu
GOLD = ROOT / "tests" / "golden"
FILM14 = (14, 14, 2, 2.5)


def _npz_matvec(a, x):
    perm = a["perm"]
    xp = x[perm]
    near = sps.csr_matrix((a["near_data"], a["near_indices"], a["near_indptr"]), shape=tuple(a["near_shape"]))
    y = a["diag_jump"][perm] * xp + near @ xp
    U, V = a["far_U_flat"], a["far_V_flat"]
    for m in a["far_meta"]:
        rs, re, cs, ce, k = (int(m[n]) for n in ("row_start", "row_stop", "col_start", "col_stop", "rank"))
        Ub = U[m["u_offset"]:m["u_offset"] + m["u_size"]].reshape(re - rs, k)
        Vb = V[m["v_offset"]:m["v_offset"] + m["v_size"]].reshape(k, ce - cs)
        y[rs:re] += Ub @ (Vb @ xp[cs:ce])
    out = np.empty_like(x)
    out[perm] = y
    return out


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def spx():
    import spinfemx_b200 as spx
    return spx


def _x(n, seed=5):
    return np.random.default_rng(seed).standard_normal(n)


def test_reference_cache_loads_and_applies(spx):
    import torch
    X, T = omesh.kuhn_box(*FILM14)
    geom = spx.BoundaryGeometry(X, T)
    cfg = spx.HMatrixBuildConfig(epsilon=1e-4, eta=2.0, leaf_size=16)
    a = np.load(GOLD / "hcache_film14.npz", allow_pickle=False)
    H, meta = spx.HMatrixGPUPackedFused.load(GOLD / "hcache_film14.npz", geom, cfg, precision="f64")
    assert np.array_equal(H.perm, a["perm"])
    assert json.loads(str(a["metadata_json"].item()))["Nb"] == geom.Nb == meta["Nb"]
    x = _x(geom.Nb)
    y = H.matvec(torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert _rel(y, _npz_matvec(a, x)) < 1e-13
    # our own build of the same operator agrees within the ACA tolerance
    H2 = spx.HMatrixGPUPackedFused(geom, cfg, precision="f64")
    y2 = H2.matvec(torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert _rel(y2, y) < 1e-3


def test_save_writes_reference_schema_and_reloads(spx, tmp_path):
    import torch
    X, T = omesh.kuhn_box(*FILM14)
    geom = spx.BoundaryGeometry(X, T)
    cfg = spx.HMatrixBuildConfig(epsilon=1e-4, eta=2.0, leaf_size=16)
    H = spx.HMatrixGPUPackedFused(geom, cfg, precision="f64")
    path = tmp_path / "h.npz"
    H.save(path, compressed=False, metadata={"Nb": geom.Nb})
    a = np.load(path, allow_pickle=False)
    ref = np.load(GOLD / "hcache_film14.npz", allow_pickle=False)
    assert sorted(a.files) == sorted(ref.files)
    for k in ref.files:  # metadata_json is a unicode scalar of its own length
        assert (a[k].dtype.kind == ref[k].dtype.kind) if k == "metadata_json" else (a[k].dtype == ref[k].dtype), k
    assert a["far_meta"].dtype.names == ref["far_meta"].dtype.names
    assert np.count_nonzero(a["near_data"] == 0.0) == 0
    x = _x(geom.Nb, 6)
    y = H.matvec(torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert _rel(_npz_matvec(a, x), y) < 1e-13
    H2, _ = spx.HMatrixGPUPackedFused.load(path, geom, cfg, precision="f64")
    y2 = H2.matvec(torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert _rel(y2, y) < 1e-13


def test_build_or_load_validates_the_cache(spx, tmp_path):
    import torch
    from spinfemx_b200.hmatrix import build_or_load_hmatrix
    X, T = omesh.kuhn_box(*FILM14)
    cfg = spx.HMatrixBuildConfig(epsilon=1e-4, eta=2.0, leaf_size=16)
    path = tmp_path / "cache.npz"
    H1 = build_or_load_hmatrix(path, X, T, cfg, precision="f64")
    assert path.exists() and H1.metadata["cache_loaded"] is False
    H2 = build_or_load_hmatrix(path, X, T, cfg, precision="f64")
    assert H2.metadata["cache_loaded"] is True
    x = torch.as_tensor(_x(H1.size, 7), device="cuda")
    assert _rel(H2.matvec(x).cpu().numpy(), H1.matvec(x).cpu().numpy()) < 1e-13
    H3 = build_or_load_hmatrix(path, X, T, spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=16),
                               precision="f64")
    assert H3.metadata["cache_loaded"] is False  # other configuration: rebuilt and rewritten
    X2 = X.copy()
    X2[:, 2] *= 1.01
    H4 = build_or_load_hmatrix(path, X2, T, spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=16),
                               precision="f64")
    assert H4.metadata["cache_loaded"] is False  # other geometry


def test_demag_uses_the_cache(spx, tmp_path):
    import torch
    X, T = omesh.kuhn_box(*FILM14)
    kw = dict(boundary_backend="hmatrix", hmatrix_epsilon=1e-4, hmatrix_leaf_size=16, precision="f64",
              ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10)
    N = X.shape[0]
    m = np.tile([0.6, 0.8, 0.0], (N, 1)) + 0.05 * np.random.default_rng(3).standard_normal((N, 3))
    m = torch.as_tensor((m / np.linalg.norm(m, axis=1)[:, None]).ravel(), device="cuda")
    d0 = spx.DemagFieldLindholmGPU(X, T, 8e5, **kw)
    H0 = torch.empty_like(m)
    d0.compute_vec(m, H0)
    path = tmp_path / "demag_cache.npz"
    for loaded in (False, True):
        d = spx.DemagFieldLindholmGPU(X, T, 8e5, hmatrix_cache_path=path, **kw)
        assert d.hmatrix_metadata["cache_loaded"] is loaded
        H = torch.empty_like(m)
        d.compute_vec(m, H)
        assert float(torch.linalg.norm(H - H0) / torch.linalg.norm(H0)) < 1e-9


def test_borrowed_handle_of_a_demag_object(spx, tmp_path):
    """The H-matrix a demag object lends out (spx_demag_hmat) is a full handle: it saves in the
    cache schema and reloads to the same operator, the demag object keeps working, and
    destroying it through the ABI is refused (it goes with the demag object)."""
    import ctypes as C

    import torch
    from spinfemx_b200 import _lib
    X, T = omesh.kuhn_box(*FILM14)
    d = spx.DemagFieldLindholmGPU(X, T, 8e5, boundary_backend="hmatrix", hmatrix_epsilon=1e-4,
                                  hmatrix_leaf_size=16, precision="f64")
    m = np.tile([0.6, 0.8, 0.0], X.shape[0])
    Hf = torch.empty(3 * X.shape[0], dtype=torch.float64, device="cuda")
    d.compute_vec(torch.as_tensor(m, device="cuda"), Hf)
    before = Hf.cpu().numpy().copy()
    B = d.B_hmatrix_gpu
    path = tmp_path / "borrowed.npz"
    B.save(path, compressed=False)  # export through the borrowed handle
    geom = spx.BoundaryGeometry(X, T)
    cfg = spx.HMatrixBuildConfig(epsilon=1e-4, eta=2.0, leaf_size=16)
    H2, _ = spx.HMatrixGPUPackedFused.load(path, geom, cfg, precision="f64")
    x = torch.as_tensor(_x(geom.Nb, 7), device="cuda")
    assert _rel(H2.matvec(x).cpu().numpy(), B.matvec(x).cpu().numpy()) < 1e-13
    assert _lib.lib().spx_hmat_destroy(B.handle) != 0  # refused, nothing freed
    d.compute_vec(torch.as_tensor(m, device="cuda"), Hf)
    assert np.array_equal(Hf.cpu().numpy(), before)
