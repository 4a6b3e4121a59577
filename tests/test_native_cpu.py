"""libspx on the CPU: exported symbols, host set-up code vs the oracle, error paths."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from oracle import fem as ofem
from oracle import lindholm as olin
from oracle import mesh as omesh

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def spx():
    import importlib.util
    spec = importlib.util.spec_from_file_location("spx_build", ROOT / "fenicsx-micromagnetics_b200" / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build()
    import spinfemx_b200
    from spinfemx_b200 import _lib
    _lib.lib()
    return spinfemx_b200


def test_library_exports_every_header_symbol(spx):
    from spinfemx_b200 import _lib
    header = (ROOT / "include" / "spx.h").read_text()
    names = set(re.findall(r"\b(spx_[a-z0-9_]+)\s*\(", header))
    assert len(names) > 40
    raw = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(raw, n)]
    assert not missing, missing
    # every exported name has a Python binding signature
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_device_count_without_gpu(spx):
    from spinfemx_b200 import _lib
    import torch
    n = _lib.device_count()
    assert n >= 0
    if not torch.cuda.is_available():
        assert n == 0


@pytest.mark.parametrize("dims", [(20, 20, 5, 2.0), (30, 30, 2, 2.5), (7, 5, 3, 1.5)])
def test_boundary_data_matches_oracle(spx, dims):
    X, T = omesh.kuhn_box(*dims)
    X2, T2 = spx.kuhn_box(*dims)
    assert np.array_equal(X, X2) and np.array_equal(T, T2)
    got = spx.boundary_data(X, T)
    ref = olin.boundary_data(X, T)
    assert np.array_equal(got["bverts"], ref["bverts"])
    assert np.array_equal(got["tri_lid"], ref["tri_lid"])
    assert np.array_equal(got["Xb"], ref["Xb"])
    assert np.abs(got["ntri"] - ref["ntri"]).max() < 1e-15
    assert np.abs(got["area"] - ref["area"]).max() < 1e-12
    assert np.abs(got["omega_sum"] - ref["omega_sum"]).max() < 1e-12


def test_fem_assembly_matches_oracle(spx):
    X, T = omesh.kuhn_box(9, 7, 4, 2.0)
    f = spx.fem_assemble(X, T)
    import scipy.sparse as sp
    N = X.shape[0]
    A = sp.csr_matrix((f["A"], f["col"], f["rowptr"]), shape=(N, N))
    Ao = ofem.stiffness(X, T)
    assert abs(A - Ao).max() < 1e-13
    Ms = 8e5
    # Div [N, 3N] from the 3-plane scalar-pattern storage
    rows = np.repeat(np.arange(N), np.diff(f["rowptr"]))
    D = sp.csr_matrix((f["Div"].ravel() * Ms, (np.repeat(rows, 3), (3 * f["col"][:, None] + np.arange(3)).ravel())),
                      shape=(N, 3 * N))
    assert abs(D - ofem.divergence(X, T, Ms)).max() < 1e-8
    G = sp.csr_matrix((f["G"].ravel(), ((3 * rows[:, None] + np.arange(3)).ravel(), np.repeat(f["col"], 3))),
                      shape=(3 * N, N))
    assert abs(G - ofem.gradient_op(X, T)).max() < 1e-13
    assert np.abs(f["vol"] - ofem.lumped_volume(X, T)).max() < 1e-12


def test_cluster_tree_bit_exact_vs_reference(spx, golden):
    g = golden("trees.npz")
    cases = {"box20": (20, 20, 5, 2.0), "film30": (30, 30, 2, 2.5), "film48": (48, 48, 2, 2.5)}
    for name, dims in cases.items():
        bd = spx.boundary_data(*omesh.kuhn_box(*dims))
        for leaf in (16, 32, 64):
            perm = spx.cluster_tree_perm(bd["Xb"], leaf)
            assert np.array_equal(perm, g[f"{name}_leaf{leaf}"]), (name, leaf)


def test_gpu_calls_fail_loudly_without_device(spx):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    X, T = omesh.kuhn_box(3, 3, 3, 1.0)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        spx.BoundaryGeometry(X, T)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        spx.DemagFieldLindholmGPU(X, T, 8e5)


def test_invalid_arguments_raise_value_error(spx):
    X, T = omesh.kuhn_box(2, 2, 2, 1.0)
    bad = T.copy()
    bad[0, 0] = X.shape[0] + 5
    with pytest.raises(ValueError, match="out of range"):
        spx.boundary_data(X, bad)
    with pytest.raises(ValueError):
        spx.cluster_tree_perm(np.zeros((0, 3)), 8)
    with pytest.raises(ValueError):
        spx.HMatrixBuildConfig(epsilon=-1.0)
    with pytest.raises(ValueError):
        spx.HMatrixBuildConfig(compressor="svd")


def test_geometry_hash_matches_the_reference_cache(spx):
    """The cache key's geometry hash (sha256 of the boundary points and triangles,
    builder.py:98-103) equals the one the reference wrote into its own cache of the
    14x14x2 film (tests/golden/hcache_film14.npz)."""
    import json
    from spinfemx_b200.hmatrix import geometry_hash
    a = np.load(Path(__file__).resolve().parent / "golden" / "hcache_film14.npz", allow_pickle=False)
    meta = json.loads(str(np.asarray(a["metadata_json"]).item()))
    X, T = omesh.kuhn_box(14, 14, 2, 2.5)
    bd = spx.boundary_data(X, T)
    assert bd["Xb"].shape[0] == meta["Nb"]
    assert geometry_hash(bd["Xb"], bd["tri_lid"]) == meta["geometry_hash"]
    X2 = X.copy()
    X2[:, 2] *= 1.01  # another geometry, another key
    assert geometry_hash(spx.boundary_data(X2, T)["Xb"], bd["tri_lid"]) != meta["geometry_hash"]
