"""Mesh and state IO (spinfemx_b200.io): the reference's example meshes (XDMF with
gzip-compressed HDF5 heavy data, read without h5py), the XDMF writer round trip, and the GPU
pipeline on the example chain mesh against the oracle."""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "fenicsx-micromagnetics_b200"))
sys.path.insert(0, str(ROOT))
from oracle.ref_build import REF_ROOT  # noqa: E402
from spinfemx_b200 import io as sio  # noqa: E402

EXAMPLES = REF_ROOT.parents[1] / "examples"  # the reference checkout's examples, when present
GOLD = ROOT / "tests" / "golden"


def _volumes(X, T):
    P = X[T]
    return np.einsum("ij,ij->i", np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), P[:, 3] - P[:, 0]) / 6.0


@pytest.mark.skipif(not EXAMPLES.exists(), reason="the reference's examples are not present")
@pytest.mark.parametrize("ex,total_volume", [("gpu/FMR/disk", math.pi * 50 ** 2 * 4),
                                             ("cpu/Current-Driven_Vortex/cube", 100 * 100 * 10),
                                             ("cpu/hysteresis_octahedral_nanoparticles/chain", None)])
def test_reference_example_meshes(ex, total_volume):
    import xml.etree.ElementTree as ET
    path = EXAMPLES / f"{ex}.xdmf"
    X, T, attrs = sio.read_xdmf_mesh(path)
    root = ET.parse(path).getroot()
    geo = [int(v) for v in root.find(".//Geometry/DataItem").get("Dimensions").split()]
    top = [int(v) for v in root.find(".//Topology/DataItem").get("Dimensions").split()]
    assert list(X.shape) == geo and list(T.shape) == top
    v = _volumes(X, T)
    assert (v > 0).all()
    used = np.zeros(X.shape[0], bool)
    used[T.ravel()] = True
    assert used.all()
    if total_volume is not None:  # polygonal disk: a little under the circle's area
        assert 0.99 * total_volume < v.sum() <= total_volume * (1 + 1e-12)
    for a in attrs.values():
        assert a.shape[0] == T.shape[0]
    if ex.endswith("chain"):  # the committed fixture is this mesh
        g = np.load(GOLD / "example_chain_mesh.npz")
        assert np.array_equal(g["X"], X) and np.array_equal(g["tets"], T)


def test_xdmf_writer_round_trip(tmp_path):
    from oracle import mesh as omesh
    X, T = omesh.kuhn_box(4, 3, 2, 2.0)
    w = sio.XDMFWriter(tmp_path / "run.xdmf", X, T)
    rng = np.random.default_rng(0)
    states = [rng.normal(size=3 * X.shape[0]) for _ in range(3)]
    for k, m in enumerate(states):
        w.write_function(m, time=1e-12 * k)
    X2, T2, _ = sio.read_xdmf_mesh(tmp_path / "run.xdmf")
    assert np.array_equal(X2, X) and np.array_equal(T2, T)
    series = sio.read_xdmf_series(tmp_path / "run.xdmf", "m")
    assert [t for t, _ in series] == [0.0, 1e-12, 2e-12]
    for (_, a), m in zip(series, states):
        assert np.array_equal(a.ravel(), m)


torch = pytest.importorskip("torch")


@pytest.mark.gpu
def test_chain_mesh_demag_and_llg_vs_oracle():
    """Demag field and a short RK4 trajectory on the reference's unstructured example mesh."""
    import spinfemx_b200 as spx
    from oracle import demag as odemag
    from oracle import llg as ollg
    g = np.load(GOLD / "example_chain_mesh.npz")
    X, T = g["X"], g["tets"]
    N = X.shape[0]
    rng = np.random.default_rng(4)
    m = rng.normal(size=(N, 3)) + np.array([1.0, 0.2, 0.0])
    m = (m / np.linalg.norm(m, axis=1)[:, None]).ravel()
    tight = dict(ksp_rtol_u1=1e-13, ksp_rtol_u2=1e-13, ksp_atol=0.0, ksp_maxit_u1=20000, ksp_maxit_u2=20000)
    o = odemag.DemagOracle(X, T, 4.8e5)
    d = spx.DemagFieldLindholmGPU(X, T, 4.8e5, boundary_backend="dense", **tight)
    H = torch.empty(3 * N, dtype=torch.float64, device="cuda")
    d.compute_vec(torch.as_tensor(m, device="cuda"), H)
    ref = o.compute(m)
    assert np.linalg.norm(H.cpu().numpy() - ref) / np.linalg.norm(ref) < 1e-9
    F = ollg.EffectiveFieldOracle(X, T, 4.8e5, Aex=1.1e-11, alpha=0.5, demag=o)
    mo = m.copy()
    for _ in range(5):
        mo = ollg.rk4_step(F.llg_rhs, mo, 1e-14)
    hef = spx.EffectiveField(X, T, 4.8e5, Aex=1.1e-11, alpha=0.5, use_demag=True,
                             demag_kwargs=dict(boundary_backend="dense", **tight))
    hef.set_state(torch.as_tensor(m, device="cuda"))
    hef.step(1e-14, 5)
    assert np.abs(hef.get_state().cpu().numpy() - mo).max() < 1e-9


def test_checkpoint_round_trip(tmp_path):
    """write_mesh / write_function / read_mesh / read_function (the adios4dolfinx calls of the
    reference's save and restart) round-trip the mesh and several states exactly; a missing
    time or name raises KeyError; values of the wrong length are refused."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "fenicsx-micromagnetics_b200"))
    from spinfemx_b200 import io as sio
    from oracle import mesh as omesh
    X, T = omesh.kuhn_box(3, 2, 2, 2.0)
    rng = np.random.default_rng(0)
    f = tmp_path / "Relax.bp"
    sio.write_mesh(f, X, T)
    m0, m1 = rng.normal(size=3 * X.shape[0]), rng.normal(size=3 * X.shape[0])
    sio.write_function(f, m0, time=0.0, name="m")
    sio.write_function(f, m1, time=1e-12, name="m")
    sio.write_function(f, m1 * 2, time=0.0, name="H")
    Xr, Tr = sio.read_mesh(f)
    assert np.array_equal(Xr, X) and np.array_equal(Tr, T)
    assert np.array_equal(sio.read_function(f, 0.0, "m"), m0)
    assert np.array_equal(sio.read_function(f, 1e-12, "m"), m1)
    assert np.array_equal(sio.read_function(f, 0.0, "H"), m1 * 2)
    sio.write_function(f, m1, time=0.0, name="m")          # replaces the entry at t = 0
    assert np.array_equal(sio.read_function(f, 0.0, "m"), m1)
    with pytest.raises(KeyError):
        sio.read_function(f, 2e-12, "m")
    with pytest.raises(ValueError):
        sio.write_function(f, m0[:-3], time=3.0)
