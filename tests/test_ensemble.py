"""Ensembles of independent samples (one disjoint-union mesh, block-diagonal boundary
operator): each sample's demag field and trajectory must equal those of the sample run on
its own, and the oracle's for a dense sample."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import demag as odemag
from oracle import llg as ollg
from oracle import mesh as omesh

BOXES = [(6, 5, 2), (9, 7, 3), (12, 10, 2)]  # Nb 106, 224, 330
DENSE_MAX = 200  # sample 0 dense, samples 1 and 2 H-matrices (merged into one)
MAT = dict(Ms=1.1e6, Aex=1.6e-11, Ku=8e5, D_int=3e-3, alpha=0.3)
TIGHT = dict(ksp_rtol_u1=1e-12, ksp_rtol_u2=1e-12, ksp_atol=0.0, ksp_maxit_u1=20000, ksp_maxit_u2=20000)
HM = dict(hmatrix_epsilon=1e-7, hmatrix_leaf_size=16)


def _meshes():
    return [omesh.kuhn_box(nx, ny, nz, 2.0) for nx, ny, nz in BOXES]


def _m0(N, seed):
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(N, 3))
    return (m / np.linalg.norm(m, axis=1)[:, None]).ravel()


def test_ensemble_mesh_union():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "fenicsx-micromagnetics_b200"))
    from spinfemx_b200.ensemble import ensemble_mesh
    ms = _meshes()
    X, T, off = ensemble_mesh(ms)
    assert off.tolist() == [0] + np.cumsum([m[0].shape[0] for m in ms]).tolist()
    assert T.shape[0] == sum(m[1].shape[0] for m in ms)
    for k, (Xs, Ts) in enumerate(ms):
        assert np.array_equal(X[off[k]:off[k + 1]], Xs)
        sel = T[(T[:, 0] >= off[k]) & (T[:, 0] < off[k + 1])]
        assert np.array_equal(sel - off[k], Ts)


torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def spx():
    import spinfemx_b200 as spx
    return spx


def _t(x):
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device="cuda")


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_ensemble_demag_equals_per_sample(spx, precision):
    ms = _meshes()
    X, T, off = spx.ensemble_mesh(ms)
    kw = dict(precision=precision, **TIGHT, **HM)
    d = spx.DemagFieldLindholmGPU(X, T, MAT["Ms"], boundary_backend="ensemble", sample_offsets=off,
                                  dense_max_nb=DENSE_MAX, **kw)
    m = np.concatenate([_m0(Xs.shape[0], 10 + k) for k, (Xs, _) in enumerate(ms)])
    H = torch.empty(3 * X.shape[0], dtype=torch.float64, device="cuda")
    d.compute_vec(_t(m), H)
    H = H.cpu().numpy()
    for k, (Xs, Ts) in enumerate(ms):
        ds = spx.DemagFieldLindholmGPU(Xs, Ts, MAT["Ms"], boundary_backend="dense" if k == 0 else "hmatrix", **kw)
        Hs = torch.empty(3 * Xs.shape[0], dtype=torch.float64, device="cuda")
        ds.compute_vec(_t(m[3 * off[k]:3 * off[k + 1]]), Hs)
        Hs = Hs.cpu().numpy()
        err = np.linalg.norm(H[3 * off[k]:3 * off[k + 1]] - Hs) / np.linalg.norm(Hs)
        assert err < (1e-9 if precision == "f64" else 2e-6), (k, err)
        if k == 0:
            ref = odemag.DemagOracle(Xs, Ts, MAT["Ms"]).compute(m[3 * off[k]:3 * off[k + 1]])
            assert np.linalg.norm(Hs - ref) / np.linalg.norm(ref) < (1e-9 if precision == "f64" else 2e-6)


@pytest.mark.gpu
def test_ensemble_trajectory_equals_per_sample(spx):
    ms = _meshes()
    Bz = [0.3, -0.2, 0.45]
    mu0 = 4e-7 * np.pi
    dk = dict(precision="f64", **TIGHT, **HM)
    ens = spx.LLGEnsemble(ms, MAT["Ms"], Aex=MAT["Aex"], Ku=MAT["Ku"], D_int=MAT["D_int"], alpha=MAT["alpha"],
                          H0=[[0.0, 0.0, b / mu0] for b in Bz], dense_max_nb=DENSE_MAX, precision="f64",
                          demag_kwargs=dk)
    m0 = [_m0(Xs.shape[0], 20 + k) for k, (Xs, _) in enumerate(ms)]
    ens.set_state(m0)
    nsteps, dt = 10, 2e-14
    ens.step(dt, nsteps)
    mE = ens.split(ens.get_state().cpu().numpy())
    for k, (Xs, Ts) in enumerate(ms):
        N = Xs.shape[0]
        kw = dict(dk, boundary_backend="dense" if k == 0 else "hmatrix")
        hef = spx.EffectiveField(Xs, Ts, MAT["Ms"], Aex=MAT["Aex"], Ku=MAT["Ku"], n_ani_vec=[0.0, 0.0, 1.0],
                                 D_int=MAT["D_int"], n0_int_vec=[0.0, 0.0, 1.0], alpha=MAT["alpha"],
                                 H0_static=[0.0, 0.0, Bz[k] / mu0], use_demag=True, demag_kwargs=kw)
        hef.set_state(_t(m0[k]))
        hef.step(dt, nsteps)
        ms_ = hef.get_state().cpu().numpy()
        assert np.abs(mE[k] - ms_).max() < 1e-10, k
        if k == 0:  # and the FP64 oracle for the dense sample
            o = ollg.EffectiveFieldOracle(Xs, Ts, MAT["Ms"], Aex=MAT["Aex"], Ku=MAT["Ku"],
                                          n_ani=np.tile([0.0, 0.0, 1.0], N), D_int=MAT["D_int"],
                                          n_int=np.tile([0.0, 0.0, 1.0], N), H0=np.tile([0.0, 0.0, Bz[k] / mu0], N),
                                          demag=odemag.DemagOracle(Xs, Ts, MAT["Ms"]), alpha=MAT["alpha"])
            mo = m0[k].copy()
            for _ in range(nsteps):
                mo = ollg.rk4_step(o.llg_rhs, mo, dt)
            assert np.abs(mE[k] - mo).max() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_graph_replayed_steps_equal_ordinary_steps(spx, precision):
    """RK4 steps replayed from CUDA graphs (with per-stage extrapolated Krylov starts) give the
    ordinary steps' results exactly; a field change recaptures."""
    ms = _meshes()
    mu0 = 4e-7 * np.pi
    dk = dict(precision=precision, ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10, warm_start="extrapolate_corrected", **HM)
    runs = []
    for graph in (False, True):
        ens = spx.LLGEnsemble(ms, MAT["Ms"], Aex=MAT["Aex"], Ku=MAT["Ku"], D_int=MAT["D_int"], alpha=MAT["alpha"],
                              H0=[[0.0, 0.0, b / mu0] for b in (0.3, -0.2, 0.45)], dense_max_nb=DENSE_MAX,
                              precision=precision, demag_kwargs=dk)
        ens.hef.set_graph(graph)
        ens.set_state([_m0(Xs.shape[0], 30 + k) for k, (Xs, _) in enumerate(ms)])
        ens.step(2e-14, 13)  # 8 replays: not a multiple of the ring period before the recapture
        a = ens.get_state().cpu().numpy()
        ens.hef.set_uniform_field(0.0, 1e5, 0.0)
        ens.step(2e-14, 7)
        runs.append((a, ens.get_state().cpu().numpy(), ens.hef.graph_stats()))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    # five ordinary steps fill the five-deep extrapolation rings, then every step is replayed
    assert runs[1][2]["replayed_steps"] == 8 + 7 and runs[1][2]["active"]
    assert runs[0][2]["replayed_steps"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision,R", [("f64", 2), ("mixed", 4), ("mixed", 8)])
def test_batch_of_one_mesh_shares_the_u1_hierarchy(spx, precision, R):
    """R films of one mesh: the u1 system is one block repeated on the diagonal, solved with the
    block's matrix and AMG hierarchy stored once; every film's field equals the film run alone."""
    Xs, Ts = omesh.kuhn_box(40, 40, 2, 2.5)  # 5,043 nodes per film
    X, T, off = spx.ensemble_mesh([(Xs, Ts)] * R)
    kw = dict(precision=precision, ksp_rtol_u1=1e-12, ksp_rtol_u2=1e-12, ksp_atol=0.0, ksp_maxit_u1=20000,
              ksp_maxit_u2=20000, hmatrix_epsilon=1e-7, hmatrix_leaf_size=32)
    d = spx.DemagFieldLindholmGPU(X, T, MAT["Ms"], boundary_backend="ensemble", sample_offsets=off, dense_max_nb=0,
                                  **kw)
    assert d.amg_levels()[0]["rows"] == Xs.shape[0]  # the hierarchy of one film
    m = np.concatenate([_m0(Xs.shape[0], 40 + k) for k in range(R)])
    H = torch.empty(3 * X.shape[0], dtype=torch.float64, device="cuda")
    d.compute_vec(_t(m), H)
    d.compute_vec(_t(m), H)  # a second (warm) solve
    H = H.cpu().numpy()
    ds = spx.DemagFieldLindholmGPU(Xs, Ts, MAT["Ms"], boundary_backend="hmatrix", **kw)
    Hs = torch.empty(3 * Xs.shape[0], dtype=torch.float64, device="cuda")
    for k in range(R):
        ds.compute_vec(_t(m[3 * off[k]:3 * off[k + 1]]), Hs)
        ref = Hs.cpu().numpy()
        err = np.linalg.norm(H[3 * off[k]:3 * off[k + 1]] - ref) / np.linalg.norm(ref)
        assert err < (1e-9 if precision == "f64" else 2e-6), (k, err)
