"""Spin-transfer (Zhang-Li) and spin-orbit torques on the CUDA path against the oracle, whose
per-node formulas are pinned to the reference's own kernel bodies (tests/test_oracle.py)."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import demag as odemag
from oracle import llg as ollg
from oracle import mesh as omesh
from oracle import torques

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
DEV = "cuda"
TIGHT = dict(boundary_backend="dense", ksp_rtol_u1=1e-13, ksp_rtol_u2=1e-13, ksp_atol=0.0, ksp_maxit_u1=20000)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def _t(x):
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=DEV)


@pytest.fixture(scope="module")
def spx():
    import spinfemx_b200 as spx
    return spx


def _setup(with_demag, seed=3):
    X, T = omesh.kuhn_box(9, 7, 3, 2.0)
    N = X.shape[0]
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(N, 3))
    m = (m / np.linalg.norm(m, axis=1)[:, None]).ravel()
    nani = np.tile([0.0, 0.0, 1.0], N)
    nz = np.tile([0.0, 0.0, 1.0], N)
    H0 = np.tile([1e4, -2e4, 3e4], N)
    kw = dict(Ms=8e5, Aex=1.3e-11, Ku=3e5, D_int=2e-3, alpha=0.2)
    demag = odemag.DemagOracle(X, T, kw["Ms"]) if with_demag else None
    o = ollg.EffectiveFieldOracle(X, T, kw["Ms"], Aex=kw["Aex"], Ku=kw["Ku"], n_ani=nani, D_int=kw["D_int"],
                                  n_int=nz, H0=H0, demag=demag, alpha=kw["alpha"])
    return X, T, N, m, nani, nz, H0, kw, o


@pytest.mark.parametrize("with_demag", [False, True])
def test_stt_rhs_jv_pc_vs_oracle(spx, with_demag):
    X, T, N, m, nani, nz, H0, kw, o = _setup(with_demag)
    Jdir = np.tile([0.8, 0.6, 0.0], N) + 0.1 * np.random.default_rng(4).normal(size=3 * N)
    J, P, beta = 2e12, 0.5, 0.04
    hef = spx.EffectiveFieldSTTGPU(X, T, kw["Ms"], Aex=kw["Aex"], Ku=kw["Ku"], n_ani_vec=nani, D_int=kw["D_int"],
                                   n0_int_vec=nz, H0_static=H0, alpha=kw["alpha"], Jmagnitude=J, Jdir_vec=Jdir,
                                   P=P, beta=beta, use_demag=with_demag, demag_kwargs=TIGHT)
    Z = torques.zhang_li_matrix(X, T, Jdir)
    prefZ = torques.pref_zhang(J, P, beta, kw["Ms"], kw["alpha"])
    assert abs(hef.prefZhang - prefZ) <= 1e-15 * abs(prefZ)
    out = torch.empty(3 * N, dtype=torch.float64, device=DEV)
    hef.zhang_li_vec(_t(m), out)
    zm = torques.apply3(Z, m)
    assert rel(out.cpu().numpy(), zm) < 1e-12
    hef.llg_rhs_STT_vec(_t(m), out)
    ref = torques.rhs_stt(m, o.h_eff(m), zm, o.prefactor, kw["alpha"], 1.0, o.stab, prefZ, beta)
    assert rel(out.cpu().numpy(), ref) < (1e-9 if with_demag else 1e-12)
    # Jacobian (demag excluded, like the reference) and the block preconditioner
    hef.update_jac_state_STT(_t(m))
    v = np.random.default_rng(5).normal(size=3 * N)
    hef.jac_vec_times_STT_vec(_t(v), out)
    refj = torques.jv_stt(m, o.h_jac(m), zm, v, o.linear(v), torques.apply3(Z, v), o.prefactor, kw["alpha"], 1.0,
                          o.stab, prefZ, beta)
    assert rel(out.cpu().numpy(), refj) < 1e-11
    ctx = spx.JvContextSTT(hef)
    c1 = hef.gamma / (1 + hef.alpha ** 2)
    c2 = hef.gamma * hef.alpha / (1 + hef.alpha ** 2)
    for shift, inc, absk in ((3e11, True, True), (5e11, False, False)):
        ctx.update_pc_full_fast_gpu(shift, include_stab=inc, use_abs_kappa=absk)
        y = torch.empty_like(out)
        ctx.apply(None, _t(v), y)
        inv = torques.pc_build_stt(m, o.h_jac(m), zm, o.diagK, shift, c1, c2, ctx.c3, ctx.c4, o.stab,
                                   include_stab=inc, use_abs_kappa=absk)
        assert rel(y.cpu().numpy(), np.einsum("nij,nj->ni", inv, v.reshape(-1, 3)).ravel()) < 1e-11


@pytest.mark.parametrize("with_demag", [False, True])
def test_sot_rhs_jv_pc_vs_oracle(spx, with_demag):
    X, T, N, m, nani, nz, H0, kw, o = _setup(with_demag, seed=7)
    pol = np.tile([0.0, 1.0, 0.0], N) + 0.2 * np.random.default_rng(8).normal(size=3 * N)
    Hdl, Hfl = 4e4, -1.5e4
    hef = spx.EffectiveFieldSOTGPU(X, T, kw["Ms"], Aex=kw["Aex"], Ku=kw["Ku"], n_ani_vec=nani, D_int=kw["D_int"],
                                   n0_int_vec=nz, H0_static=H0, alpha=kw["alpha"], H_dl=Hdl, H_fl=Hfl,
                                   polarization_vec=pol, use_demag=with_demag, demag_kwargs=TIGHT)
    p = pol.reshape(-1, 3) / np.linalg.norm(pol.reshape(-1, 3), axis=1)[:, None]
    c_fl, c_dl = torques.sot_coefficients(hef.gamma, hef.alpha, Hdl, Hfl)
    assert abs(hef.c_fl - c_fl) <= 1e-15 * abs(c_fl) and abs(hef.c_dl - c_dl) <= 1e-15 * abs(c_dl)
    out = torch.empty(3 * N, dtype=torch.float64, device=DEV)
    hef.llg_rhs_SOT_vec(_t(m), out)
    ref = torques.rhs_sot(m, o.h_eff(m), p, o.prefactor, kw["alpha"], 1.0, o.stab, c_fl, c_dl)
    assert rel(out.cpu().numpy(), ref) < (1e-9 if with_demag else 1e-12)
    hef.update_jac_state_SOT(_t(m))
    v = np.random.default_rng(9).normal(size=3 * N)
    hef.jac_vec_times_SOT_vec(_t(v), out)
    refj = torques.jv_sot(m, o.h_jac(m), p, v, o.linear(v), o.prefactor, kw["alpha"], 1.0, o.stab, c_fl, c_dl)
    assert rel(out.cpu().numpy(), refj) < 1e-11
    ctx = spx.JvContextSOT(hef)
    for shift, absd in ((3e11, False), (5e11, True)):
        ctx.update_pc_full_fast_gpu(shift, use_abs_diag=absd)
        y = torch.empty_like(out)
        ctx.apply(None, _t(v), y)
        inv = torques.pc_build_sot(m, o.h_jac(m), p, o.diagK, shift, o.prefactor, kw["alpha"], 1.0, o.stab, c_fl,
                                   c_dl, use_abs_diag=absd)
        assert rel(y.cpu().numpy(), np.einsum("nij,nj->ni", inv, v.reshape(-1, 3)).ravel()) < 1e-11
    # set_sot changes the coefficients (and the polarisation)
    hef.set_sot(H_dl=1e4, H_fl=2e4, polarization_vec=[1.0, 0.0, 0.0])
    hef.llg_rhs_SOT_vec(_t(m), out)
    c_fl, c_dl = torques.sot_coefficients(hef.gamma, hef.alpha, 1e4, 2e4)
    ref = torques.rhs_sot(m, o.h_eff(m), np.tile([1.0, 0.0, 0.0], N), o.prefactor, kw["alpha"], 1.0, o.stab,
                          c_fl, c_dl)
    assert rel(out.cpu().numpy(), ref) < (1e-9 if with_demag else 1e-12)


def test_stt_rk4_trajectory_vs_oracle(spx):
    X, T, N, m, nani, nz, H0, kw, o = _setup(True, seed=11)
    Jdir = np.tile([1.0, 0.0, 0.0], N)
    J, P, beta = 5e12, 0.7, 0.02
    hef = spx.EffectiveFieldSTTGPU(X, T, kw["Ms"], Aex=kw["Aex"], Ku=kw["Ku"], n_ani_vec=nani, D_int=kw["D_int"],
                                   n0_int_vec=nz, H0_static=H0, alpha=kw["alpha"], Jmagnitude=J, Jdir_vec=Jdir,
                                   P=P, beta=beta, use_demag=True, demag_kwargs=TIGHT)
    Z = torques.zhang_li_matrix(X, T, Jdir)
    prefZ = torques.pref_zhang(J, P, beta, kw["Ms"], kw["alpha"])

    def f(mm):
        return torques.rhs_stt(mm, o.h_eff(mm), torques.apply3(Z, mm), o.prefactor, kw["alpha"], 1.0, o.stab,
                               prefZ, beta)
    mo = m.copy()
    for _ in range(8):
        mo = ollg.rk4_step(f, mo, 2e-14)
    hef.set_state(_t(m))
    hef.step(2e-14, 8)
    assert np.abs(hef.get_state().cpu().numpy() - mo).max() < 1e-9
