"""Time-dependent applied field and the adaptive explicit driver against the oracle.

* H_time_func (llg_module_GPU.py:909-956): a uniform pulse and a nodal field evaluated at the
  RK4 stage times; 30 RK4 steps on a small box with dense FP64 demag: max |dm| 1e-9.
* relax_explicit (llg_module_GPU.py:1790-1970): Dormand-Prince 5(4) with the TSAdapt "basic"
  options of the reference, from a random state on the same box: the same number of accepted
  and rejected steps as the oracle, step sizes within 1e-6 relative, final state within 1e-8;
  with the dm/dt stopper (StopByMaxDmdtFDGPU, :314-382) both stop at the same step.
* relax (llg_module_GPU.py:2052-2381): BDF(2) with Newton-GMRES stage solves (block
  preconditioner on and off, with and without a time-dependent field) against
  oracle/implicit.py, with the same bars plus Newton / GMRES iteration totals within 2 %.
"""
import math

import numpy as np
import pytest

from oracle import demag as odemag
from oracle import llg as ollg
from oracle import mesh as omesh

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

MS, AEX, ALPHA = 8e5, 1.3e-11, 0.5
TIGHT = dict(boundary_backend="dense", ksp_rtol_u1=1e-13, ksp_rtol_u2=1e-13, ksp_atol=0.0, ksp_maxit_u1=20000,
             ksp_maxit_u2=20000)


@pytest.fixture(scope="module")
def box():
    X, T = omesh.kuhn_box(10, 8, 3, 2.0)
    return X, T, odemag.DemagOracle(X, T, MS)


def _m0(N, seed):
    rng = np.random.default_rng(seed)
    m = rng.normal(size=(N, 3))
    return (m / np.linalg.norm(m, axis=1)[:, None]).ravel()


def _pulse(t):
    return np.array([0.0, 2e4 * math.cos(2e11 * t), 5e4 * math.sin(3e11 * t)])


@pytest.mark.parametrize("kind", ["uniform", "nodal"])
def test_time_field_rk4_vs_oracle(box, kind):
    import spinfemx_b200 as spx
    X, T, od = box
    N = X.shape[0]
    w = (X[:, 0] - X[:, 0].mean()) / 10.0
    if kind == "uniform":
        def f_prod(t, x):
            return _pulse(t)
        f_or = _pulse
    else:
        def f_or(t):
            return (w[:, None] * _pulse(t)[None, :]).ravel()

        def f_prod(t, x):
            assert x.shape == (N, 3)
            return f_or(t).reshape(N, 3)
    ohef = ollg.EffectiveFieldOracle(X, T, MS, Aex=AEX, alpha=ALPHA, demag=od, H_time=f_or)
    m0 = _m0(N, 3)
    dt, n = 1e-14, 30
    m = m0.copy()
    for k in range(n):
        m = ollg.rk4_step_t(ohef.llg_rhs, k * dt, m, dt)
    hef = spx.EffectiveField(X, T, MS, Aex=AEX, alpha=ALPHA, use_demag=True, demag_kwargs=TIGHT,
                             H_time_func=f_prod)
    hef.set_state(torch.as_tensor(m0, device="cuda"))
    hef.step(dt, n)
    assert abs(hef.current_time - n * dt) < 1e-25
    assert np.abs(hef.get_state().cpu().numpy() - m).max() < 1e-9
    # the field at the current time enters H_eff
    mt = torch.as_tensor(m, device="cuda")
    out = torch.empty_like(mt)
    hef.compute_H_eff_vec(mt, out)
    ref = ohef.h_eff(m, hef.current_time)
    assert np.linalg.norm(out.cpu().numpy() - ref) <= 1e-9 * np.linalg.norm(ref)


@pytest.mark.parametrize("stop,t_final", [(0.0, 2e-11), (1e4, 1e-10)])
def test_relax_explicit_dp5_vs_oracle(box, stop, t_final, tmp_path):
    import spinfemx_b200 as spx
    X, T, od = box
    N = X.shape[0]
    ohef = ollg.EffectiveFieldOracle(X, T, MS, Aex=AEX, alpha=ALPHA, demag=od, H0=np.tile([0.0, 0.0, 3e4], N))
    m0 = _m0(N, 5)
    dt0, tol = 1e-12, 1e-6   # the first attempts are rejected until the step is stable
    mo, so = ollg.relax_explicit(ohef.llg_rhs, m0, 0.0, t_final, dt0, tol, tol, stopping_dmdt=stop, check_every=5)
    llg = spx.LLG_GPU(X, T, MS, alpha=ALPHA)
    llg.add_exchange(AEX)
    llg.add_demag(**TIGHT)
    llg.add_external_field(H0_vec=[0.0, 0.0, 3e4])
    dts = []
    m, _, st = llg.relax_explicit(m0, 0.0, t_final, dt0, ts_rtol=tol, ts_atol=tol, stopping_dmdt=stop,
                                  check_every_stop=5, return_stats=True, output_dir=str(tmp_path),
                                  monitor_fn=lambda step, t, u: dts.append(t))
    assert so["nsteps"] > 100 and so["rejected"] > 5 and st["nsteps"] == so["nsteps"]
    assert st["reason"] == so["reason"] == (2 if stop else 1)
    assert st["rejected"] == so["rejected"]
    assert np.allclose(np.diff([0.0] + dts), so["dts"], rtol=1e-6, atol=0.0)
    assert abs(st["t_end"] - so["t_end"]) <= 1e-6 * so["t_end"]
    assert np.abs(m.cpu().numpy() - mo).max() < 1e-8


# ---------------------------------------------------------------- implicit driver (relax)
# LLG_GPU.relax (llg_module_GPU.py:2052-2381) against oracle/implicit.py: the same BDF(2)
# step sequence (accepted and rejected attempts), step sizes within 1e-6 relative, Newton and
# GMRES iteration totals within 2 %, final state within 1e-8.

@pytest.mark.parametrize("stop,t_final,use_pc", [(0.0, 2e-12, True), (1e3, 1e-9, True), (0.0, 1e-12, False)])
def test_relax_implicit_bdf_vs_oracle(box, stop, t_final, use_pc, tmp_path):
    import spinfemx_b200 as spx
    from oracle import implicit as oimp
    X, T, od = box
    N = X.shape[0]
    ohef = ollg.EffectiveFieldOracle(X, T, MS, Aex=AEX, alpha=ALPHA, demag=od, H0=np.tile([0.0, 0.0, 3e4], N))
    m0 = _m0(N, 7)
    dt0, tol = 1e-13, 1e-6
    mo, so = oimp.relax_implicit(ohef, m0, 0.0, t_final, dt0, tol, tol, stopping_dmdt=stop, check_every=5,
                                 use_pc=use_pc)
    llg = spx.LLG_GPU(X, T, MS, alpha=ALPHA)
    llg.add_exchange(AEX)
    llg.add_demag(**TIGHT)
    llg.add_external_field(H0_vec=[0.0, 0.0, 3e4])
    ts = []
    m, ctx, _, st = llg.relax(m0, 0.0, t_final, dt0, ts_rtol=tol, ts_atol=tol, stopping_dmdt=stop,
                              check_every_stop=5, return_stats=True, save_final_state=False, use_pc_python=use_pc,
                              output_dir=str(tmp_path),
                              monitor_fn=lambda step, t, u: ts.append(t))
    assert so["nsteps"] > 50 and so["rejected"] >= 1
    assert st["nsteps"] == so["nsteps"] and st["rejected"] == so["rejected"]
    assert st["reason"] == so["reason"] == (2 if stop else 1)
    assert st["snes_failures"] == so["snes_failures"]
    assert np.allclose(np.diff([0.0] + ts), so["dts"], rtol=1e-6, atol=0.0)
    assert abs(st["newton_its"] - so["newton_its"]) <= 0.02 * so["newton_its"]
    assert abs(st["linear_its"] - so["linear_its"]) <= 0.02 * so["linear_its"]
    assert ctx.linear_its == st["linear_its"]
    assert np.abs(m.cpu().numpy() - mo).max() < 1e-8


def test_relax_implicit_time_field_vs_oracle(box, tmp_path):
    import spinfemx_b200 as spx
    from oracle import implicit as oimp
    X, T, od = box
    N = X.shape[0]
    ohef = ollg.EffectiveFieldOracle(X, T, MS, Aex=AEX, alpha=ALPHA, demag=od, H_time=_pulse)
    m0 = _m0(N, 8)
    mo, so = oimp.relax_implicit(ohef, m0, 0.0, 1e-12, 1e-13, 1e-6, 1e-6)
    llg = spx.LLG_GPU(X, T, MS, alpha=ALPHA)
    llg.add_exchange(AEX)
    llg.add_demag(**TIGHT)
    llg.add_external_field(H_time_func=lambda t: _pulse(t))
    m, _, _, st = llg.relax(m0, 0.0, 1e-12, 1e-13, return_stats=True, save_final_state=True,
                            output_dir=str(tmp_path))
    assert st["nsteps"] == so["nsteps"] and st["rejected"] == so["rejected"]
    assert np.abs(m.cpu().numpy() - mo).max() < 1e-8
    # restart from the checkpoint: the state read back is the final state bit for bit
    from spinfemx_b200 import io as sio
    assert np.array_equal(sio.read_function(tmp_path / "Relax.bp", time=0.0, name="m"), m.cpu().numpy())
