"""The host side of relax_explicit on CPU: LLG_GPU's step-size loop with its device calls
(spx_llg_rk_attempt / _rk_accept) answered by the oracle's Dormand-Prince attempt retraces
the oracle's relax_explicit step for step (accepted and rejected attempts, step sizes)."""
import numpy as np

from oracle import llg as ollg
from oracle import mesh as omesh


class OracleStepper:
    """Stands in for EffectiveField's device calls."""

    def __init__(self, f, m0):
        self.f, self.m, self.current_time, self.N = f, m0.copy(), 0.0, m0.size // 3
        self.k1 = None
        self.cand = None

    def rk_attempt(self, dt, rtol, atol, reuse_fsal=True):
        y5, en, k7 = ollg.dp5_attempt(self.f, self.current_time, self.m, dt, rtol, atol,
                                      self.k1 if reuse_fsal else None)
        self.cand = (y5, k7)
        return en

    def rk_accept(self, dt):
        self.m, self.k1 = self.cand
        self.current_time += dt

    def get_state(self):
        return self.m


def test_relax_explicit_host_loop_matches_oracle(tmp_path):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "fenicsx-micromagnetics_b200"))
    from spinfemx_b200.llg import LLG_GPU
    X, T = omesh.kuhn_box(6, 5, 3, 2.0)
    N = X.shape[0]
    ohef = ollg.EffectiveFieldOracle(X, T, 8e5, Aex=1.3e-11, alpha=0.5, H0=np.tile([0.0, 0.0, 3e4], N))
    rng = np.random.default_rng(2)
    m0 = rng.normal(size=(N, 3))
    m0 = (m0 / np.linalg.norm(m0, axis=1)[:, None]).ravel()
    mo, so = ollg.relax_explicit(ohef.llg_rhs, m0, 0.0, 1e-11, 1e-12, 1e-6, 1e-6)
    llg = LLG_GPU(X, T, 8e5, alpha=0.5)
    llg.hef = OracleStepper(ohef.llg_rhs, m0)
    ts = []
    m, _, st = llg.relax_explicit(None, 0.0, 1e-11, 1e-12, ts_rtol=1e-6, ts_atol=1e-6, return_stats=True,
                                  output_dir=str(tmp_path), monitor_fn=lambda step, t, u: ts.append(t))
    assert so["rejected"] > 0 and st["rejected"] == so["rejected"]
    assert st["nsteps"] == so["nsteps"] and st["reason"] == so["reason"] == 1
    assert np.allclose(np.diff([0.0] + ts), so["dts"], rtol=1e-12, atol=0.0)
    assert np.array_equal(m, mo)


class OracleBDF:
    """Stands in for EffectiveField's implicit device calls (spx_llg_bdf_attempt / _accept)."""

    def __init__(self, hef, m0):
        from oracle import implicit as oimp
        self.b = oimp.BDFOracle(hef, m0)
        self.current_time = 0.0

    def bdf_reset(self):
        self.b.reset()

    def bdf_attempt(self, dt, o):
        self.b.rtol, self.b.atol = o.rtol, o.atol
        self.b.current_time = self.current_time
        r = self.b.attempt(dt)
        return dict(r, newton_its=0, linear_its=0, fevals=0)

    def bdf_accept(self, dt):
        self.b.accept()
        self.current_time += dt

    def get_state(self):
        return self.b.m


def test_relax_implicit_host_loop_matches_oracle(tmp_path):
    """LLG_GPU.relax's step-size loop (TSAdapt basic with the implicit options, failed-solve
    scaling, reject limit) with its device calls answered by the oracle's BDF attempts retraces
    oracle.implicit.relax_implicit step for step."""
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "fenicsx-micromagnetics_b200"))
    from oracle import implicit as oimp
    from spinfemx_b200.llg import LLG_GPU
    X, T = omesh.kuhn_box(5, 4, 3, 2.0)
    N = X.shape[0]
    ohef = ollg.EffectiveFieldOracle(X, T, 8e5, Aex=1.3e-11, alpha=0.5, H0=np.tile([0.0, 0.0, 3e4], N))
    rng = np.random.default_rng(4)
    m0 = rng.normal(size=(N, 3))
    m0 = (m0 / np.linalg.norm(m0, axis=1)[:, None]).ravel()
    mo, so = oimp.relax_implicit(ohef, m0, 0.0, 1e-12, 1e-13, 1e-6, 1e-6)
    llg = LLG_GPU(X, T, 8e5, alpha=0.5)
    llg.hef = OracleBDF(ohef, m0)
    ts = []
    m, ctx, _, st = llg.relax(None, 0.0, 1e-12, 1e-13, ts_rtol=1e-6, ts_atol=1e-6, return_stats=True,
                              save_final_state=True, output_dir=str(tmp_path),
                              monitor_fn=lambda step, t, u: ts.append(t))
    assert so["rejected"] > 0 and st["rejected"] == so["rejected"]
    assert st["nsteps"] == so["nsteps"] and st["reason"] == so["reason"] == 1
    assert np.allclose(np.diff([0.0] + ts), so["dts"], rtol=1e-12, atol=0.0)
    assert np.array_equal(m, mo)
    # the restart checkpoint and the XDMF of the final state
    from spinfemx_b200 import io as sio
    Xr, Tr = sio.read_mesh(tmp_path / "Relax.bp")
    assert np.array_equal(Xr, X) and np.array_equal(Tr, T)
    assert np.array_equal(sio.read_function(tmp_path / "Relax.bp", time=0.0, name="m"), m)
    (t_last, mx), = sio.read_xdmf_series(tmp_path / "Relax.xdmf", "m")
    assert t_last == st["t_end"] and np.array_equal(mx.ravel(), m)
