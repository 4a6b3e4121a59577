"""The LaBonte-BB minimiser's host logic (step length, non-monotone acceptance, back-tracking,
restarts and stopping rules of LaBonteBBMinimizerGPU.minimize) on CPU: its two device calls
are replaced by the oracle's FP64 evaluation of the same quantities, so the loop must retrace
the oracle's restatement (Minimizer_GPU.py:171-845) step for step."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "fenicsx-micromagnetics_b200"))
from oracle import llg as ollg  # noqa: E402
from oracle import mesh as omesh  # noqa: E402
from oracle import minimizer as omin  # noqa: E402

torch = pytest.importorskip("torch")


class _FakeField:
    def __init__(self, m0):
        self.state = torch.as_tensor(np.asarray(m0, dtype=np.float64).ravel())
        self.local_size = self.state.numel()
        self.local_dofs = self.local_size // 3

    def get_state(self, out):
        out.copy_(self.state)

    def set_state(self, m):
        self.state = m.clone()


def _host_loop(F, m0):
    """LaBonteBBMinimizerGPU with its device calls (spx_llg_min_eval / spx_llg_min_trial)
    answered by the oracle on CPU tensors."""
    from spinfemx_b200.minimizer import LaBonteBBMinimizerGPU

    class HostOnly(LaBonteBBMinimizerGPU):
        def __init__(self, hef):  # CPU tensors instead of device buffers
            self.hef = hef
            self.local_size, self.local_dofs = hef.local_size, hef.local_dofs
            z = lambda: torch.zeros(self.local_size, dtype=torch.float64)  # noqa: E731
            self.m, self.m_old, self.m_trial = z(), z(), z()
            self.d, self.d_old, self.d_trial = z(), z(), z()
            self._out = np.zeros(5)
            self.last_energy = self.last_max_grad = None
            self.last_iterations = self.evaluations = self._it = 0

        def _eval(self, normalize):
            m = self.m.numpy().reshape(-1, 3)
            if normalize:
                m = m / np.maximum(np.linalg.norm(m, axis=1), 1e-30)[:, None]
                self.m.copy_(torch.as_tensor(m.ravel()))
            E, d, g = omin.evaluate(F, self.m.numpy())
            self.d.copy_(torch.as_tensor(d))
            self.evaluations += 1
            return E, g

        def _trial(self, alpha):
            mo, do = self.m_old.numpy(), self.d_old.numpy()
            mt = omin.cayley(mo, do, alpha)
            Et, dt, gt = omin.evaluate(F, mt)
            self.m_trial.copy_(torch.as_tensor(mt))
            self.d_trial.copy_(torch.as_tensor(dt))
            s, y = mt - mo, do - dt
            self.evaluations += 1
            return Et, gt, float(s @ y), float(s @ s), float(y @ y)

    hef = _FakeField(np.asarray(m0).reshape(-1, 3) / np.linalg.norm(np.asarray(m0).reshape(-1, 3), axis=1)[:, None])
    mn = HostOnly(hef)
    st = mn.minimize(max_iter=400, tol=1.0)
    return hef.state.numpy(), st


@pytest.mark.parametrize("case", ["uniaxial", "dmi_field"])
def test_host_loop_retraces_the_oracle(case):
    X, T = omesh.kuhn_box(6, 5, 3, 2.0)
    N = X.shape[0]
    rng = np.random.default_rng(2)
    m0 = (np.tile([0.3, 0.1, 1.0], (N, 1)) + 0.2 * rng.normal(size=(N, 3))).ravel()
    if case == "uniaxial":
        F = ollg.EffectiveFieldOracle(X, T, 8e5, Aex=1.3e-11, Ku=4e5, n_ani=np.tile([0.0, 0.0, 1.0], N))
    else:
        F = ollg.EffectiveFieldOracle(X, T, 8e5, Aex=1.3e-11, Ku=2e5, n_ani=np.tile([0.0, 0.0, 1.0], N),
                                      D_int=2e-3, n_int=np.tile([0.0, 0.0, 1.0], N),
                                      H0=np.tile([2e4, 0.0, -1e4], N))
    m_host, st = _host_loop(F, m0)
    m_ref, ref = omin.minimize(F, m0, max_iter=400, tol=1.0)
    assert st["stop_reason"] == ref["stop_reason"]
    assert st["iterations"] == ref["iterations"]
    assert st["energy"] == pytest.approx(ref["energy"], rel=1e-12, abs=0.0)
    assert np.abs(m_host - m_ref).max() < 1e-12
