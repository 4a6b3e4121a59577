"""The checkpointing schedule of ``llg_trajectory`` (host logic of the hand-written adjoint) on
CPU: a field object whose step and step-VJP are a small nonlinear map stands in for the
library's, and the gradients in m0, Ku and H0 must equal torch autograd of the same map for
every checkpoint interval (segments of one step, ragged last segments, one segment)."""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "fenicsx-micromagnetics_b200"))
torch = pytest.importorskip("torch")


class _MapField:
    """m <- m + dt (tanh(W m) + (Ku per node) m + H0 per node), with its exact VJP."""

    device = "cpu"

    def __init__(self, N, seed=0):
        g = torch.Generator().manual_seed(seed)
        self.N, self.local_size = N, 3 * N
        self.W = torch.randn(3 * N, 3 * N, generator=g, dtype=torch.float64) / (3 * N) ** 0.5
        self.Ku = torch.zeros(N, dtype=torch.float64)
        self.H0 = torch.zeros(3, dtype=torch.float64)
        self.m = torch.zeros(3 * N, dtype=torch.float64)
        self.steps = 0

    def set_anisotropy_map(self, ku):
        self.Ku = torch.as_tensor(np.asarray(ku, dtype=np.float64))

    def set_uniform_field(self, hx, hy, hz):
        self.H0 = torch.tensor([hx, hy, hz], dtype=torch.float64)

    def set_state(self, m):
        self.m = m.detach().clone()

    def get_state(self):
        return self.m.clone()

    @staticmethod
    def f(m, W, Ku, H0, dt):
        return m + dt * (torch.tanh(W @ m) + Ku.repeat_interleave(3) * m + H0.repeat(m.numel() // 3))

    def step(self, dt, k):
        for _ in range(k):
            self.m = self.f(self.m, self.W, self.Ku, self.H0, dt)
            self.steps += 1

    def step_vjp(self, m, dt, lam_in, lam_out, gKu, gH0):
        t = torch.tanh(self.W @ m)
        lam = lam_in.clone()
        out = lam + dt * (self.W.T @ (lam * (1.0 - t * t)) + self.Ku.repeat_interleave(3) * lam)
        if gKu is not None:
            gKu += dt * (lam * m).reshape(-1, 3).sum(1)
        if gH0 is not None:
            gH0 += dt * lam.reshape(-1, 3).sum(0)
        lam_out.copy_(out)


@pytest.mark.parametrize("every", [1, 3, 4, 10, 25])
def test_checkpointed_adjoint_equals_autograd(every):
    from spinfemx_b200.adjoint import llg_trajectory
    N, nsteps, dt = 6, 10, 0.05
    g = torch.Generator().manual_seed(3)
    m0 = torch.randn(3 * N, generator=g, dtype=torch.float64)
    Ku = torch.rand(N, generator=g, dtype=torch.float64)
    H0 = torch.randn(3, generator=g, dtype=torch.float64)
    w = torch.randn(3 * N, generator=g, dtype=torch.float64)
    hef = _MapField(N)
    a = [t.clone().requires_grad_(True) for t in (m0, Ku, H0)]
    mT = llg_trajectory(hef, a[0], dt, nsteps, Ku=a[1], H0=a[2], checkpoint_every=every)
    (mT * w).sum().backward()
    # forward steps plus the recomputation inside each segment (all but its last step)
    nseg = -(-nsteps // every)
    assert hef.steps == nsteps + (nsteps - nseg)
    b = [t.clone().requires_grad_(True) for t in (m0, Ku, H0)]
    m = b[0]
    for _ in range(nsteps):
        m = _MapField.f(m, hef.W, b[1], b[2], dt)
    assert torch.allclose(mT.detach(), m.detach(), rtol=0, atol=1e-14)
    (m * w).sum().backward()
    for x, y in zip(a, b):
        assert torch.allclose(x.grad, y.grad, rtol=1e-12, atol=1e-14)


def test_invalid_schedule_rejected():
    from spinfemx_b200.adjoint import llg_trajectory
    hef = _MapField(2)
    m0 = torch.zeros(6, dtype=torch.float64)
    with pytest.raises(ValueError):
        llg_trajectory(hef, m0, 0.1, 4, checkpoint_every=0)
    with pytest.raises(ValueError):
        llg_trajectory(hef, m0, -0.1, 4)
