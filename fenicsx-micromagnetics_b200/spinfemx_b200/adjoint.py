"""Differentiable LLG trajectories (no counterpart in the reference).

``llg_trajectory`` integrates ``nsteps`` classic RK4 steps with an ``EffectiveField`` and is
a ``torch.autograd.Function``: its backward pass is the hand-written discrete adjoint of the
integrator (``spx_llg_step_vjp``, one reverse RK4 sweep per step with the demag adjoint
D^T inside), not autograd of a traced graph.  Every ``checkpoint_every``-th state is kept
during the forward pass; the backward pass recomputes each segment's states from its
checkpoint and sweeps it in reverse.  Gradients flow to the initial magnetisation, the
nodal Ku map (J/m^3) and the uniform applied field H0 (A/m); compose with torch for other
parametrisations (a per-cell map averaged to the nodes, B = mu0 H0, ...).

``trajectory_tangent`` is the forward-mode counterpart (``spx_llg_step_jvp``): the
directional derivative of m(T) along (dm0, dKu, dH0).
"""
from __future__ import annotations

import numpy as np


def _device(hef):
    """Device of the field object's state (the GPU for the library's field objects)."""
    return getattr(hef, "device", "cuda")


def _dev_f64(x, n, name, device="cuda"):
    import torch
    t = torch.as_tensor(x, dtype=torch.float64, device=device).contiguous().reshape(-1)
    if t.numel() != n:
        raise ValueError(f"{name} must have {n} entries")
    return t


def _make_function():
    import torch

    class LLGTrajectory(torch.autograd.Function):
        @staticmethod
        def forward(ctx, m0, Ku, H0, hef, dt, nsteps, every):
            if nsteps < 0 or every < 1 or dt <= 0.0:
                raise ValueError("nsteps >= 0, checkpoint_every >= 1 and dt > 0 are required")
            _apply_params(hef, Ku, H0)
            m = _dev_f64(m0.detach(), hef.local_size, "m0", _device(hef))
            hef.set_state(m)
            ckpts = []
            n = 0
            while n < nsteps:
                ckpts.append(hef.get_state().clone())
                k = min(every, nsteps - n)
                hef.step(dt, k)
                n += k
            mT = hef.get_state()
            ctx.hef, ctx.dt, ctx.nsteps, ctx.every = hef, float(dt), int(nsteps), int(every)
            ctx.ckpts = ckpts
            ctx.params = (None if Ku is None else Ku.detach().clone(), None if H0 is None else H0.detach().clone())
            ctx.want = (Ku is not None, H0 is not None)
            ctx.H0_device = None if H0 is None else H0.device
            return mT

        @staticmethod
        def backward(ctx, gT):
            hef, dt, every = ctx.hef, ctx.dt, ctx.every
            Ku, H0 = ctx.params
            _apply_params(hef, Ku, H0)
            lam = gT.detach().to(torch.float64).contiguous().clone()
            dev = _device(hef)
            gKu = torch.zeros(hef.N, dtype=torch.float64, device=dev) if ctx.want[0] else None
            gH0 = torch.zeros(3, dtype=torch.float64, device=dev) if ctx.want[1] else None
            for seg in range(len(ctx.ckpts) - 1, -1, -1):
                n0 = seg * every
                k = min(every, ctx.nsteps - n0)
                states = [ctx.ckpts[seg]]
                hef.set_state(ctx.ckpts[seg])
                for _ in range(k - 1):
                    hef.step(dt, 1)
                    states.append(hef.get_state().clone())
                for j in range(k - 1, -1, -1):
                    hef.step_vjp(states[j], dt, lam, lam, gKu, gH0)
            gH0o = None if gH0 is None else gH0.to(ctx.H0_device)
            return lam, gKu, gH0o, None, None, None, None

    return LLGTrajectory


_FN = None


def _apply_params(hef, Ku, H0):
    import torch
    if Ku is not None:
        hef.set_anisotropy_map(Ku.detach().to("cpu", dtype=torch.float64).numpy())
    if H0 is not None:
        h = H0.detach().to("cpu", dtype=torch.float64).numpy().reshape(3)
        hef.set_uniform_field(float(h[0]), float(h[1]), float(h[2]))


def llg_trajectory(hef, m0, dt, nsteps, Ku=None, H0=None, checkpoint_every=20):
    """m(T) after ``nsteps`` RK4 steps of size ``dt`` from ``m0``, differentiable in m0, Ku
    (nodal map, length N, needs an anisotropy axis) and H0 (uniform field, length 3, A/m)."""
    global _FN
    if _FN is None:
        _FN = _make_function()
    return _FN.apply(m0, Ku, H0, hef, float(dt), int(nsteps), int(checkpoint_every))


def trajectory_tangent(hef, m0, dt, nsteps, dm0=None, dKu=None, dH0=None, Ku=None, H0=None):
    """(m(T), dm(T)): the trajectory and its directional derivative along (dm0, dKu, dH0)."""
    import torch
    _apply_params(hef, None if Ku is None else torch.as_tensor(Ku),
                  None if H0 is None else torch.as_tensor(H0))
    n3 = hef.local_size
    m = _dev_f64(m0, n3, "m0").clone()
    dm = torch.zeros_like(m) if dm0 is None else _dev_f64(dm0, n3, "dm0").clone()
    dku = None if dKu is None else _dev_f64(dKu, hef.N, "dKu")
    dh0 = None if dH0 is None else np.asarray(dH0, dtype=np.float64).reshape(3)
    m2, dm2 = torch.empty_like(m), torch.empty_like(m)
    for _ in range(int(nsteps)):
        hef.step_jvp(m, dm, dt, m2, dm2, dku, dh0)
        m, m2 = m2, m
        dm, dm2 = dm2, dm
    return m, dm


__all__ = ["llg_trajectory", "trajectory_tangent"]
