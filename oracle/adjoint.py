"""Adjoint and tangent products of the demag map and of the LLG RK4 step (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

The reference has no adjoint: its LLG path (gpu/solvers/llg_module_GPU.py) evaluates the
right-hand side (:100-122, :1261-1285) and a Jacobian-vector product without the demag term
(:125-164) for its Newton-Krylov solver.  These functions differentiate the oracle's own
forward pipeline exactly, with explicit transposes of the scipy operators, so that the
CUDA adjoint can be checked against an independent restatement, and they give the
trajectory gradient whose central finite differences pin it:

* ``demag_transpose``  D^T w for D: m -> H of ``DemagOracle.compute``
  (Demag_Lindholm_GPU.py:569-670 restated in oracle/demag.py);
* ``rhs_vjp`` / ``rhs_jvp``  J^T w and J v of ``llg.rhs`` with H = ``h_eff(m)``, plus the
  derivatives with respect to a nodal Ku map and the uniform applied field H0;
* ``step_vjp`` / ``step_jvp`` / ``trajectory_grad``  classic RK4 (``llg.rk4_step``).
"""
from __future__ import annotations

import numpy as np

from . import fem
from .demag import MU0


def demag_solve_u1(D, b):
    """Pi A^+ Pi b (the u1 solve of DemagOracle.solve_u1 for a given right-hand side)."""
    b = b - b.mean()
    u = np.zeros(D.N)
    u[1:] = D._lu1.solve(b[1:])
    return u - u.mean()


def demag_transpose(D, w, B_T_apply=None):
    """D^T w:  Div^T Pi A^+ Pi (psi + E^T B^T (psi_B - A_BI A_II^-1 psi_I)),  psi = (G/V)^T w."""
    w = np.asarray(w, dtype=np.float64).reshape(-1, 3)
    psi = D.G.T @ (w / D.vol[:, None]).ravel()
    if D._lu2 is not None:
        xI = D._lu2.solve(psi[D.interior])
        gbar = psi[D.bverts] - D.A_IB.T @ xI
    else:
        gbar = psi[D.bverts].copy()
    if B_T_apply is None:
        yb = D.B.T @ gbar
    else:
        yb = B_T_apply(gbar)
    u1bar = psi.copy()
    u1bar[D.bverts] += yb
    return D.Div.T @ demag_solve_u1(D, u1bar)


def _cross(a, b):
    return np.cross(a, b)


def _parts(F, m):
    m3 = np.asarray(m, dtype=np.float64).reshape(-1, 3)
    H3 = F.h_eff(np.asarray(m, dtype=np.float64).ravel()).reshape(-1, 3)
    return m3, H3


def lin_transpose(F, u, B_T_apply=None):
    """L^T u for the linear field L m = K_lin m + anisotropy + demag."""
    out = F.K_lin.T @ u
    if F.has_ani:
        out = out + fem.anisotropy_field(u, F.n_ani, F.Ku, F.Ms)
    if F.demag is not None:
        out = out + demag_transpose(F.demag, u, B_T_apply)
    return out


def lin_apply(F, v):
    H = F.linear(v)
    if F.demag is not None:
        H = H + F.demag.compute(v)
    return H


def rhs_vjp(F, m, w, B_T_apply=None):
    """(J^T w, dL/dKu [N], dL/dH0 [3]) for f(m) = llg.rhs(m, h_eff(m))."""
    m3, H3 = _parts(F, m)
    w3 = np.asarray(w, dtype=np.float64).reshape(-1, 3)
    pref, al, p, st = F.prefactor, F.alpha, F.do_precess, F.stab
    mm = np.sum(m3 * m3, axis=1)[:, None]
    mw = np.sum(m3 * w3, axis=1)[:, None]
    wm = _cross(w3, m3)
    a = pref * (p * _cross(H3, w3) + al * (_cross(_cross(m3, H3), w3) + _cross(H3, wm))) \
        + st * (1.0 - mm) * w3 - 2.0 * st * mw * m3
    u = pref * (p * wm + al * _cross(wm, m3))
    a = a.ravel() + lin_transpose(F, u.ravel(), B_T_apply)
    gH0 = u.sum(axis=0)
    gKu = np.zeros(F.N)
    if F.has_ani:
        gKu = 2.0 / (MU0 * F.Ms) * np.sum(m3 * F.n_ani, axis=1) * np.sum(F.n_ani * u, axis=1)
    return a, gKu, gH0


def rhs_jvp(F, m, v, dKu=None, dH0=None):
    """J v + df/dKu dKu + df/dH0 dH0."""
    m3, H3 = _parts(F, m)
    v3 = np.asarray(v, dtype=np.float64).reshape(-1, 3)
    g3 = lin_apply(F, np.asarray(v, dtype=np.float64).ravel()).reshape(-1, 3)
    if dKu is not None and F.has_ani:
        g3 = g3 + (2.0 / (MU0 * F.Ms) * np.asarray(dKu) * np.sum(m3 * F.n_ani, axis=1))[:, None] * F.n_ani
    if dH0 is not None:
        g3 = g3 + np.asarray(dH0, dtype=np.float64).reshape(1, 3)
    pref, al, p, st = F.prefactor, F.alpha, F.do_precess, F.stab
    mm = np.sum(m3 * m3, axis=1)[:, None]
    mv = np.sum(m3 * v3, axis=1)[:, None]
    mH = _cross(m3, H3)
    t = pref * (p * (_cross(v3, H3) + _cross(m3, g3))
                + al * (_cross(v3, mH) + _cross(m3, _cross(v3, H3)) + _cross(m3, _cross(m3, g3)))) \
        + st * (1.0 - mm) * v3 - 2.0 * st * mv * m3
    return t.ravel()


def step_stages(F, m, dt):
    f = F.llg_rhs
    y1 = np.asarray(m, dtype=np.float64).ravel()
    k1 = f(y1)
    y2 = y1 + 0.5 * dt * k1
    k2 = f(y2)
    y3 = y1 + 0.5 * dt * k2
    k3 = f(y3)
    y4 = y1 + dt * k3
    k4 = f(y4)
    return (y1, y2, y3, y4), (k1, k2, k3, k4)


def step_vjp(F, m, dt, lam, B_T_apply=None):
    """(lam_n, dL/dKu, dL/dH0) of one RK4 step from m given lam = dL/dm_(n+1)."""
    ys, _ = step_stages(F, m, dt)
    lam = np.asarray(lam, dtype=np.float64).ravel()
    gKu = np.zeros(F.N)
    gH0 = np.zeros(3)
    out = lam.copy()
    cl = (dt / 6.0, dt / 3.0, dt / 3.0, dt / 6.0)
    ca = (0.5 * dt, 0.5 * dt, dt, 0.0)
    ap = np.zeros_like(lam)
    for s in (3, 2, 1, 0):
        w = cl[s] * lam + ca[s] * ap
        a, gk, gh = rhs_vjp(F, ys[s], w, B_T_apply)
        out += a
        gKu += gk
        gH0 += gh
        ap = a
    return out, gKu, gH0


def step_jvp(F, m, dm, dt, dKu=None, dH0=None):
    """(m_(n+1), tangent) of one RK4 step."""
    ys, ks = step_stages(F, m, dt)
    dm = np.asarray(dm, dtype=np.float64).ravel()
    d1 = rhs_jvp(F, ys[0], dm, dKu, dH0)
    d2 = rhs_jvp(F, ys[1], dm + 0.5 * dt * d1, dKu, dH0)
    d3 = rhs_jvp(F, ys[2], dm + 0.5 * dt * d2, dKu, dH0)
    d4 = rhs_jvp(F, ys[3], dm + dt * d3, dKu, dH0)
    mn = ys[0] + dt / 6.0 * (ks[0] + 2 * ks[1] + 2 * ks[2] + ks[3])
    return mn, dm + dt / 6.0 * (d1 + 2 * d2 + 2 * d3 + d4)


def set_params(F, Ku=None, H0=None):
    """Set the nodal Ku map and the uniform applied field of an EffectiveFieldOracle."""
    if Ku is not None:
        F.Ku = np.asarray(Ku, dtype=np.float64).copy()
    if H0 is not None:
        F.H0 = np.tile(np.asarray(H0, dtype=np.float64).reshape(3), F.N)


def trajectory(F, m0, dt, nsteps):
    from .llg import rk4_step
    m = np.asarray(m0, dtype=np.float64).ravel().copy()
    states = [m]
    for _ in range(nsteps):
        m = rk4_step(F.llg_rhs, m, dt)
        states.append(m)
    return states


def trajectory_grad(F, m0, dt, nsteps, dLdmT, B_T_apply=None):
    """Gradient of L(m_T) with respect to (m0, Ku map, H0) given dL/dm_T (reverse sweep)."""
    states = trajectory(F, m0, dt, nsteps)
    lam = np.asarray(dLdmT, dtype=np.float64).ravel().copy()
    gKu = np.zeros(F.N)
    gH0 = np.zeros(3)
    for n in range(nsteps - 1, -1, -1):
        lam, gk, gh = step_vjp(F, states[n], dt, lam, B_T_apply)
        gKu += gk
        gH0 += gh
    return lam, gKu, gH0
