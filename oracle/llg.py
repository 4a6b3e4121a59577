"""LLG right-hand side, Jacobian-vector product, block preconditioner, RK4.

Restates, FP64 numpy, AoS vectors (node-major, 3 components):

* ``rhs``      _LLG_RHS_KERNEL  gpu/solvers/llg_module_GPU.py:100-122;
               CPU llg_rhs cpu/solvers/llg_module.py:902-930
* ``jv``       _JAC_VEC_KERNEL  gpu/solvers/llg_module_GPU.py:125-164;
               CPU jac_vec_local_kernel cpu/solvers/llg_module.py:25-74
* ``pc_build`` _PC_BUILD_INV3_KERNEL gpu/solvers/llg_module_GPU.py:167-293
* ``pc_apply`` _PC_APPLY_KERNEL gpu/solvers/llg_module_GPU.py:296-308
* constants    prefactorEQ = -gamma/(1+alpha^2), Stab = Ms gamma/(1+alpha^2)/2
               (llg_module_GPU.py:430-431)
* ``EffectiveFieldOracle``  EffectiveField.compute_H_eff_vec (:972-1006),
               compute_H_jac_vec (:1232-1257), diagK (:674-691)
* ``EffectiveFieldOracle(H_time=...)`` adds the time-dependent field H_time(t) (the
  reference's H_time_func, llg_module_GPU.py:909-956, 998-1000) at the evaluation time.
* ``dp5_attempt`` / ``relax_explicit``: the reference's explicit relaxation
  (llg_module_GPU.py:1724-1970): PETSc TS rk/5dp (Dormand-Prince 5(4), coefficients of
  Dormand & Prince 1980) with the TSAdapt "basic" options it sets (clip 0.1-3, safety 0.9,
  reject safety 0.1, dt in [1e-18, 1e-10], weighted RMS error norm, exponent -1/5), and the
  dm/dt stopper StopByMaxDmdtFDGPU (:314-382).  PETSc itself is not in this image, so the
  step sequence is pinned by this restatement, not by PETSc output.
* ``rk4_step`` the fixed-step scheme used for every trajectory comparison.
  The reference integrates with PETSc TS rk/5dp (adaptive) or BDF; neither
  exposes a fixed step (llg_module_GPU.py:1746-1772), so the oracle and the
  product both use classic RK4 (4 RHS evaluations per step).
"""
from __future__ import annotations

import numpy as np

from . import fem


def constants(Ms, gamma, alpha):
    return -gamma / (1.0 + alpha * alpha), Ms * gamma / (1.0 + alpha * alpha) * 0.5


def rhs(m, H, prefactor, alpha, do_precess, stab):
    m = np.asarray(m).reshape(-1, 3)
    H = np.asarray(H).reshape(-1, 3)
    mc = np.cross(m, H)
    mcm = np.cross(m, mc)
    norm2 = np.sum(m * m, axis=1)
    s = stab * (1.0 - norm2)
    return (prefactor * (do_precess * mc + alpha * mcm) + s[:, None] * m).ravel()


def jv(m, Hm, v, Hv, gamma, alpha, do_precess, stab):
    m = np.asarray(m).reshape(-1, 3)
    h = np.asarray(Hm).reshape(-1, 3)
    v = np.asarray(v).reshape(-1, 3)
    hv = np.asarray(Hv).reshape(-1, 3)
    cv = np.cross(v, h)
    cm = np.cross(m, hv)
    mdHm = np.sum(m * h, axis=1)[:, None]
    mdHv = np.sum(m * hv, axis=1)[:, None]
    vdHm = np.sum(v * h, axis=1)[:, None]
    mdv = np.sum(m * v, axis=1)[:, None]
    mdmm = np.sum(m * m, axis=1)[:, None]
    damp = v * mdHm - 2.0 * h * mdv + m * (vdHm + mdHv) - hv * mdmm
    coef = -gamma / (1.0 + alpha * alpha)
    out = coef * (do_precess * (cv + cm) + alpha * damp) + stab * (1.0 - mdmm) * v - 2.0 * stab * m * mdv
    return out.ravel()


def pc_build(m, H, diagK, shift, c1, c2, stab, include_stab=True, use_abs_kappa=True,
             eps_reg=1e-14, det_eps=1e-30, diag_cubic=None):
    """Per-node inverse of A_i = (shift+eps) I - J_i, returned as [N,3,3]."""
    m = np.asarray(m).reshape(-1, 3)
    h = np.asarray(H).reshape(-1, 3)
    d = np.asarray(diagK).reshape(-1, 3).copy()
    if diag_cubic is not None:
        d = d + np.asarray(diag_cubic).reshape(-1, 3)
    kappa = (np.abs(d).sum(axis=1) if use_abs_kappa else d.sum(axis=1)) / 3.0
    mx, my, mz = m[:, 0], m[:, 1], m[:, 2]
    hx, hy, hz = h[:, 0], h[:, 1], h[:, 2]
    mdH = mx * hx + my * hy + mz * hz
    mdm = mx * mx + my * my + mz * mz
    n = m.shape[0]
    J = np.zeros((n, 3, 3))
    J[:, 0, 1] = -c1 * (-hz - kappa * (-mz))
    J[:, 0, 2] = -c1 * (hy - kappa * my)
    J[:, 1, 0] = -c1 * (hz - kappa * mz)
    J[:, 1, 2] = -c1 * (-hx - kappa * (-mx))
    J[:, 2, 0] = -c1 * (-hy - kappa * (-my))
    J[:, 2, 1] = -c1 * (hx - kappa * mx)
    Bm = np.empty((n, 3, 3))
    Bm[:, 0, 0] = mdH - hx * mx
    Bm[:, 1, 1] = mdH - hy * my
    Bm[:, 2, 2] = mdH - hz * mz
    Bm[:, 0, 1] = mx * hy - 2.0 * hx * my
    Bm[:, 0, 2] = mx * hz - 2.0 * hx * mz
    Bm[:, 1, 0] = my * hx - 2.0 * hy * mx
    Bm[:, 1, 2] = my * hz - 2.0 * hy * mz
    Bm[:, 2, 0] = mz * hx - 2.0 * hz * mx
    Bm[:, 2, 1] = mz * hy - 2.0 * hz * my
    C = m[:, :, None] * m[:, None, :] - mdm[:, None, None] * np.eye(3)[None]
    J = J + c2 * (Bm + kappa[:, None, None] * C)
    if include_stab:
        J = J + stab * ((1.0 - mdm)[:, None, None] * np.eye(3)[None] - 2.0 * m[:, :, None] * m[:, None, :])
    s = shift + eps_reg
    A = s * np.eye(3)[None] - J
    det = (A[:, 0, 0] * (A[:, 1, 1] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 1])
           - A[:, 0, 1] * (A[:, 1, 0] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 0])
           + A[:, 0, 2] * (A[:, 1, 0] * A[:, 2, 1] - A[:, 1, 1] * A[:, 2, 0]))
    small = np.abs(det) < det_eps
    sgn = np.where(det + det_eps > 0.0, 1.0, -1.0)
    det = np.where(small, det + sgn * det_eps, det)
    inv = np.empty_like(A)
    inv[:, 0, 0] = (A[:, 1, 1] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 1])
    inv[:, 0, 1] = -(A[:, 0, 1] * A[:, 2, 2] - A[:, 0, 2] * A[:, 2, 1])
    inv[:, 0, 2] = (A[:, 0, 1] * A[:, 1, 2] - A[:, 0, 2] * A[:, 1, 1])
    inv[:, 1, 0] = -(A[:, 1, 0] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 0])
    inv[:, 1, 1] = (A[:, 0, 0] * A[:, 2, 2] - A[:, 0, 2] * A[:, 2, 0])
    inv[:, 1, 2] = -(A[:, 0, 0] * A[:, 1, 2] - A[:, 0, 2] * A[:, 1, 0])
    inv[:, 2, 0] = (A[:, 1, 0] * A[:, 2, 1] - A[:, 1, 1] * A[:, 2, 0])
    inv[:, 2, 1] = -(A[:, 0, 0] * A[:, 2, 1] - A[:, 0, 1] * A[:, 2, 0])
    inv[:, 2, 2] = (A[:, 0, 0] * A[:, 1, 1] - A[:, 0, 1] * A[:, 1, 0])
    return inv / det[:, None, None]


def pc_apply(inv, x):
    x = np.asarray(x).reshape(-1, 3)
    return np.einsum("nij,nj->ni", inv, x).ravel()


class EffectiveFieldOracle:
    """H_eff = K_lin m + H_ani(m) + H_demag(m) + H0 (+ H(t))."""

    def __init__(self, X, tets, Ms, Aex=0.0, Ku=0.0, n_ani=None, D_int=0.0, n_int=None,
                 H0=None, demag=None, gamma=2.211e5, alpha=0.5, do_precess=1.0, bd=None, H_time=None,
                 D_bulk=0.0):
        import scipy.sparse as sp
        from . import lindholm
        self.X = np.asarray(X, dtype=np.float64)
        self.tets = np.asarray(tets, dtype=np.int64)
        N = self.X.shape[0]
        self.N = N
        self.Ms = float(Ms)
        self.gamma, self.alpha, self.do_precess = float(gamma), float(alpha), float(do_precess)
        self.prefactor, self.stab = constants(self.Ms, self.gamma, self.alpha)
        self.vol = fem.lumped_volume(self.X, self.tets)
        K = sp.csr_matrix((3 * N, 3 * N))
        if Aex != 0.0:
            K = K + fem.exchange_matrix(self.X, self.tets, Aex, self.Ms, self.vol)
        if D_int != 0.0:
            bd = lindholm.boundary_data(self.X, self.tets) if bd is None else bd
            nvec = np.asarray(n_int, dtype=np.float64).reshape(N, 3)
            K = K + fem.dmi_interfacial_matrix(self.X, self.tets, D_int, self.Ms, nvec,
                                               bd["tris"], bd["ntri"], self.vol)
        if D_bulk != 0.0:
            bd = lindholm.boundary_data(self.X, self.tets) if bd is None else bd
            K = K + fem.dmi_bulk_matrix(self.X, self.tets, D_bulk, self.Ms, bd["tris"], bd["ntri"], self.vol)
        self.K_lin = K.tocsr()
        self.Ku = Ku
        self.has_ani = np.any(np.asarray(Ku) != 0.0)
        if self.has_ani:
            n = np.asarray(n_ani, dtype=np.float64).reshape(N, 3)
            self.n_ani = n / np.maximum(np.linalg.norm(n, axis=1), 1e-300)[:, None]
        self.H0 = np.zeros(3 * N) if H0 is None else np.asarray(H0, dtype=np.float64).ravel()
        self.demag = demag
        self.H_time = H_time
        self.diagK = self.K_lin.diagonal()
        if self.has_ani:
            self.diagK = self.diagK + fem.anisotropy_diag(self.n_ani, self.Ku, self.Ms)

    def linear(self, m):
        H = self.K_lin @ m
        if self.has_ani:
            H = H + fem.anisotropy_field(m, self.n_ani, self.Ku, self.Ms)
        return H

    def h_time(self, t):
        if self.H_time is None:
            return 0.0
        v = np.asarray(self.H_time(float(t)), dtype=np.float64)
        return np.tile(v, self.N) if v.size == 3 else v.reshape(-1)

    def h_eff(self, m, t=0.0):
        H = self.linear(m)
        if self.demag is not None:
            H = H + self.demag.compute(m)
        return H + self.H0 + self.h_time(t)

    def h_jac(self, m, t=0.0):
        return self.linear(m) + self.H0 + self.h_time(t)

    def llg_rhs(self, m, t=0.0):
        return rhs(m, self.h_eff(m, t), self.prefactor, self.alpha, self.do_precess, self.stab)


def rk4_step(f, m, dt):
    k1 = f(m)
    k2 = f(m + 0.5 * dt * k1)
    k3 = f(m + 0.5 * dt * k2)
    k4 = f(m + dt * k3)
    return m + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)


def rk4_step_t(f, t, m, dt):
    """Classic RK4 for a time-dependent right-hand side f(m, t)."""
    k1 = f(m, t)
    k2 = f(m + 0.5 * dt * k1, t + 0.5 * dt)
    k3 = f(m + 0.5 * dt * k2, t + 0.5 * dt)
    k4 = f(m + dt * k3, t + dt)
    return m + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)


DP_C = [0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0]
DP_A = [[],
        [1 / 5],
        [3 / 40, 9 / 40],
        [44 / 45, -56 / 15, 32 / 9],
        [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
        [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
        [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]]
DP_B4 = [5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40]


def dp5_attempt(f, t, m, dt, rtol, atol, k1=None):
    """One Dormand-Prince 5(4) attempt: (y5, weighted RMS error norm, k7)."""
    k = [f(m, t) if k1 is None else k1]
    y = None
    for i in range(1, 7):
        y = m + dt * sum(a * kj for a, kj in zip(DP_A[i], k))
        k.append(f(y, t + DP_C[i] * dt))
    y5 = y
    e = dt * sum((b5 - b4) * kj for b5, b4, kj in zip(DP_A[6] + [0.0], DP_B4, k))
    y4 = y5 - e
    tol = atol + rtol * np.maximum(np.abs(y5), np.abs(y4))
    return y5, float(np.sqrt(np.mean((e / tol) ** 2))), k[6]


def relax_explicit(f, m0, t0, t_final, dt_init, rtol=1e-6, atol=1e-6, stopping_dmdt=0.0, check_every=5,
                   max_steps=10 ** 7):
    """The explicit adaptive relaxation loop: returns (m, stats) with stats t_end, dt_last,
    nsteps, reason (1 final time reached, 2 dm/dt below the threshold), rejected, dts."""
    clip, safety0, rsafety, dt_min, dt_max = (0.1, 3.0), 0.9, 0.1, 1e-18, 1e-10
    t, m, dt = float(t0), np.asarray(m0, dtype=np.float64).copy(), min(max(dt_init, dt_min), dt_max)
    k1 = None
    steps, rejected, reason, dts = 0, 0, 0, []
    u_prev, t_prev, last = None, None, float("nan")
    nxt = dt
    while steps < max_steps:
        if t >= t_final:
            reason = 1
            break
        accept_prev = True
        while True:
            y5, en, k7 = dp5_attempt(f, t, m, dt, rtol, atol, k1)
            safety = safety0
            if en > 1.0:
                if not accept_prev:
                    safety *= rsafety
                accept = dt < (1.0 + 1.4901161193847656e-08) * dt_min
            else:
                accept = True
            hfac = safety * en ** (-1.0 / 5.0) if en > 0.0 else float("inf")
            nxt = min(max(dt * min(max(hfac, clip[0]), clip[1]), dt_min), dt_max)
            if accept:
                break
            rejected += 1
            accept_prev = False
            k1 = f(m, t) if k1 is None else k1
            dt = nxt
        m, t, k1 = y5, t + dt, k7
        dts.append(dt)
        steps += 1
        stop = False
        if stopping_dmdt > 0.0 and (check_every <= 1 or steps % check_every == 0):
            if t_prev is None or t - t_prev <= 0.0:
                u_prev, t_prev = m.copy(), t
            else:
                du = (m - u_prev).reshape(-1, 3)
                last = float(np.sqrt((du * du).sum(axis=1)).max()) / (t - t_prev) * (180.0 / np.pi) * 1e-9
                u_prev, t_prev = m.copy(), t
                stop = last < stopping_dmdt
        dt = nxt
        if stop:
            reason = 2
            break
    return m, {"t_end": t, "dt_last": dt, "nsteps": steps, "reason": reason, "rejected": rejected, "dts": dts,
               "maxdmdt_deg_ns": last}
