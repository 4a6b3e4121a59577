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
                 H0=None, demag=None, gamma=2.211e5, alpha=0.5, do_precess=1.0, bd=None):
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
        self.K_lin = K.tocsr()
        self.Ku = Ku
        self.has_ani = np.any(np.asarray(Ku) != 0.0)
        if self.has_ani:
            n = np.asarray(n_ani, dtype=np.float64).reshape(N, 3)
            self.n_ani = n / np.maximum(np.linalg.norm(n, axis=1), 1e-300)[:, None]
        self.H0 = np.zeros(3 * N) if H0 is None else np.asarray(H0, dtype=np.float64).ravel()
        self.demag = demag
        self.diagK = self.K_lin.diagonal()
        if self.has_ani:
            self.diagK = self.diagK + fem.anisotropy_diag(self.n_ani, self.Ku, self.Ms)

    def linear(self, m):
        H = self.K_lin @ m
        if self.has_ani:
            H = H + fem.anisotropy_field(m, self.n_ani, self.Ku, self.Ms)
        return H

    def h_eff(self, m):
        H = self.linear(m)
        if self.demag is not None:
            H = H + self.demag.compute(m)
        return H + self.H0

    def h_jac(self, m):
        return self.linear(m) + self.H0

    def llg_rhs(self, m):
        return rhs(m, self.h_eff(m), self.prefactor, self.alpha, self.do_precess, self.stab)


def rk4_step(f, m, dt):
    k1 = f(m)
    k2 = f(m + 0.5 * dt * k1)
    k3 = f(m + 0.5 * dt * k2)
    k4 = f(m + dt * k3)
    return m + (dt / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
