"""Spin-transfer (Zhang-Li) and spin-orbit torques of the LLG right-hand side (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  FP64 numpy restatements of:

* ``zhang_li_matrix``  ZhangLiGPU (gpu/solvers/llg_stt_module_GPU.py:402-429): the P1 form
  int (J . grad u) v dx with the nodal current direction J, row-scaled by 1/V_i, applied to
  each component;
* ``rhs_stt`` / ``jv_stt`` / ``pc_build_stt``  _LLG_RHS_STT_KERNEL (:101-139),
  _JAC_VEC_STT_KERNEL (:142-215), _PC_BUILD_INV3_STT_KERNEL (:218-393) with the coefficients
  of EffectiveFieldSTTGPU (:571-581) and JvContextSTT (:1240-1246);
* ``rhs_sot`` / ``jv_sot`` / ``pc_build_sot``  _LLG_RHS_SOT_KERNEL
  (gpu/solvers/llg_SOT_module_GPU.py:170-205), _JAC_VEC_SOT_KERNEL (:208-275),
  _PC_BUILD_INV3_SOT_KERNEL (:278-437) with c_fl / c_dl of :814-817.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import fem

E_CHARGE = 1.6021766e-19
MU_B = 9.27400915e-24


def pref_zhang(J, P, beta, Ms, alpha):
    return J * P * MU_B / (E_CHARGE * Ms * (1.0 + beta ** 2)) / (1.0 + alpha ** 2) / 1e-9


def sot_coefficients(gamma, alpha, H_dl, H_fl):
    den = 1.0 + alpha * alpha
    return -gamma * (H_fl - alpha * H_dl) / den, -gamma * (H_dl + alpha * H_fl) / den


def zhang_li_matrix(X, tets, J, vol=None):
    """Scalar N x N operator Z with (Z m_c)_i = (1/V_i) int v_i (J . grad m_c)."""
    X = np.asarray(X, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    J = np.asarray(J, dtype=np.float64).reshape(-1, 3)
    N = X.shape[0]
    vt, grads = fem.tet_geometry(X, tets)          # volumes [E], gradients [E, 4, 3]
    rows, cols, vals = [], [], []
    for a in range(4):
        for b in range(4):
            s = np.zeros(tets.shape[0])
            for k in range(4):
                w = vt / 20.0 * (2.0 if a == k else 1.0)
                s += w * np.sum(J[tets[:, k]] * grads[:, b, :], axis=1)
            rows.append(tets[:, a])
            cols.append(tets[:, b])
            vals.append(s)
    K = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(N, N))
    if vol is None:
        vol = fem.lumped_volume(X, tets)
    return (sp.diags(1.0 / vol) @ K).tocsr()


def apply3(Z, m):
    m3 = np.asarray(m, dtype=np.float64).reshape(-1, 3)
    return (Z @ m3).ravel()


def _c(a, b):
    return np.cross(a, b)


def rhs_stt(m, H, z, prefactor, alpha, do_precess, stab, prefZ, beta):
    m, H, z = (np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in (m, H, z))
    mc = _c(m, H)
    zc = _c(m, z)
    s = stab * (1.0 - np.sum(m * m, axis=1))[:, None]
    return (prefactor * (do_precess * mc + alpha * _c(m, mc))
            - prefZ * ((beta - alpha) * zc + (1.0 + alpha * beta) * _c(m, zc)) + s * m).ravel()


def _jv_base(m, h, v, hv, prefactor, alpha, do_precess, stab):
    cv = _c(v, h)
    cm = _c(m, hv)
    mdH = np.sum(m * h, axis=1)[:, None]
    mdHv = np.sum(m * hv, axis=1)[:, None]
    vdH = np.sum(v * h, axis=1)[:, None]
    mdv = np.sum(m * v, axis=1)[:, None]
    mdm = np.sum(m * m, axis=1)[:, None]
    damp = v * mdH - 2.0 * h * mdv + m * (vdH + mdHv) - hv * mdm
    return prefactor * (do_precess * (cv + cm) + alpha * damp) + stab * (1.0 - mdm) * v - 2.0 * stab * m * mdv


def jv_stt(m, h, jm, v, hv, jv, prefactor, alpha, do_precess, stab, prefZ, beta):
    m, h, jm, v, hv, jv = (np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in (m, h, jm, v, hv, jv))
    out = _jv_base(m, h, v, hv, prefactor, alpha, do_precess, stab)
    mdv = np.sum(m * v, axis=1)[:, None]
    mdm = np.sum(m * m, axis=1)[:, None]
    MjV = np.sum(m * jv, axis=1)[:, None]
    VjM = np.sum(v * jm, axis=1)[:, None]
    MjM = np.sum(m * jm, axis=1)[:, None]
    out += -(beta - alpha) * prefZ * (_c(m, jv) + _c(v, jm))
    out += -(1.0 + beta * alpha) * prefZ * (v * MjM + m * VjM + m * MjV - jv * mdm - 2.0 * jm * mdv)
    return out.ravel()


def _inv3(A, det_rule):
    det = (A[:, 0, 0] * (A[:, 1, 1] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 1])
           - A[:, 0, 1] * (A[:, 1, 0] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 0])
           + A[:, 0, 2] * (A[:, 1, 0] * A[:, 2, 1] - A[:, 1, 1] * A[:, 2, 0]))
    det = det_rule(det)
    inv = np.empty_like(A)
    inv[:, 0, 0] = A[:, 1, 1] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 1]
    inv[:, 0, 1] = -(A[:, 0, 1] * A[:, 2, 2] - A[:, 0, 2] * A[:, 2, 1])
    inv[:, 0, 2] = A[:, 0, 1] * A[:, 1, 2] - A[:, 0, 2] * A[:, 1, 1]
    inv[:, 1, 0] = -(A[:, 1, 0] * A[:, 2, 2] - A[:, 1, 2] * A[:, 2, 0])
    inv[:, 1, 1] = A[:, 0, 0] * A[:, 2, 2] - A[:, 0, 2] * A[:, 2, 0]
    inv[:, 1, 2] = -(A[:, 0, 0] * A[:, 1, 2] - A[:, 0, 2] * A[:, 1, 0])
    inv[:, 2, 0] = A[:, 1, 0] * A[:, 2, 1] - A[:, 1, 1] * A[:, 2, 0]
    inv[:, 2, 1] = -(A[:, 0, 0] * A[:, 2, 1] - A[:, 0, 1] * A[:, 2, 0])
    inv[:, 2, 2] = A[:, 0, 0] * A[:, 1, 1] - A[:, 0, 1] * A[:, 1, 0]
    return inv / det[:, None, None]


def pc_build_stt(m, H, g, diagK, shift, c1, c2, c3, c4, stab, include_stab=True, use_abs_kappa=True,
                 eps_reg=1e-14, det_eps=1e-30):
    """Per-node (shift + eps) I - J_i with the STT terms, inverted: [N, 3, 3]."""
    m3 = np.asarray(m, dtype=np.float64).reshape(-1, 3)
    g3 = np.asarray(g, dtype=np.float64).reshape(-1, 3)
    Jl = _llg_local_jacobian(m3, np.asarray(H, dtype=np.float64).reshape(-1, 3),
                             np.asarray(diagK, dtype=np.float64).reshape(-1, 3), c1, c2, stab, include_stab,
                             use_abs_kappa)
    gx, gy, gz = g3[:, 0], g3[:, 1], g3[:, 2]
    mx, my, mz = m3[:, 0], m3[:, 1], m3[:, 2]
    mdG = mx * gx + my * gy + mz * gz
    Js = np.zeros_like(Jl)
    Js[:, 0, 1] = c3 * (-gz)
    Js[:, 0, 2] = c3 * gy
    Js[:, 1, 0] = c3 * gz
    Js[:, 1, 2] = c3 * (-gx)
    Js[:, 2, 0] = c3 * (-gy)
    Js[:, 2, 1] = c3 * gx
    Bg = np.empty_like(Jl)
    Bg[:, 0, 0] = mdG - gx * mx
    Bg[:, 1, 1] = mdG - gy * my
    Bg[:, 2, 2] = mdG - gz * mz
    Bg[:, 0, 1] = mx * gy - 2.0 * gx * my
    Bg[:, 0, 2] = mx * gz - 2.0 * gx * mz
    Bg[:, 1, 0] = my * gx - 2.0 * gy * mx
    Bg[:, 1, 2] = my * gz - 2.0 * gy * mz
    Bg[:, 2, 0] = mz * gx - 2.0 * gz * mx
    Bg[:, 2, 1] = mz * gy - 2.0 * gz * my
    J = Jl + Js + c4 * Bg
    A = (shift + eps_reg) * np.eye(3)[None] - J

    def rule(det):
        small = np.abs(det) < det_eps
        sgn = np.where(det + det_eps >= 0.0, 1.0, -1.0)
        return np.where(small, det + sgn * det_eps, det)
    return _inv3(A, rule)


def _llg_local_jacobian(m, h, d, c1, c2, stab, include_stab, use_abs_kappa):
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
    B = np.empty((n, 3, 3))
    B[:, 0, 0] = mdH - hx * mx
    B[:, 1, 1] = mdH - hy * my
    B[:, 2, 2] = mdH - hz * mz
    B[:, 0, 1] = mx * hy - 2.0 * hx * my
    B[:, 0, 2] = mx * hz - 2.0 * hx * mz
    B[:, 1, 0] = my * hx - 2.0 * hy * mx
    B[:, 1, 2] = my * hz - 2.0 * hy * mz
    B[:, 2, 0] = mz * hx - 2.0 * hz * mx
    B[:, 2, 1] = mz * hy - 2.0 * hz * my
    C = m[:, :, None] * m[:, None, :] - mdm[:, None, None] * np.eye(3)[None]
    J = J + c2 * (B + kappa[:, None, None] * C)
    if include_stab:
        J = J + stab * ((1.0 - mdm)[:, None, None] * np.eye(3)[None] - 2.0 * m[:, :, None] * m[:, None, :])
    return J


def rhs_sot(m, H, p, prefactor, alpha, do_precess, stab, c_fl, c_dl):
    m, H, p = (np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in (m, H, p))
    mc = _c(m, H)
    sp_ = _c(m, p)
    s = stab * (1.0 - np.sum(m * m, axis=1))[:, None]
    return (prefactor * (do_precess * mc + alpha * _c(m, mc)) + c_fl * sp_ + c_dl * _c(m, sp_) + s * m).ravel()


def jv_sot(m, h, p, v, hv, prefactor, alpha, do_precess, stab, c_fl, c_dl):
    m, h, p, v, hv = (np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in (m, h, p, v, hv))
    out = _jv_base(m, h, v, hv, prefactor, alpha, do_precess, stab)
    q = _c(m, p)
    dq = _c(v, p)
    return (out + c_fl * dq + c_dl * (_c(v, q) + _c(m, dq))).ravel()


def pc_build_sot(m, H, p, diagK, shift, prefactor, alpha, do_precess, stab, c_fl, c_dl, use_abs_diag=False,
                 eps_reg=1e-14, det_eps=1e-30):
    m3 = np.asarray(m, dtype=np.float64).reshape(-1, 3)
    h3 = np.asarray(H, dtype=np.float64).reshape(-1, 3)
    p3 = np.asarray(p, dtype=np.float64).reshape(-1, 3)
    k = np.asarray(diagK, dtype=np.float64).reshape(-1, 3)
    if use_abs_diag:
        k = np.abs(k)
    n = m3.shape[0]
    J = np.empty((n, 3, 3))
    for c in range(3):
        v = np.zeros((n, 3))
        v[:, c] = 1.0
        hv = np.zeros((n, 3))
        hv[:, c] = k[:, c]
        J[:, :, c] = jv_sot(m3, h3, p3, v, hv, prefactor, alpha, do_precess, stab, c_fl, c_dl).reshape(n, 3)
    A = (shift + eps_reg) * np.eye(3)[None] - J

    def rule(det):
        small = np.abs(det) < det_eps
        sgn = np.where(det >= 0.0, 1.0, -1.0)
        return np.where(small, det + sgn * det_eps, det)
    return _inv3(A, rule)
