"""LaBonte / Barzilai-Borwein energy minimiser (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  FP64 numpy restatement of
LaBonteBBMinimizerGPU (gpu/solvers/Minimizer_GPU.py:171-845) on the oracle's effective field:
_CAYLEY_KERNEL (:46-74), _PROJDIR_KERNEL (:77-88), the BB step (:397-522, adaptive / bb1 /
bb2), the non-monotone acceptance with back-tracking, alpha restarts on stagnation and the
stopping rules (:527-845); the energy is the lumped one of compute_Energy_minimize_gpu
(gpu/solvers/llg_module_GPU.py:1014-1229, without the anisotropy offset).
"""
from __future__ import annotations

import numpy as np

from .demag import MU0


def cayley(m, d, alpha):
    m = np.asarray(m).reshape(-1, 3)
    d = np.asarray(d).reshape(-1, 3)
    c = 0.5 * alpha * np.cross(m, d)
    b = m + np.cross(c, m)
    cb = np.cross(c, b)
    cdb = np.sum(c * b, axis=1)[:, None]
    c2 = np.sum(c * c, axis=1)[:, None]
    return ((b + cb + c * cdb) / (1.0 + c2)).ravel()


def evaluate(F, m):
    """(E [J], d, max |d|) at m for an EffectiveFieldOracle F (mesh in nm)."""
    m3 = np.asarray(m).reshape(-1, 3)
    H = F.h_eff(np.asarray(m).ravel()).reshape(-1, 3)
    H0 = F.H0.reshape(-1, 3)
    E = MU0 * F.Ms * 1e-27 * float(np.sum(F.vol * np.sum(m3 * (-0.5 * H - 0.5 * H0), axis=1)))
    d = H - np.sum(m3 * H, axis=1)[:, None] * m3
    return E, d.ravel(), float(np.sqrt(np.sum(d * d, axis=1)).max())


def minimize(F, m0, max_iter=5000, tol=1.0, alpha0=5e-11, alpha_min=1e-13, alpha_max=1e-8, bb_variant="adaptive",
             bb_adaptive_tau0=0.5, bb_adaptive_Malpha=2, bb_adaptive_tau_min=1e-12, bb_adaptive_tau_max=1e12,
             nonmonotone_window=10, max_backtracking=10, shrink=0.5, energy_accept_rtol=1e-10,
             energy_accept_atol=1e-24, energy_stagnation_rtol=1e-10, energy_stagnation_atol=1e-24,
             stagnation_window=30, max_rejected_at_alpha_min=30, alpha_restart=5e-11, max_alpha_restarts=3,
             restart_residual_factor=50.0, stagnation_residual_stop=50):
    m = np.asarray(m0, dtype=np.float64).reshape(-1, 3)
    m = (m / np.maximum(np.linalg.norm(m, axis=1), 1e-30)[:, None]).ravel()
    E, d, g = evaluate(F, m)
    hist = [E]
    alpha = min(max(alpha0, alpha_min), alpha_max)
    tau = min(max(bb_adaptive_tau0, bb_adaptive_tau_min), bb_adaptive_tau_max)
    a2hist = []
    rej = restarts = 0
    reason = "max_iter"
    it = 0
    for it in range(max_iter):
        if g < tol:
            reason = "projected_field_tol"
            break
        if len(hist) > stagnation_window:
            Eo, En = hist[-stagnation_window], hist[-1]
            if abs(En - Eo) <= energy_stagnation_atol + energy_stagnation_rtol * max(abs(Eo), abs(En), 1e-300):
                if g <= restart_residual_factor * tol:
                    reason = "energy_stagnation_low_residual"
                    break
                if restarts < max_alpha_restarts:
                    alpha = min(max(alpha_restart, alpha_min), alpha_max)
                    restarts += 1
                    rej = 0
                    hist = [E]
                    continue
                if g < stagnation_residual_stop:
                    reason = "energy_stagnation_high_residual"
                    break
        m_old, d_old = m.copy(), d.copy()
        E_ref = max(hist[-nonmonotone_window:])
        accepted = False
        alpha_try = alpha
        for _ in range(max_backtracking + 1):
            mt = cayley(m_old, d_old, alpha_try)
            Et, dt, gt = evaluate(F, mt)
            if Et <= E_ref + energy_accept_atol + energy_accept_rtol * max(abs(E_ref), abs(Et), 1e-300):
                m, d, E, g = mt, dt, Et, gt
                hist.append(E)
                accepted = True
                rej = 0
                break
            alpha_try = max(alpha_try * shrink, alpha_min)
        if not accepted:
            rej += 1
            alpha = alpha_min
            if rej >= max_rejected_at_alpha_min:
                reason = "repeated_rejection_at_alpha_min"
                break
            continue
        s = m - m_old
        y = d_old - d
        sty, sts, yty = float(s @ y), float(s @ s), float(y @ y)
        if sts < 1e-300 or yty < 1e-300:
            alpha = min(max(alpha_try, alpha_min), alpha_max)
        elif bb_variant == "adaptive":
            if sty <= 1e-300:
                alpha = alpha_max
            else:
                a1 = min(max(sts / sty, alpha_min), alpha_max)
                a2 = min(max(sty / yty, alpha_min), alpha_max)
                a2hist = (a2hist + [a2])[-max(bb_adaptive_Malpha + 1, 1):]
                if a2 / max(a1, 1e-300) <= tau:
                    alpha, tau = min(a2hist), tau * 0.9
                else:
                    alpha, tau = a1, tau * 1.1
                tau = min(max(tau, bb_adaptive_tau_min), bb_adaptive_tau_max)
        elif abs(sty) < 1e-300:
            alpha = min(max(alpha_try, alpha_min), alpha_max)
        else:
            alpha = abs(sts / sty if bb_variant == "bb1" else sty / yty)
        alpha = min(max(alpha, alpha_min), alpha_max)
    m3 = m.reshape(-1, 3)
    m = (m3 / np.maximum(np.linalg.norm(m3, axis=1), 1e-30)[:, None]).ravel()
    E, d, g = evaluate(F, m)
    return m, {"iterations": it, "energy": E, "max_projected_field": g, "stop_reason": reason,
               "converged": reason in ("projected_field_tol", "energy_stagnation_low_residual")}
