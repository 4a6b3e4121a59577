"""LaBonte / Barzilai-Borwein energy minimiser (drop-in for gpu/solvers/Minimizer_GPU.py).

``LaBonteBBMinimizerGPU.minimize`` follows the reference algorithm (:171-845): projected
effective field d = H - (m . H) m, norm-preserving Cayley update m(alpha) along d, BB step
lengths (bb1 / bb2 / the adaptive GPSS rule), non-monotone energy acceptance over a window,
back-tracking, alpha restarts on energy stagnation, and the same stopping rules and stats.
Each trial state costs one device call (``spx_llg_min_trial``: Cayley step, H_eff with the
demag field, projected field, lumped energy, max |d| and the BB products in one pass) and one
host read of five numbers.  ``EnergyMinimizerGPU`` is the builder-style driver (:860-1210)
with ``minimize`` and ``hysteresis``; file output (XDMF / ADIOS2) is not part of this build.
The reference's "alternate" BB variant selects no step (its branch assigns nothing); here it
alternates BB1 / BB2 by iteration parity.
"""
from __future__ import annotations

import time

import numpy as np

from . import _lib
from ._lib import call, ptr


class LaBonteBBMinimizerGPU:
    def __init__(self, effective_field):
        import torch
        self.hef = effective_field
        self.local_size = effective_field.local_size
        self.local_dofs = effective_field.local_dofs
        z = lambda: torch.zeros(self.local_size, dtype=torch.float64, device="cuda")  # noqa: E731
        self.m = z()
        self.m_old, self.m_trial = z(), z()
        self.d, self.d_old, self.d_trial = z(), z(), z()
        self._out = np.zeros(5)
        self.last_energy = None
        self.last_max_grad = None
        self.last_iterations = 0
        self.evaluations = 0
        self._it = 0

    # ------------------------------------------------------------ device calls
    def _eval(self, normalize):
        call("spx_llg_min_eval", self.hef.handle, ptr(self.m), ptr(self.d), 1 if normalize else 0, ptr(self._out),
             _lib.stream_ptr())
        self.evaluations += 1
        return float(self._out[0]), float(self._out[1])

    def _trial(self, alpha):
        call("spx_llg_min_trial", self.hef.handle, ptr(self.m_old), ptr(self.d_old), float(alpha),
             ptr(self.m_trial), ptr(self.d_trial), ptr(self._out), _lib.stream_ptr())
        self.evaluations += 1
        return tuple(float(v) for v in self._out)

    # ------------------------------------------------------------ BB step (:397-522)
    def _bb_step(self, alpha_old, alpha_min, alpha_max, variant, sty, sts, yty):
        key = str(variant).lower().replace("-", "_")
        if sts < 1e-300 or yty < 1e-300:
            self.bb_last_rule = "reuse_old_degenerate"
            return min(max(float(alpha_old), alpha_min), alpha_max)
        if key in ("adaptive", "gpss", "loris", "exl", "loris_zanni"):
            if sty <= 1e-300:
                self.bb_last_alpha1 = self.bb_last_alpha2 = None
                self.bb_last_rule = "adaptive_alpha_max_nonpositive_sty"
                self.bb_adaptive_alpha_max_count += 1
                return float(alpha_max)
            a1 = min(max(sts / sty, alpha_min), alpha_max)
            a2 = min(max(sty / yty, alpha_min), alpha_max)
            self.bb_last_alpha1, self.bb_last_alpha2 = a1, a2
            self.bb_alpha2_history.append(a2)
            keep = max(int(self.bb_Malpha) + 1, 1)
            self.bb_alpha2_history = self.bb_alpha2_history[-keep:]
            if a2 / max(a1, 1e-300) <= self.bb_tau:
                alpha = min(self.bb_alpha2_history)
                self.bb_tau *= 0.9
                self.bb_last_rule = "adaptive_recent_min_bb2"
                self.bb_adaptive_alpha2_count += 1
            else:
                alpha = a1
                self.bb_tau *= 1.1
                self.bb_last_rule = "adaptive_bb1"
                self.bb_adaptive_alpha1_count += 1
            self.bb_tau = min(max(self.bb_tau, self.bb_tau_min), self.bb_tau_max)
            return min(max(alpha, alpha_min), alpha_max)
        if abs(sty) < 1e-300:
            self.bb_last_rule = "reuse_old_small_sty"
            return min(max(float(alpha_old), alpha_min), alpha_max)
        a1, a2 = sts / sty, sty / yty
        self.bb_last_alpha1, self.bb_last_alpha2 = a1, a2
        if key == "bb1":
            alpha, self.bb_last_rule = a1, "bb1"
        elif key == "bb2":
            alpha, self.bb_last_rule = a2, "bb2"
        else:  # alternate
            alpha = a1 if self._it % 2 == 0 else a2
            self.bb_last_rule = "alternate"
        return float(min(max(abs(alpha), alpha_min), alpha_max))

    # ------------------------------------------------------------ main loop (:527-845)
    def minimize(self, max_iter=5000, tol=1.0, alpha0=5e-11, alpha_min=1e-13, alpha_max=1e-8,
                 bb_variant="adaptive", bb_adaptive_tau0=0.5, bb_adaptive_Malpha=2, bb_adaptive_tau_min=1e-12,
                 bb_adaptive_tau_max=1e12, nonmonotone_window=10, max_backtracking=10, shrink=0.5, print_every=100,
                 energy_accept_rtol=1e-10, energy_accept_atol=1e-24, energy_stagnation_rtol=1e-10,
                 energy_stagnation_atol=1e-24, stagnation_window=30, max_rejected_at_alpha_min=30,
                 alpha_restart=5e-11, max_alpha_restarts=3, restart_residual_factor=50.0,
                 stagnation_residual_stop=50, verbose=False):
        self.bb_tau = min(max(float(bb_adaptive_tau0), float(bb_adaptive_tau_min)), float(bb_adaptive_tau_max))
        self.bb_Malpha = max(int(bb_adaptive_Malpha), 0)
        self.bb_tau_min, self.bb_tau_max = float(bb_adaptive_tau_min), float(bb_adaptive_tau_max)
        self.bb_alpha2_history = []
        self.bb_adaptive_alpha1_count = self.bb_adaptive_alpha2_count = self.bb_adaptive_alpha_max_count = 0
        self.bb_last_rule, self.bb_last_alpha1, self.bb_last_alpha2 = "init", None, None
        self.hef.get_state(self.m)
        E, max_g = self._eval(normalize=True)
        hist = [E]
        alpha = min(max(float(alpha0), alpha_min), alpha_max)
        rej = 0
        restarts = 0
        reason = "max_iter"
        for it in range(max_iter):
            self._it = it
            self.last_iterations = it
            self.last_max_grad = max_g
            if verbose and (it == 0 or it % print_every == 0):
                print(f"[LaBonte-BB] it={it:06d} E={E:.12e} max|projH|={max_g:.6e} alpha={alpha:.6e}", flush=True)
            if max_g < tol:
                reason = "projected_field_tol"
                break
            if len(hist) > stagnation_window:
                E_old, E_new = hist[-stagnation_window], hist[-1]
                if abs(E_new - E_old) <= energy_stagnation_atol + energy_stagnation_rtol * max(abs(E_old), abs(E_new),
                                                                                            1e-300):
                    if max_g <= restart_residual_factor * tol:
                        reason = "energy_stagnation_low_residual"
                        break
                    if restarts < max_alpha_restarts:
                        alpha = min(max(alpha_restart, alpha_min), alpha_max)
                        restarts += 1
                        rej = 0
                        hist = [E]
                        E, max_g = self._eval(normalize=False)
                        continue
                    if max_g < stagnation_residual_stop:
                        reason = "energy_stagnation_high_residual"
                        break
            self.m_old.copy_(self.m)
            self.d_old.copy_(self.d)
            E_ref = max(hist[-nonmonotone_window:])
            accepted = False
            alpha_try = alpha
            for _ in range(max_backtracking + 1):
                Et, gt, sty, sts, yty = self._trial(alpha_try)
                if Et <= E_ref + energy_accept_atol + energy_accept_rtol * max(abs(E_ref), abs(Et), 1e-300):
                    self.m, self.m_trial = self.m_trial, self.m
                    self.d, self.d_trial = self.d_trial, self.d
                    E, max_g = Et, gt
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
                E, max_g = self._eval(normalize=False)
                continue
            alpha = self._bb_step(alpha_try, alpha_min, alpha_max, bb_variant, sty, sts, yty)
            alpha = min(max(alpha, alpha_min), alpha_max)
        E, max_g = self._eval(normalize=True)
        self.last_energy, self.last_max_grad = E, max_g
        self.hef.set_state(self.m)
        return {"iterations": int(self.last_iterations), "energy": float(E), "max_projected_field": float(max_g),
                "alpha": float(alpha), "bb_variant": str(bb_variant), "bb_last_rule": str(self.bb_last_rule),
                "bb_last_alpha1": self.bb_last_alpha1, "bb_last_alpha2": self.bb_last_alpha2,
                "bb_adaptive_tau": float(self.bb_tau), "bb_adaptive_Malpha": int(self.bb_Malpha),
                "bb_adaptive_alpha1_count": int(self.bb_adaptive_alpha1_count),
                "bb_adaptive_alpha2_count": int(self.bb_adaptive_alpha2_count),
                "bb_adaptive_alpha_max_count": int(self.bb_adaptive_alpha_max_count),
                "alpha_restarts": int(restarts), "rejected_at_alpha_min": int(rej),
                "energy_history_len": int(len(hist)), "stop_reason": reason,
                "converged": reason in ("projected_field_tol", "energy_stagnation_low_residual"),
                "field_evaluations": int(self.evaluations)}


class EnergyMinimizerGPU:
    """Builder-style driver (Minimizer_GPU.py:860-1210): add_* interactions, then minimize."""

    def __init__(self, X, tets, Ms, gamma=2.211e5, alpha=0.5, do_precess=1.0, precision="f64"):
        from .geometry import as_mesh
        self.X, self.tets = as_mesh(X, tets)
        self.Ms, self.gamma, self.alpha, self.do_precess = float(Ms), float(gamma), float(alpha), float(do_precess)
        self.precision = precision
        self._kw = dict(Aex=0.0, Ku=0.0, n_ani_vec=None, D_int=0.0, n0_int_vec=None, H0_static=None, Ku_nodes=None)
        self._demag = None
        self.hef = None

    def add_exchange(self, Aex):
        self._kw["Aex"] = float(Aex)

    def add_demag(self, method="lindholm", **kwargs):
        self._demag = dict(kwargs)

    def add_anisotropy(self, Ku, n_vec):
        self._kw.update(Ku=float(Ku), n_ani_vec=n_vec)

    add_uniaxial_anisotropy = add_anisotropy

    def add_dmi_interfacial(self, D_int, n0_vec):
        self._kw.update(D_int=float(D_int), n0_int_vec=n0_vec)

    def add_dmi_bulk(self, D_bulk):
        self._kw["D_bulk"] = float(D_bulk)

    def add_cubic_anisotropy(self, Kc1, u1_vec, u2_vec):
        raise NotImplementedError("cubic anisotropy is not part of this build")

    def add_external_field(self, H0_vec=None, H_time_func=None):
        """Static field and, optionally, H_time_func evaluated at the field object's
        current_time, which the minimiser keeps fixed (llg_module_GPU.py:1185-1194)."""
        self._kw["H0_static"] = H0_vec
        self._kw["H_time_func"] = H_time_func
        if self.hef is not None:
            self.hef.H_time_func = H_time_func
            self.hef._ht_time = None
        if self.hef is not None and H0_vec is not None:
            self.hef.set_uniform_field(*np.asarray(H0_vec, dtype=np.float64).reshape(3))

    def set_uniform_field(self, Hx, Hy, Hz):
        self._kw["H0_static"] = [float(Hx), float(Hy), float(Hz)]
        if self.hef is not None:
            self.hef.set_uniform_field(Hx, Hy, Hz)

    def _build(self):
        from .llg import EffectiveField
        if self.hef is None:
            self.hef = EffectiveField(self.X, self.tets, self.Ms, gamma=self.gamma, alpha=self.alpha,
                                      do_precess=self.do_precess, use_demag=self._demag is not None,
                                      demag_kwargs=self._demag, precision=self.precision, **self._kw)
        return self.hef

    def minimize(self, m0_array=None, method="labonte", max_iter=3000, tol=1.0, print_every=25, verbose=False,
                 **kwargs):
        """Returns (m as a CUDA tensor, stats, elapsed seconds)."""
        import torch
        if str(method).lower().replace("-", "_") not in ("labonte", "labonte_bb", "bb", "minimize"):
            raise ValueError(f"Unsupported GPU minimization method {method!r}. Use method='labonte'.")
        hef = self._build()
        if m0_array is not None:
            hef.set_state(torch.as_tensor(np.asarray(m0_array, dtype=np.float64).ravel(), device="cuda"))
        hef._sync_time_field()
        t0 = time.perf_counter()
        alg = LaBonteBBMinimizerGPU(hef)
        stats = alg.minimize(max_iter=max_iter, tol=tol, print_every=print_every, verbose=verbose, **kwargs)
        torch.cuda.synchronize()
        return hef.get_state(), stats, time.perf_counter() - t0

    def hysteresis(self, m0_array, H_steps, method="labonte", max_iter=3000, tol=1.0, **kwargs):
        """Quasistatic loop (:1216-1400): relax at each applied field, continuing from the last state.
        Returns a list of (H, <m>, stats)."""
        out = []
        m = m0_array
        for H in np.asarray(list(H_steps), dtype=np.float64).reshape(-1, 3):
            self.set_uniform_field(*H)
            y, st, _ = self.minimize(m, method=method, max_iter=max_iter, tol=tol, **kwargs)
            m = None
            out.append((H.copy(), y.reshape(-1, 3).mean(dim=0).cpu().numpy(), st))
        return out
