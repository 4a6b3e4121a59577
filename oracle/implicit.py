"""Implicit relaxation: variable-step BDF(2) with Newton-Krylov stage solves.

Test infrastructure (the oracle): FP64 numpy restatement of the reference's implicit driver
LLG_GPU.relax / _ensure_solver (gpu/solvers/llg_module_GPU.py:2052-2381).  The reference
hands the problem to PETSc:

* TS "bdf" (order 2), IFunction F = ydot - f(t, y) (EffectiveField.ifunction, :1328-1340);
* TSAdapt "basic": clip (0.1, 3.0), safety 0.9, reject safety 0.1, scale 0.25 after a failed
  nonlinear solve, dt in [1e-17, 1e-10] (:2074-2081); ExactFinalTime STEPOVER;
* SNES newtonls, line search "bt" of order 2 (quadratic backtracking), rtol 1e-2,
  atol 1e-4, at most 8 iterations (:2082-2088);
* KSP gmres, rtol 1e-4, at most 200 iterations (:2089-2093, 2110-2111), left preconditioned by
  the python PC of JvContext (:1412-1547): the per-node inverse of (shift I - J_i), rebuilt in
  every IJacobian call together with the Jacobian state (update_jac_state, :1287-1290);
* operator y = shift x - J(m) x (JvContext.mult, :1510-1517), J from _JAC_VEC_KERNEL with the
  field derivative of compute_H_jac_vec / apply_jacobian_field_vec (no demag, :860-884);
* the dm/dt stopper StopByMaxDmdtFDGPU (:314-382) after every step.

PETSc is not in this image, so this file states the algorithms as published and is the
specification both implementations follow; step-for-step agreement with PETSc itself is
unpinned.  The pieces:

* variable-step BDF through the Lagrange polynomial on the step's nodes: ydot(t_{n+1}) =
  sum_j L_j'(t_{n+1}) y_j, so shift = L_0'(t_{n+1}) and the rest is a fixed vector;
* the predictor (Newton's initial guess) extrapolates the polynomial through the last k+1
  points; a start (no history) first takes a backward-Euler half step to t + dt/2 and uses it
  as the second point (PETSc TSBDF's restart);
* the local error estimate is (dt / (t_{n+1} - t_oldest)) (y_{n+1} - y_pred) with t_oldest the
  predictor's oldest node (1 / (k+1) at constant steps, the BDF-k residual error constant,
  Shampine & Reichelt, "The MATLAB ODE suite", SIAM J. Sci. Comput. 18 (1997) 1-22), measured
  in the weighted RMS norm with tol_i = atol + rtol max(|y_{n+1,i}|, |y_{n,i}|); the adaptor's
  order is k+1;
* Newton with quadratic backtracking (Dennis & Schnabel, "Numerical Methods for Unconstrained
  Optimization and Nonlinear Equations", 1983, section 6.3, sufficient-decrease constant 1e-4,
  step fraction clipped to [0.1, 0.5]); convergence on ||F|| < atol, ||F|| <= rtol ||F_0|| or
  ||dy|| < 1e-8 ||y||;
* restarted GMRES(30) (Saad & Schultz 1986) from a zero guess: classical Gram-Schmidt, Givens
  rotations, convergence on the preconditioned residual <= max(rtol ||P^-1 F||, atol), the
  explicit residual recomputed at each restart.
"""
from __future__ import annotations

import math

import numpy as np

from . import llg as ollg

# convergence / divergence codes (signs and meanings follow PETSc's enums)
KSP_CONVERGED_RTOL, KSP_CONVERGED_ATOL, KSP_CONVERGED_HAPPY = 2, 3, 5
KSP_DIVERGED_ITS, KSP_DIVERGED_DTOL, KSP_DIVERGED_NAN, KSP_DIVERGED_NULL = -3, -4, -9, -2
SNES_CONVERGED_FNORM_ABS, SNES_CONVERGED_FNORM_RELATIVE, SNES_CONVERGED_SNORM = 2, 3, 4
SNES_DIVERGED_LINEAR_SOLVE, SNES_DIVERGED_FNORM_NAN, SNES_DIVERGED_MAX_IT = -3, -4, -5
SNES_DIVERGED_LINE_SEARCH, SNES_DIVERGED_DTOL = -6, -10

DEFAULTS = dict(snes_rtol=1e-2, snes_atol=1e-4, snes_stol=1e-8, snes_max_it=8, snes_divtol=1e4,
                ksp_rtol=1e-4, ksp_atol=1e-50, ksp_dtol=1e5, ksp_max_it=200, ksp_restart=30,
                ls_alpha=1e-4, ls_minlambda=1e-12, ls_maxstep=1e8, ls_max_it=40, use_pc=True)


def lagrange_values(x, ts):
    """L_j(x) on the nodes ts."""
    n = len(ts)
    out = []
    for j in range(n):
        v = 1.0
        for m in range(n):
            if m != j:
                v *= (x - ts[m]) / (ts[j] - ts[m])
        out.append(v)
    return out


def lagrange_derivs(x, ts):
    """L_j'(x) on the nodes ts."""
    n = len(ts)
    out = []
    for j in range(n):
        d = 0.0
        for m in range(n):
            if m == j:
                continue
            p = 1.0 / (ts[j] - ts[m])
            for q in range(n):
                if q != j and q != m:
                    p *= (x - ts[q]) / (ts[j] - ts[q])
            d += p
        out.append(d)
    return out


def gmres_left(A, P, b, rtol, atol, dtol, max_it, restart, haptol=1e-30):
    """Left-preconditioned restarted GMRES from x = 0: (x, iterations, reason)."""
    x = np.zeros_like(b)
    r = P(b)
    its, reason, rnorm0, ttol = 0, 0, None, None
    while True:
        beta = float(np.linalg.norm(r))
        if rnorm0 is None:
            rnorm0 = beta
            ttol = max(rtol * rnorm0, atol)
        if not math.isfinite(beta):
            return x, its, KSP_DIVERGED_NAN
        if beta <= ttol:
            return x, its, KSP_CONVERGED_ATOL if beta <= atol else KSP_CONVERGED_RTOL
        if beta >= dtol * rnorm0:
            return x, its, KSP_DIVERGED_DTOL
        V = [r / beta]
        Hh = np.zeros((restart + 1, restart))
        cs, sn = np.zeros(restart), np.zeros(restart)
        g = np.zeros(restart + 1)
        g[0] = beta
        loc = 0
        while reason == 0 and loc < restart and its < max_it:
            w = P(A(V[loc]))
            h = np.array([float(np.dot(V[i], w)) for i in range(loc + 1)])
            for i in range(loc + 1):
                w = w - h[i] * V[i]
            tt = float(np.linalg.norm(w))
            Hh[:loc + 1, loc] = h
            Hh[loc + 1, loc] = tt
            hapbnd = min(abs(tt / g[loc]), haptol)
            hapend = tt < hapbnd
            if not hapend:
                V.append(w / tt if tt > 0.0 else np.zeros_like(w))
            for i in range(loc):        # previous rotations on the new column
                a0, a1 = Hh[i, loc], Hh[i + 1, loc]
                Hh[i, loc] = cs[i] * a0 + sn[i] * a1
                Hh[i + 1, loc] = cs[i] * a1 - sn[i] * a0
            if not hapend:
                a0, a1 = Hh[loc, loc], Hh[loc + 1, loc]
                d = math.sqrt(a0 * a0 + a1 * a1)
                if d == 0.0:
                    reason = KSP_DIVERGED_NULL
                    break
                cs[loc], sn[loc] = a0 / d, a1 / d
                g[loc + 1] = -(sn[loc] * g[loc])
                g[loc] = cs[loc] * g[loc]
                Hh[loc, loc] = cs[loc] * a0 + sn[loc] * a1
                res = abs(g[loc + 1])
            else:
                res = 0.0
            loc += 1
            its += 1
            if not math.isfinite(res):
                reason = KSP_DIVERGED_NAN
            elif res <= ttol:
                reason = KSP_CONVERGED_ATOL if res <= atol else KSP_CONVERGED_RTOL
            elif res >= dtol * rnorm0:
                reason = KSP_DIVERGED_DTOL
            if hapend:
                if reason == 0:
                    reason = KSP_CONVERGED_HAPPY
                break
        if loc > 0 and reason != KSP_DIVERGED_NULL:   # x += V y, H y = g (back substitution)
            y = np.zeros(loc)
            for k in range(loc - 1, -1, -1):
                s = g[k]
                for j in range(k + 1, loc):
                    s -= Hh[k, j] * y[j]
                y[k] = s / Hh[k, k]
            for j in range(loc):
                x = x + y[j] * V[j]
        if reason != 0:
            return x, its, reason
        if its >= max_it:
            return x, its, KSP_DIVERGED_ITS
        r = P(b - A(x))


class StageProblem:
    """F(y) = shift y + base - f(t1, y) with the Jacobian pieces of the LLG right-hand side."""

    def __init__(self, hef, t1, shift, base, use_pc=True):
        self.hef, self.t1, self.shift, self.base, self.use_pc = hef, t1, shift, base, use_pc
        self.fevals = 0
        self.Mstate = self.Hm = self.inv = None

    def F(self, y):
        self.fevals += 1
        return self.shift * y + self.base - self.hef.llg_rhs(y, self.t1)

    def setup(self, y):
        """IJacobian: Jacobian state at y and the block preconditioner for the shift."""
        h = self.hef
        self.Mstate = y.copy()
        self.Hm = h.h_jac(y, self.t1)
        if self.use_pc:
            c1 = h.gamma * h.do_precess / (1.0 + h.alpha * h.alpha)
            c2 = h.gamma * h.alpha / (1.0 + h.alpha * h.alpha)
            self.inv = ollg.pc_build(self.Mstate, self.Hm, h.diagK, self.shift, c1, c2, h.stab)

    def A(self, v):
        h = self.hef
        return self.shift * v - ollg.jv(self.Mstate, self.Hm, v, h.linear(v), h.gamma, h.alpha, h.do_precess, h.stab)

    def P(self, v):
        return ollg.pc_apply(self.inv, v) if self.use_pc else v.copy()


def line_search_bt(pb, y, F, fnorm, Y, o):
    """Quadratic backtracking: (ok, y_new, F_new, fnorm_new, xnorm, ynorm)."""
    xnorm, ynorm = float(np.linalg.norm(y)), float(np.linalg.norm(Y))
    if ynorm == 0.0:
        return False, y, F, fnorm, xnorm, ynorm
    if ynorm > o["ls_maxstep"]:
        Y = Y * (o["ls_maxstep"] / ynorm)
        ynorm = o["ls_maxstep"]
    f = fnorm * fnorm
    slope = float(np.dot(F, pb.A(Y)))
    if slope > 0.0:
        slope = -slope
    if slope == 0.0:
        slope = -1.0
    alpha, lam = o["ls_alpha"], 1.0
    w = y - lam * Y
    G = pb.F(w)
    g = float(np.dot(G, G))
    if not math.isfinite(g):
        return False, w, G, math.sqrt(g) if g >= 0 else g, xnorm, ynorm
    if 0.5 * g <= 0.5 * f + lam * alpha * slope:
        return True, w, G, math.sqrt(g), float(np.linalg.norm(w)), ynorm
    if o["snes_stol"] * xnorm > ynorm:
        return False, w, G, math.sqrt(g), xnorm, ynorm
    for _ in range(o["ls_max_it"] + 1):
        if lam <= o["ls_minlambda"]:
            return False, w, G, math.sqrt(g), xnorm, ynorm
        lt = -slope * lam * lam / (g - f - 2.0 * lam * slope)
        if lt > 0.5 * lam:
            lt = 0.5 * lam
        lam = 0.1 * lam if lt <= 0.1 * lam else lt
        w = y - lam * Y
        G = pb.F(w)
        g = float(np.dot(G, G))
        if not math.isfinite(g):
            return False, w, G, g, xnorm, ynorm
        if 0.5 * g < 0.5 * f + lam * alpha * slope:
            return True, w, G, math.sqrt(g), float(np.linalg.norm(w)), ynorm
    return False, w, G, math.sqrt(g), xnorm, ynorm


def newton_solve(pb, y0, o):
    """SNES newtonls on pb from y0: (y, reason, newton iterations, linear iterations)."""
    y = y0.copy()
    F = pb.F(y)
    fnorm = float(np.linalg.norm(F))
    if not math.isfinite(fnorm):
        return y, SNES_DIVERGED_FNORM_NAN, 0, 0
    fnorm0, ttol = fnorm, fnorm * o["snes_rtol"]
    if fnorm < o["snes_atol"]:
        return y, SNES_CONVERGED_FNORM_ABS, 0, 0
    lin = 0
    for i in range(o["snes_max_it"]):
        pb.setup(y)
        Y, lits, kr = gmres_left(pb.A, pb.P, F, o["ksp_rtol"], o["ksp_atol"], o["ksp_dtol"], o["ksp_max_it"],
                                 o["ksp_restart"])
        lin += lits
        if kr < 0 and kr != KSP_DIVERGED_ITS:
            return y, SNES_DIVERGED_LINEAR_SOLVE, i + 1, lin
        ok, y, F, fnorm, xnorm, ynorm = line_search_bt(pb, y, F, fnorm, Y, o)
        if not ok:
            if o["snes_stol"] * xnorm > ynorm:
                return y, SNES_CONVERGED_SNORM, i + 1, lin
            return y, SNES_DIVERGED_LINE_SEARCH, i + 1, lin
        if not math.isfinite(fnorm):
            return y, SNES_DIVERGED_FNORM_NAN, i + 1, lin
        if fnorm < o["snes_atol"]:
            return y, SNES_CONVERGED_FNORM_ABS, i + 1, lin
        if fnorm <= ttol:
            return y, SNES_CONVERGED_FNORM_RELATIVE, i + 1, lin
        if ynorm < o["snes_stol"] * xnorm:
            return y, SNES_CONVERGED_SNORM, i + 1, lin
        if fnorm > o["snes_divtol"] * fnorm0:
            return y, SNES_DIVERGED_DTOL, i + 1, lin
    return y, SNES_DIVERGED_MAX_IT, o["snes_max_it"], lin


class BDFOracle:
    """History, stage solves and error estimate of the BDF(2) driver; the state is (t, m)."""

    def __init__(self, hef, m0, t0=0.0, rtol=1e-6, atol=1e-6, **opts):
        self.hef = hef
        self.m = np.asarray(m0, dtype=np.float64).copy()
        self.current_time = float(t0)
        self.rtol, self.atol = float(rtol), float(atol)
        self.o = dict(DEFAULTS, **opts)
        self.hist = []          # [(t, y)] past points, newest first (at most 2)
        self.cand = None
        self.newton_its = self.linear_its = self.fevals = 0

    def reset(self):
        self.hist = []

    def _stage(self, t1, nodes, pred_nodes):
        """Solve the BDF equation at t1 over nodes [(t, y)] from the predictor through pred_nodes."""
        ts = [t1] + [p[0] for p in nodes]
        a = lagrange_derivs(t1, ts)
        base = np.zeros_like(self.m)
        for aj, (_, yj) in zip(a[1:], nodes):
            base = base + aj * yj
        lv = lagrange_values(t1, [p[0] for p in pred_nodes])
        ypred = np.zeros_like(self.m)
        for lj, (_, yj) in zip(lv, pred_nodes):
            ypred = ypred + lj * yj
        pb = StageProblem(self.hef, t1, a[0], base, self.o["use_pc"])
        y, reason, nits, lits = newton_solve(pb, ypred, self.o)
        self.newton_its += nits
        self.linear_its += lits
        self.fevals += pb.fevals
        return y, ypred, reason

    def attempt(self, dt):
        t, m = self.current_time, self.m
        t1 = t + dt
        restarted = not self.hist
        if restarted:
            th = t + 0.5 * dt
            yh, _, reason = self._stage(th, [(t, m)], [(t, m)])
            if reason < 0:
                self.cand = None
                return {"snes_reason": reason, "wlte": -1.0, "order": 2, "restarted": True}
            nodes = [(th, yh), (t, m)]
            pred = nodes
        else:
            nodes = [(t, m), self.hist[0]]
            pred = [(t, m)] + self.hist[:2]
        y, ypred, reason = self._stage(t1, nodes, pred)
        if reason < 0:
            self.cand = None
            return {"snes_reason": reason, "wlte": -1.0, "order": len(pred), "restarted": restarted}
        t_old = min(p[0] for p in pred)
        lte = (dt / (t1 - t_old)) * (y - ypred)
        tol = self.atol + self.rtol * np.maximum(np.abs(y), np.abs(m))
        wlte = float(np.sqrt(np.mean((lte / tol) ** 2)))
        self.cand = (t1, y, nodes if restarted else None)
        return {"snes_reason": reason, "wlte": wlte, "order": len(pred), "restarted": restarted}

    def accept(self):
        t1, y, rnodes = self.cand
        if rnodes is not None:
            self.hist = list(rnodes)
        else:
            self.hist = [(self.current_time, self.m)] + self.hist[:1]
        self.m, self.current_time = y, t1
        self.cand = None

    def get_state(self):
        return self.m


def adapt_choose(h, enorm, order, accept_prev, clip=(0.1, 3.0), safety=0.9, reject_safety=0.1, dt_min=1e-17,
                 dt_max=1e-10):
    """TSAdapt basic: (accept, next h)."""
    if enorm < 0.0:
        return True, min(max(h, dt_min), dt_max)
    s = safety
    if enorm > 1.0:
        if not accept_prev:
            s *= reject_safety
        accept = h < (1.0 + 1.4901161193847656e-08) * dt_min
    else:
        accept = True
    hfac = s * enorm ** (-1.0 / order) if enorm > 0.0 else float("inf")
    hfac = min(max(hfac, clip[0]), clip[1])
    return accept, min(max(h * hfac, dt_min), dt_max)


def relax_implicit(hef, m0, t0, t_final, dt_init, rtol=1e-6, atol=1e-6, stopping_dmdt=0.0, check_every=10,
                   max_steps=10 ** 7, max_reject=10, **opts):
    """The implicit relaxation loop: (m, stats) with stats t_end, nsteps, reason (1 final time,
    2 dm/dt below the threshold, -2 too many rejections in one step), rejected, snes_failures,
    newton_its, linear_its, fevals, dts."""
    bdf = BDFOracle(hef, m0, t0, rtol, atol, **opts)
    dt = min(max(float(dt_init), 1e-17), 1e-10)
    steps = rejected = failures = reason = 0
    dts = []
    u_prev, t_prev, last = None, None, float("nan")
    while steps < max_steps:
        if bdf.current_time >= t_final:
            reason = 1
            break
        accept_prev, nrej, nxt = True, 0, dt
        while True:
            r = bdf.attempt(dt)
            if r["snes_reason"] < 0:
                failures += 1
                accept = False
                nxt = dt * 0.25
            else:
                accept, nxt = adapt_choose(dt, r["wlte"], r["order"], accept_prev)
            if accept:
                break
            rejected += 1
            nrej += 1
            accept_prev = False
            dt = nxt
            if nrej > max_reject:
                reason = -2
                break
        if reason == -2:
            break
        bdf.accept()
        dts.append(dt)
        steps += 1
        t = bdf.current_time
        stop = False
        if stopping_dmdt > 0.0 and (check_every <= 1 or steps % check_every == 0):
            if t_prev is None or t - t_prev <= 0.0:
                u_prev, t_prev = bdf.m.copy(), t
            else:
                du = (bdf.m - u_prev).reshape(-1, 3)
                last = float(np.sqrt((du * du).sum(axis=1)).max()) / (t - t_prev) * (180.0 / np.pi) * 1e-9
                u_prev, t_prev = bdf.m.copy(), t
                stop = last < stopping_dmdt
        dt = nxt
        if stop:
            reason = 2
            break
    return bdf.m, {"t_end": bdf.current_time, "dt_last": dt, "nsteps": steps, "reason": reason,
                   "rejected": rejected, "snes_failures": failures, "newton_its": bdf.newton_its,
                   "linear_its": bdf.linear_its, "fevals": bdf.fevals, "dts": dts, "maxdmdt_deg_ns": last}
