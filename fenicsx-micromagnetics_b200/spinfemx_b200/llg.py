"""Effective field, LLG right-hand side, Jv, block preconditioner and driver.

Mirrors ``gpu/solvers/llg_module_GPU.py``:

* ``EffectiveField`` (:387-1408): ``compute_H_eff_vec``, ``compute_H_jac_vec``,
  ``llg_rhs_vec``, ``update_jac_state``, ``jac_vec_times_vec``,
  ``apply_jacobian_field_vec``, ``set_uniform_field``, ``rhs_function``,
  ``ifunction`` and the ``LLGSteps`` / ``JacSteps`` counters;
* ``JvContext`` (:1412-1543): ``update_pc_full_fast_gpu``, ``mult``, ``apply``;
* ``LLG_GPU`` (:1549): ``add_exchange``, ``add_demag``, ``add_anisotropy``,
  ``add_dmi_interfacial``, ``add_external_field`` and ``run_fixed`` (classic RK4 at a
  fixed step; the reference drives PETSc TS rk/5dp or BDF instead).

Vectors are CUDA float64 torch tensors of length 3N (AoS).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call, ptr
from .demag import DemagFieldLindholmGPU
from .geometry import as_mesh


def _vec3(a, N, name):
    if a is None:
        return None
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))
    if a.size == 3:
        a = np.tile(a, N)
    if a.size != 3 * N:
        raise ValueError(f"{name} must have 3 or 3N entries")
    return a


# Dormand-Prince 5(4) stage times (fractions of the step), see csrc/drivers.cu
DP5_C = (0.0, 0.2, 0.3, 0.8, 8.0 / 9.0, 1.0, 1.0)
RK4_C = (0.0, 0.5, 0.5, 1.0)


class EffectiveField:
    def __init__(self, X, tets, Ms, Aex=0.0, Ku=0.0, n_ani_vec=None, D_bulk=0.0, D_int=0.0, n0_int_vec=None,
                 gamma=2.211e5, alpha=0.5, do_precess=1, use_demag=False, demag_method="lindholm",
                 demag_kwargs=None, H0_static=None, Ku_nodes=None, precision="f64", H_time_func=None,
                 _stt=None, _sot=None):
        if str(demag_method).lower() not in {"lindholm", "lindholm_gpu"}:
            raise NotImplementedError("only the Lindholm FEM/BEM demag method is implemented")
        X, tets = as_mesh(X, tets)
        self.X, self.tets = X, tets
        self.N = X.shape[0]
        self.local_dofs = self.N
        self.local_size = 3 * self.N
        self.Ms, self.gamma, self.alpha = float(Ms), float(gamma), float(alpha)
        self.do_precess = float(do_precess)
        self.A, self.Ku, self.D_int, self.D_bulk = float(Aex), float(Ku), float(D_int), float(D_bulk)
        self.prefactorEQ = -self.gamma / (1.0 + self.alpha ** 2)
        self.Stab = self.Ms * self.gamma / (1.0 + self.alpha ** 2) * 0.5
        self.LLGSteps = 0
        self.JacSteps = 0
        self.current_time = 0.0
        self.H_time_func = H_time_func
        self._ht_time = None  # time of the field last handed to the library
        self.demag_field = None
        if use_demag:
            kw = dict(demag_kwargs or {})
            kw.setdefault("precision", precision)
            self.demag_field = DemagFieldLindholmGPU(X, tets, self.Ms, **kw)
            precision = self.demag_field.precision
        self.precision = precision
        self._keep = []
        p = _lib.LLGParams()
        p.Ms, p.gamma, p.alpha, p.do_precess = self.Ms, self.gamma, self.alpha, self.do_precess
        p.Aex, p.Ku, p.D_int, p.D_bulk = self.A, self.Ku, self.D_int, self.D_bulk
        n_ani = _vec3(n_ani_vec, self.N, "n_ani_vec")
        n_int = _vec3(n0_int_vec, self.N, "n0_int_vec")
        H0 = _vec3(H0_static, self.N, "H0_static")
        kun = None if Ku_nodes is None else np.ascontiguousarray(Ku_nodes, dtype=np.float64).reshape(-1)
        if kun is not None and kun.size != self.N:
            raise ValueError("Ku_nodes must have N entries")
        if (self.Ku != 0.0 or kun is not None) and n_ani is None:
            raise ValueError("anisotropy needs n_ani_vec")
        for a in (n_ani, n_int, H0, kun):
            if a is not None:
                self._keep.append(a)
        p.n_ani = ptr(n_ani).value if n_ani is not None and (self.Ku != 0.0 or kun is not None) else None
        p.Ku_nodes = ptr(kun).value if kun is not None else None
        p.n_int = ptr(n_int).value if n_int is not None and self.D_int != 0.0 else None
        p.H0_nodes = ptr(H0).value if H0 is not None else None
        self._H0 = H0 if H0 is not None else np.zeros(3 * self.N)
        p.use_demag = 1 if use_demag else 0
        p.precision = _lib.PREC[precision]
        if _stt is not None:  # (J, P, beta, direction [3N])
            jd = _vec3(_stt[3], self.N, "Jdir_vec")
            self._keep.append(jd)
            p.stt_J, p.stt_P, p.stt_beta, p.stt_dir = float(_stt[0]), float(_stt[1]), float(_stt[2]), ptr(jd).value
        if _sot is not None:  # (H_dl, H_fl, polarisation [3N])
            pv = _vec3(_sot[2], self.N, "polarization_vec")
            self._keep.append(pv)
            p.sot_Hdl, p.sot_Hfl, p.sot_p = float(_sot[0]), float(_sot[1]), ptr(pv).value
        self._h = C.c_void_p()
        dh = self.demag_field.handle if self.demag_field is not None else None
        call("spx_llg_create", dh, ptr(X), self.N, ptr(tets), tets.shape[0], C.byref(p), C.byref(self._h))
        self._H0_dev = None

    # -------------------------------------------------------------- helpers
    def _chk(self, v, name):
        import torch
        if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float64 and v.is_contiguous()):
            raise TypeError(f"{name} must be a contiguous CUDA float64 tensor")
        if v.numel() < self.local_size:
            raise RuntimeError(f"{name} needs {self.local_size} entries")

    def _tail(self, v):
        if v.numel() > self.local_size:
            v[self.local_size:] = 0.0

    @property
    def handle(self):
        return self._h

    # -------------------------------------------------------------- fields
    def set_uniform_field(self, Hx, Hy, Hz):
        call("spx_llg_set_uniform_field", self._h, float(Hx), float(Hy), float(Hz))
        self._H0 = np.tile([float(Hx), float(Hy), float(Hz)], self.N)
        self._H0_dev = None

    # -------------------------------------------------------------- time-dependent field
    def _eval_H_time(self, t):
        """H_time_func at time t as (uniform [3] numpy or None, nodal [3N] CUDA float64 or None):
        the callback is tried as f(t, x) with the mesh coordinates, then as f(t); it may return
        (3,), (3N,) or (N, 3), as numpy or torch (llg_module_GPU.py:909-956)."""
        import torch
        try:
            out = self.H_time_func(float(t), self.X)
        except TypeError:
            out = self.H_time_func(float(t))
        if isinstance(out, torch.Tensor):
            arr = out.detach().to(dtype=torch.float64)
            if arr.numel() == 3:
                return arr.cpu().numpy().reshape(3).copy(), None
            if arr.numel() == 3 * self.N and (arr.dim() == 1 or tuple(arr.shape) == (self.N, 3)):
                return None, arr.reshape(-1).to("cuda").contiguous()
            raise ValueError(f"Unsupported torch H_time_func shape {tuple(arr.shape)}")
        arr = np.asarray(out, dtype=np.float64)
        if arr.ndim == 1 and arr.size == 3:
            return arr.copy(), None
        if (arr.ndim == 1 and arr.size == 3 * self.N) or arr.shape == (self.N, 3):
            return None, torch.as_tensor(np.ascontiguousarray(arr.reshape(-1)), device="cuda")
        raise ValueError("H_time_func must return (3,), (local_size,), or (local_dofs, 3) values.")

    def _sync_time_field(self):
        """Hand H_time_func(current_time) to the library before an evaluation."""
        if self.H_time_func is None:
            if self._ht_time is not None:  # a callback was removed: clear its field
                call("spx_llg_set_time_field", self._h, None, None, _lib.stream_ptr())
                self._ht_time = None
            return
        if self._ht_time == self.current_time:
            return
        u, n = self._eval_H_time(self.current_time)
        call("spx_llg_set_time_field", self._h, ptr(u), ptr(n), _lib.stream_ptr())
        self._ht_time = self.current_time

    def _stage_fields(self, t, dt, cs):
        """Per-stage values of H_time_func at t + c dt: (uniform [len(cs)][3] host, nodal
        [len(cs)][3N] CUDA) with None where the callback gives no such part."""
        import torch
        vals = {}
        for c in cs:
            if c not in vals:
                vals[c] = self._eval_H_time(t + c * dt)
        if any(v[1] is not None for v in vals.values()):
            nod = torch.zeros((len(cs), self.local_size), dtype=torch.float64, device="cuda")
            for i, c in enumerate(cs):
                if vals[c][1] is not None:
                    nod[i] = vals[c][1]
        else:
            nod = None
        uni = np.zeros((len(cs), 3))
        for i, c in enumerate(cs):
            if vals[c][0] is not None:
                uni[i] = vals[c][0]
        return np.ascontiguousarray(uni), nod

    def compute_H_eff_vec(self, m_vec, out_vec):
        self._chk(m_vec, "m_vec")
        self._chk(out_vec, "out_vec")
        self._sync_time_field()
        call("spx_llg_heff", self._h, ptr(m_vec), ptr(out_vec), _lib.stream_ptr())
        self._tail(out_vec)

    def compute_H_jac_vec(self, m_vec, out_vec):
        self._chk(m_vec, "m_vec")
        self._chk(out_vec, "out_vec")
        self._sync_time_field()
        call("spx_llg_hjac", self._h, ptr(m_vec), ptr(out_vec), _lib.stream_ptr())
        self._tail(out_vec)

    def apply_jacobian_field_vec(self, m_state_vec, v_vec, out_vec):
        """dH_eff/dm v for the linear terms (exchange, anisotropy, DMI); no demag, no H0."""
        import torch
        self.compute_H_jac_vec(v_vec, out_vec)
        if self._H0_dev is None:
            self._H0_dev = torch.as_tensor(self._H0, device=out_vec.device)
        out_vec[: self.local_size] -= self._H0_dev

    def llg_rhs_vec(self, m_vec, out_vec):
        self.LLGSteps += 1
        self._chk(m_vec, "m_vec")
        self._chk(out_vec, "out_vec")
        self._sync_time_field()
        call("spx_llg_rhs", self._h, ptr(m_vec), ptr(out_vec), _lib.stream_ptr())
        self._tail(out_vec)

    def update_jac_state(self, m_vec):
        self._chk(m_vec, "m_vec")
        self._sync_time_field()
        call("spx_llg_update_jac_state", self._h, ptr(m_vec), _lib.stream_ptr())

    def jac_vec_times_vec(self, v_vec, out_vec):
        self.JacSteps += 1
        self._chk(v_vec, "v_vec")
        self._chk(out_vec, "out_vec")
        call("spx_llg_jv", self._h, ptr(v_vec), ptr(out_vec), _lib.stream_ptr())
        self._tail(out_vec)

    # PETSc TS callback shapes (llg_module_GPU.py:1328-1339, 1403-1408)
    def rhs_function(self, ts, t, y, f):
        self.current_time = float(t)
        self.llg_rhs_vec(y, f)
        return 0

    def ifunction(self, ts, t, y, ydot, f):
        import torch
        self.current_time = float(t)
        r = torch.empty_like(f)
        self.llg_rhs_vec(y, r)
        f.copy_(ydot - r)
        return 0

    # -------------------------------------------------------------- integrator
    def set_state(self, m_vec):
        self._chk(m_vec, "m_vec")
        call("spx_llg_set_state", self._h, ptr(m_vec), _lib.stream_ptr())

    def get_state(self, out_vec=None):
        import torch
        if out_vec is None:
            out_vec = torch.empty(self.local_size, dtype=torch.float64, device="cuda")
        call("spx_llg_get_state", self._h, ptr(out_vec), _lib.stream_ptr())
        return out_vec

    def step(self, dt, nsteps=1):
        """nsteps classic RK4 steps of size dt from the state; with H_time_func the field is
        evaluated at each stage time (t, t + dt/2, t + dt) and current_time advances."""
        if self.H_time_func is None:
            call("spx_llg_step", self._h, float(dt), int(nsteps), _lib.stream_ptr())
            return
        for _ in range(int(nsteps)):
            u, n = self._stage_fields(self.current_time, float(dt), RK4_C)
            call("spx_llg_step_time_field", self._h, float(dt), ptr(u), ptr(n), _lib.stream_ptr())
            self.current_time += float(dt)

    def rk_attempt(self, dt, rtol, atol, reuse_fsal=True):
        """One Dormand-Prince 5(4) attempt of size dt at current_time (not committed); returns
        the weighted RMS norm of the embedded error (<= 1: acceptable)."""
        u = n = None
        if self.H_time_func is not None:
            u, n = self._stage_fields(self.current_time, float(dt), DP5_C)
        e = _lib.c_dbl()
        call("spx_llg_rk_attempt", self._h, 0, float(dt), float(rtol), float(atol), ptr(u), ptr(n),
             1 if reuse_fsal else 0, C.byref(e), _lib.stream_ptr())
        return e.value

    def rk_accept(self, dt):
        call("spx_llg_rk_accept", self._h, _lib.stream_ptr())
        self.current_time += float(dt)

    def bdf_attempt(self, dt, opts):
        """One implicit BDF(2) attempt of size dt at current_time (spx_llg_bdf_attempt, not
        committed).  opts: a _lib.BdfOpts.  Returns a dict with snes_reason (< 0: the stage
        solve failed), wlte (weighted RMS local error estimate, < 0: none), order, restarted,
        newton_its, linear_its, fevals."""
        u = n = None
        if self.H_time_func is not None:
            u, n = self._stage_fields(self.current_time, float(dt), (0.5, 1.0))
        r = _lib.BdfResult()
        call("spx_llg_bdf_attempt", self._h, float(self.current_time), float(dt), C.byref(opts), ptr(u), ptr(n),
             C.byref(r), _lib.stream_ptr())
        return {k: getattr(r, k) for k, _ in _lib.BdfResult._fields_}

    def bdf_accept(self, dt):
        call("spx_llg_bdf_accept", self._h, _lib.stream_ptr())
        self.current_time += float(dt)
        self._ht_time = None   # the library holds the field of the last stage time

    def bdf_reset(self):
        call("spx_llg_bdf_reset", self._h)

    def set_graph(self, enable=True):
        """Replay each RK4 step from captured CUDA graphs (same results as ordinary steps)."""
        call("spx_llg_set_graph", self._h, 1 if enable else 0)

    def graph_stats(self):
        r, a = _lib.c_i64(), _lib.c_i32()
        call("spx_llg_graph_stats", self._h, C.byref(r), C.byref(a))
        return {"replayed_steps": r.value, "active": bool(a.value)}

    def run_host(self, m_host, dt, nsteps, out=None):
        """End-to-end call on host buffers (numpy or pinned torch CPU tensors)."""
        if out is None:
            out = np.empty_like(m_host)
        call("spx_llg_run_host", self._h, ptr(m_host), ptr(out), float(dt), int(nsteps))
        return out

    # -------------------------------------------------------------- gradients
    # Adjoint / tangent products (not in the reference).  gKu (N) and gH0 (3) are CUDA float64
    # accumulators that the calls add to.
    def set_anisotropy_map(self, Ku_nodes):
        """Replace the nodal Ku map (J/m^3); the anisotropy axis must have been given."""
        ku = np.ascontiguousarray(np.asarray(Ku_nodes, dtype=np.float64).reshape(-1))
        if ku.size != self.N:
            raise ValueError("Ku_nodes must have N entries")
        call("spx_llg_set_anisotropy_map", self._h, ptr(ku))

    def rhs_vjp(self, m_vec, w_vec, out_vec, gKu=None, gH0=None):
        """out = J(m)^T w, J the Jacobian of llg_rhs_vec at m (demag included)."""
        for v, n in ((m_vec, "m_vec"), (w_vec, "w_vec"), (out_vec, "out_vec")):
            self._chk(v, n)
        call("spx_llg_rhs_vjp", self._h, ptr(m_vec), ptr(w_vec), ptr(out_vec), ptr(gKu), ptr(gH0),
             _lib.stream_ptr())
        return out_vec

    def step_vjp(self, m_n, dt, lam_in, lam_out, gKu=None, gH0=None):
        """lam_out = (d m_(n+1) / d m_n)^T lam_in for one RK4 step from m_n."""
        for v, n in ((m_n, "m_n"), (lam_in, "lam_in"), (lam_out, "lam_out")):
            self._chk(v, n)
        call("spx_llg_step_vjp", self._h, ptr(m_n), float(dt), ptr(lam_in), ptr(lam_out), ptr(gKu), ptr(gH0),
             _lib.stream_ptr())
        return lam_out

    def step_jvp(self, m_n, dm, dt, m_out, dm_out, dKu=None, dH0=None):
        """One RK4 step of the state and its tangent along (dm, dKu, dH0)."""
        for v, n in ((m_n, "m_n"), (dm, "dm"), (m_out, "m_out"), (dm_out, "dm_out")):
            self._chk(v, n)
        h0 = None if dH0 is None else np.ascontiguousarray(np.asarray(dH0, dtype=np.float64).reshape(3))
        call("spx_llg_step_jvp", self._h, ptr(m_n), ptr(dm), ptr(dKu), ptr(h0), float(dt), ptr(m_out),
             ptr(dm_out), _lib.stream_ptr())
        return m_out, dm_out

    def stats(self):
        s, r, l = _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
        call("spx_llg_stats", self._h, C.byref(s), C.byref(r), C.byref(l))
        return {"steps": s.value, "rhs_evals": r.value, "launches": l.value}

    def __del__(self):
        try:
            h = getattr(self, "_h", None)
            if h is not None and h.value:
                try:
                    _lib.lib().spx_llg_destroy(h)
                except Exception:
                    pass
                self._h = C.c_void_p()
        except Exception:
            pass


class JvContext:
    """Matrix-free Jacobian context: y = shift x - J x, and the 3x3 block PC."""

    def __init__(self, hef: EffectiveField, eps_reg=1e-14, det_eps=1e-30):
        if eps_reg != 1e-14 or det_eps != 1e-30:
            raise ValueError("eps_reg=1e-14 and det_eps=1e-30 are fixed in this build")
        self.hef = hef
        self.shift = 0.0
        self.calls = 0
        self.callsPre = 0
        self._pc_ready = False
        import torch
        self._jv = torch.empty(hef.local_size, dtype=torch.float64, device="cuda")

    def update_pc_full_fast_gpu(self, shift, include_stab=True, use_abs_kappa=True):
        self.shift = float(shift)
        call("spx_llg_pc_build", self.hef.handle, self.shift, int(bool(include_stab)), int(bool(use_abs_kappa)),
             _lib.stream_ptr())
        self._pc_ready = True

    def mult(self, A, x, y):
        self.calls += 1
        self.hef.jac_vec_times_vec(x, self._jv)
        y.copy_(self.shift * x - self._jv)

    def apply(self, pc, x, y):
        self.callsPre += 1
        if not self._pc_ready:
            y.copy_(x)
            return
        call("spx_llg_pc_apply", self.hef.handle, ptr(x), ptr(y), _lib.stream_ptr())


class EffectiveFieldSTTGPU(EffectiveField):
    """EffectiveField with the Zhang-Li spin-transfer torque (gpu/solvers/llg_stt_module_GPU.py:523-1163).

    prefZhang = J P muB / (e Ms (1 + beta^2)) / (1 + alpha^2) / 1e-9; the RHS adds
    -prefZhang ((beta - alpha) m x z + (1 + alpha beta) m x (m x z)) with z = (J . grad) m / V_i.
    """

    def __init__(self, X, tets, Ms, Aex=0.0, Ku=0.0, n_ani_vec=None, D_bulk=0.0, D_int=0.0, n0_int_vec=None,
                 H0_static=None, gamma=2.211e5, alpha=0.5, do_precess=1, Jmagnitude=0.0, Jdir_vec=None, P=0.0,
                 beta=0.0, use_demag=False, demag_method="lindholm", demag_kwargs=None, H_time_func=None,
                 precision="f64", Ku_nodes=None):
        if Jdir_vec is None:
            raise ValueError("Jdir_vec is required")
        self.Jmagnitude, self.P, self.beta = float(Jmagnitude), float(P), float(beta)
        super().__init__(X, tets, Ms, Aex=Aex, Ku=Ku, n_ani_vec=n_ani_vec, D_bulk=D_bulk, D_int=D_int,
                         n0_int_vec=n0_int_vec, gamma=gamma, alpha=alpha, do_precess=do_precess,
                         use_demag=use_demag, demag_method=demag_method, demag_kwargs=demag_kwargs,
                         H0_static=H0_static, Ku_nodes=Ku_nodes, precision=precision, H_time_func=H_time_func,
                         _stt=(self.Jmagnitude, self.P, self.beta, Jdir_vec))
        e, muB = 1.6021766e-19, 9.27400915e-24
        self.prefZhang = (self.Jmagnitude * self.P * muB / (e * self.Ms * (1.0 + self.beta ** 2))
                          / (1.0 + self.alpha ** 2) / 1e-9)

    def zhang_li_vec(self, m_vec, out_vec):
        self._chk(m_vec, "m_vec")
        self._chk(out_vec, "out_vec")
        call("spx_llg_zhang_li", self._h, ptr(m_vec), ptr(out_vec), _lib.stream_ptr())
        self._tail(out_vec)

    def llg_rhs_STT_vec(self, m_vec, out_vec):
        self.llg_rhs_vec(m_vec, out_vec)

    def ifunction_STT(self, ts, t, y, ydot, f):
        return self.ifunction(ts, t, y, ydot, f)

    def update_jac_state_STT(self, m_vec):
        self.update_jac_state(m_vec)

    def jac_vec_times_STT_vec(self, v_vec, out_vec):
        self.jac_vec_times_vec(v_vec, out_vec)


class EffectiveFieldSOTGPU(EffectiveField):
    """EffectiveField with spin-orbit torques (gpu/solvers/llg_SOT_module_GPU.py:544-1150): the RHS adds
    c_fl m x p + c_dl m x (m x p), c_fl = -gamma (H_fl - alpha H_dl) / (1 + alpha^2),
    c_dl = -gamma (H_dl + alpha H_fl) / (1 + alpha^2)."""

    def __init__(self, X, tets, Ms, Aex=0.0, Ku=0.0, n_ani_vec=None, D_bulk=0.0, D_int=0.0, n0_int_vec=None,
                 H0_static=None, gamma=2.211e5, alpha=0.5, do_precess=1, H_dl=0.0, H_fl=0.0,
                 polarization_vec=None, use_demag=False, demag_method="lindholm", demag_kwargs=None,
                 H_time_func=None, precision="f64", Ku_nodes=None):
        pol = (0.0, 1.0, 0.0) if polarization_vec is None else polarization_vec
        super().__init__(X, tets, Ms, Aex=Aex, Ku=Ku, n_ani_vec=n_ani_vec, D_bulk=D_bulk, D_int=D_int,
                         n0_int_vec=n0_int_vec, gamma=gamma, alpha=alpha, do_precess=do_precess,
                         use_demag=use_demag, demag_method=demag_method, demag_kwargs=demag_kwargs,
                         H0_static=H0_static, Ku_nodes=Ku_nodes, precision=precision, H_time_func=H_time_func,
                         _sot=(float(H_dl), float(H_fl), pol))
        self.H_dl, self.H_fl = float(H_dl), float(H_fl)
        self._update_sot_coefficients()

    def _update_sot_coefficients(self):
        den = 1.0 + self.alpha * self.alpha
        self.c_fl = -self.gamma * (self.H_fl - self.alpha * self.H_dl) / den
        self.c_dl = -self.gamma * (self.H_dl + self.alpha * self.H_fl) / den

    def set_sot(self, H_dl=None, H_fl=None, polarization_vec=None):
        if H_dl is not None:
            self.H_dl = float(H_dl)
        if H_fl is not None:
            self.H_fl = float(H_fl)
        pv = None if polarization_vec is None else _vec3(polarization_vec, self.N, "polarization_vec")
        if pv is not None:
            self._keep.append(pv)
        call("spx_llg_set_sot", self._h, self.H_dl, self.H_fl, ptr(pv))
        self._update_sot_coefficients()

    def llg_rhs_SOT_vec(self, m_vec, out_vec):
        self.llg_rhs_vec(m_vec, out_vec)

    def ifunction_SOT(self, ts, t, y, ydot, f):
        return self.ifunction(ts, t, y, ydot, f)

    def update_jac_state_SOT(self, m_vec):
        self.update_jac_state(m_vec)

    def jac_vec_times_SOT_vec(self, v_vec, out_vec):
        self.jac_vec_times_vec(v_vec, out_vec)


class JvContextSTT(JvContext):
    """JvContextSTT (llg_stt_module_GPU.py:1210-1336): the 3x3 block preconditioner with the STT terms
    c3 = (beta - alpha) prefZhang, c4 = -(1 + alpha beta) prefZhang."""

    def __init__(self, hef: EffectiveFieldSTTGPU, eps_reg=1e-14, det_eps=1e-30):
        super().__init__(hef, eps_reg, det_eps)
        a, b = hef.alpha, hef.beta
        self.c3 = (b - a) * hef.prefZhang
        self.c4 = -(1.0 + a * b) * hef.prefZhang


class JvContextSOT(JvContext):
    """JvContextSOT (llg_SOT_module_GPU.py:1202-1290): column-wise local SOT Jacobian."""

    def update_pc_full_fast_gpu(self, shift, use_abs_diag=False):
        super().update_pc_full_fast_gpu(shift, include_stab=True, use_abs_kappa=use_abs_diag)


class LLG_GPU:
    """Builder-style driver (llg_module_GPU.py:1549-1700) with a fixed-step RK4 run."""

    def __init__(self, X, tets, Ms, gamma=2.211e5, alpha=0.5, do_precess=1, precision="f64"):
        self.X, self.tets = as_mesh(X, tets)
        self.Ms, self.gamma, self.alpha, self.do_precess = float(Ms), float(gamma), float(alpha), do_precess
        self.precision = precision
        self._kw = dict(Aex=0.0, Ku=0.0, n_ani_vec=None, D_int=0.0, n0_int_vec=None, H0_static=None,
                        Ku_nodes=None)
        self._demag = None
        self.hef = None

    def add_exchange(self, Aex):
        self._kw["Aex"] = float(Aex)

    def add_demag(self, method="lindholm", **kwargs):
        self._demag = dict(kwargs)

    def add_anisotropy(self, Ku, n_vec, Ku_nodes=None):
        self._kw.update(Ku=float(Ku), n_ani_vec=n_vec, Ku_nodes=Ku_nodes)

    def add_dmi_interfacial(self, D_int, n0_vec):
        self._kw.update(D_int=float(D_int), n0_int_vec=n0_vec)

    def add_dmi_bulk(self, D_bulk):
        self._kw["D_bulk"] = float(D_bulk)

    def add_external_field(self, H0_vec=None, H_time_func=None):
        self._kw["H0_static"] = H0_vec
        self._kw["H_time_func"] = H_time_func

    def _build(self):
        if self.hef is None:
            self.hef = EffectiveField(self.X, self.tets, self.Ms, gamma=self.gamma, alpha=self.alpha,
                                      do_precess=self.do_precess, use_demag=self._demag is not None,
                                      demag_kwargs=self._demag, precision=self.precision, **self._kw)
        return self.hef

    def _save_final(self, m, output_dir, stem, t, checkpoint):
        """The final state as <output_dir>/<stem>.xdmf (always, as the reference) and, with
        checkpoint, as the restart checkpoint <output_dir>/<stem>.bp (io.write_mesh +
        io.write_function at time 0, name "m": the reference's adios4dolfinx calls, in this
        package's own checkpoint format)."""
        from pathlib import Path
        from . import io as sio
        out = Path(output_dir)
        out.mkdir(parents=True, exist_ok=True)
        sio.XDMFWriter(out / f"{stem}.xdmf", self.X, self.tets).write_function(m, time=t, name="m")
        if checkpoint:
            sio.write_mesh(out / f"{stem}.bp", self.X, self.tets)
            sio.write_function(out / f"{stem}.bp", m, time=0.0, name="m")

    def relax_explicit(self, m0_array, t0, t_final, dt_init, rk_type="5dp", dt_save=None, dt_snap=None,
                       output_dir="output_explicit", ts_rtol=1e-6, ts_atol=1e-6, stopping_dmdt=0.0,
                       monitor_fn=None, save_final_state=False, check_every_stop=5, stop_print=False,
                       return_stats=False, max_steps=50_000_000):
        """Adaptive explicit relaxation (LLG_GPU.relax_explicit, llg_module_GPU.py:1790-1970).

        Dormand-Prince 5(4) steps on the device (spx_llg_rk_attempt) from t0 until t_final is
        reached or passed (PETSc ExactFinalTime STEPOVER), with the step adaptor of
        _ensure_solver_explicit (:1765-1772, PETSc TSAdapt "basic"): weighted RMS error norm
        with tol_i = atol + rtol max(|y5_i|, |y4_i|); accept when <= 1; next step
        dt * clip(safety * err^(-1/5), 0.1, 3.0), safety 0.9, times the reject safety 0.1 after
        a second rejection in a row; dt kept in [1e-18, 1e-10].  The dm/dt stopper
        (StopByMaxDmdtFDGPU, :314-382) ends the run when max_i |m_i - m_prev_i| / (t - t_prev)
        falls below stopping_dmdt deg/ns, tested every check_every_stop steps.  monitor_fn(step,
        t, m) is called after every accepted step when given.  The final state is written as
        <output_dir>/Relax_explicit.xdmf and, with save_final_state, as the restart checkpoint
        <output_dir>/Relax_explicit.bp (spinfemx_b200.io.read_mesh / read_function).
        Returns (m, elapsed) or (m, elapsed, stats)."""
        import time
        import torch
        if rk_type != "5dp":
            raise ValueError("rk_type must be '5dp' (Dormand-Prince 5(4))")
        hef = self._build()
        if m0_array is not None:
            m0 = m0_array if isinstance(m0_array, torch.Tensor) else torch.as_tensor(
                np.asarray(m0_array, dtype=np.float64))
            hef.set_state(m0.to(device="cuda", dtype=torch.float64).contiguous())
        hef.current_time = float(t0)
        ad = TSAdaptBasic()
        stopper = DmdtStopper(hef, stopping_dmdt, check_every_stop, stop_print)
        dt = min(max(float(dt_init), ad.dt_min), ad.dt_max)
        step, reason, reuse = 0, 0, False
        t_start = time.perf_counter()
        while step < max_steps:
            if hef.current_time >= float(t_final):
                reason = 1          # TS_CONVERGED_TIME
                break
            accept_prev = True
            while True:
                enorm = hef.rk_attempt(dt, ts_rtol, ts_atol, reuse_fsal=reuse)
                accept, dt_next = ad.choose(dt, enorm, accept_prev)
                if accept:
                    break
                reuse = True        # k1 of the state is still valid
                accept_prev = False
                dt = dt_next
            hef.rk_accept(dt)
            reuse = True
            step += 1
            if monitor_fn is not None:
                monitor_fn(step, hef.current_time, hef.get_state())
            if stopper(step, hef.current_time):
                reason = 2          # TS_CONVERGED_USER
                dt = dt_next
                break
            dt = dt_next
        elapsed = time.perf_counter() - t_start
        m = hef.get_state()
        self._save_final(m, output_dir, "Relax_explicit", hef.current_time, save_final_state)
        stats = {"t_end": float(hef.current_time), "dt_last": float(dt), "nsteps": int(step), "reason": int(reason),
                 "rejected": int(ad.rejected), "maxdmdt_deg_ns": float(stopper.last_max_dmdt_deg_ns)}
        if return_stats:
            return m, elapsed, stats
        return m, elapsed

    def relax(self, m0_array, t0, t_final, dt_init, dt_save=None, dt_snap=None, output_dir="output", ts_rtol=1e-6,
              ts_atol=1e-6, snes_rtol=1e-2, snes_atol=1e-4, ksp_rtol=1e-4, stopping_dmdt=0.0, monitor_fn=None,
              save_final_state=True, check_every_stop=5, stop_print=False, return_stats=False, use_pc_python=True,
              max_steps=50_000_000, max_reject=10):
        """Implicit relaxation (LLG_GPU.relax, llg_module_GPU.py:2183-2381, with the solver of
        _ensure_solver, :2052-2181).

        Variable-step BDF(2) attempts on the device (spx_llg_bdf_attempt: Newton with the
        quadratic backtracking line search, left-preconditioned GMRES(30) on shift I - J with
        the 3x3 block preconditioner when use_pc_python, else none) from t0 until t_final is
        reached or passed, with the TSAdapt "basic" options of _ensure_solver (:2074-2081):
        clip (0.1, 3.0), safety 0.9, reject safety 0.1, dt in [1e-17, 1e-10], exponent
        -1/order of the error estimate; a failed stage solve rejects the attempt and scales dt
        by 0.25.  More than max_reject rejections in one step end the run (reason -2, PETSc's
        TS_DIVERGED_STEP_REJECTED).  The dm/dt stopper (StopByMaxDmdtFDGPU, :314-382) ends the
        run below stopping_dmdt deg/ns, tested every check_every_stop steps.  monitor_fn(step,
        t, m) runs after every accepted step.  The final state is written as
        <output_dir>/Relax.xdmf and, with save_final_state, as the restart checkpoint
        <output_dir>/Relax.bp (spinfemx_b200.io.read_mesh / read_function).  Returns
        (m, ctx, elapsed) or (m, ctx, elapsed, stats), ctx an ImplicitContext."""
        import time
        import torch
        hef = self._build()
        if m0_array is not None:
            m0 = m0_array if isinstance(m0_array, torch.Tensor) else torch.as_tensor(
                np.asarray(m0_array, dtype=np.float64))
            hef.set_state(m0.to(device="cuda", dtype=torch.float64).contiguous())
        hef.current_time = float(t0)
        hef.bdf_reset()
        o = _lib.BdfOpts()
        call("spx_bdf_default_opts", C.byref(o))
        o.rtol, o.atol = float(ts_rtol), float(ts_atol)
        o.snes_rtol, o.snes_atol, o.ksp_rtol = float(snes_rtol), float(snes_atol), float(ksp_rtol)
        o.use_pc = 1 if use_pc_python else 0
        ad = TSAdaptBasic(dt_min=1e-17, dt_max=1e-10)
        ctx = ImplicitContext()
        stopper = DmdtStopper(hef, stopping_dmdt, check_every_stop, stop_print)
        dt = min(max(float(dt_init), ad.dt_min), ad.dt_max)
        step, reason, failures = 0, 0, 0
        t_start = time.perf_counter()
        while step < max_steps:
            if hef.current_time >= float(t_final):
                reason = 1          # TS_CONVERGED_TIME
                break
            accept_prev, nrej = True, 0
            while True:
                r = hef.bdf_attempt(dt, o)
                ctx.newton_its += r["newton_its"]
                ctx.linear_its += r["linear_its"]
                ctx.fevals += r["fevals"]
                if r["snes_reason"] < 0:
                    failures += 1
                    ad.rejected += 1
                    accept, dt_next = False, dt * 0.25
                else:
                    ad.order = r["order"]
                    accept, dt_next = ad.choose(dt, r["wlte"], accept_prev)
                if accept:
                    break
                nrej += 1
                accept_prev = False
                dt = dt_next
                if nrej > max_reject:
                    reason = -2     # TS_DIVERGED_STEP_REJECTED
                    break
            if reason == -2:
                break
            hef.bdf_accept(dt)
            step += 1
            if monitor_fn is not None:
                monitor_fn(step, hef.current_time, hef.get_state())
            if stopper(step, hef.current_time):
                reason = 2          # TS_CONVERGED_USER
                dt = dt_next
                break
            dt = dt_next
        elapsed = time.perf_counter() - t_start
        ctx.calls = ctx.callsPre = ctx.linear_its
        m = hef.get_state()
        self._save_final(m, output_dir, "Relax", hef.current_time, save_final_state)
        stats = {"t_end": float(hef.current_time), "dt_last": float(dt), "nsteps": int(step), "reason": int(reason),
                 "rejected": int(ad.rejected), "snes_failures": int(failures), "newton_its": ctx.newton_its,
                 "linear_its": ctx.linear_its, "fevals": ctx.fevals,
                 "maxdmdt_deg_ns": float(stopper.last_max_dmdt_deg_ns)}
        if return_stats:
            return m, ctx, elapsed, stats
        return m, ctx, elapsed

    def run_fixed(self, m0, dt, nsteps):
        """Integrate nsteps of RK4 at step dt from m0 (3N numpy or CUDA tensor); returns m (CUDA tensor)."""
        import torch
        hef = self._build()
        m = torch.as_tensor(np.asarray(m0, dtype=np.float64) if not isinstance(m0, torch.Tensor) else m0,
                            dtype=torch.float64, device="cuda").contiguous()
        hef.set_state(m)
        hef.step(dt, nsteps)
        return hef.get_state()


class ImplicitContext:
    """What relax() returns in place of the reference's JvContext (llg_module_GPU.py:1412-1547):
    the last shift and the counters of the run (calls = operator products in GMRES, callsPre
    = preconditioner applications, both one per GMRES iteration)."""

    def __init__(self):
        self.shift = 0.0
        self.calls = self.callsPre = 0
        self.newton_its = self.linear_its = self.fevals = 0


class TSAdaptBasic:
    """Step-size choice of PETSc's TSAdapt "basic" with the options the reference sets in
    _ensure_solver_explicit (llg_module_GPU.py:1765-1772): clip (0.1, 3.0), safety 0.9,
    reject safety 0.1, dt_min 1e-18, dt_max 1e-10; the error exponent is -1/5 (the
    Dormand-Prince pair's order).  The implicit driver (_ensure_solver, :2074-2081) uses
    dt_min 1e-17 and the order of each attempt's error estimate."""

    def __init__(self, clip=(0.1, 3.0), safety=0.9, reject_safety=0.1, dt_min=1e-18, dt_max=1e-10, order=5):
        self.clip, self.safety, self.reject_safety = clip, safety, reject_safety
        self.dt_min, self.dt_max, self.order = dt_min, dt_max, order
        self.rejected = 0

    def choose(self, h, enorm, accept_prev=True):
        """(accept, next h) for an attempt of size h with error norm enorm (< 0: no estimate,
        accepted with h kept)."""
        if enorm < 0.0:
            return True, min(max(h, self.dt_min), self.dt_max)
        safety = self.safety
        if enorm > 1.0:
            if not accept_prev:
                safety *= self.reject_safety
            accept = h < (1.0 + 1.4901161193847656e-08) * self.dt_min
        else:
            accept = True
        if not accept:
            self.rejected += 1
        hfac = safety * enorm ** (-1.0 / self.order) if enorm > 0.0 else float("inf")
        hfac = min(max(hfac, self.clip[0]), self.clip[1])
        return accept, min(max(h * hfac, self.dt_min), self.dt_max)


class DmdtStopper:
    """StopByMaxDmdtFDGPU (llg_module_GPU.py:314-382): every check_every steps, max over nodes
    of |m - m_prev| / (t - t_prev), in deg/ns; stops below the threshold (<= 0: never)."""

    def __init__(self, hef, stopping_dm_dt_deg_ns, check_every=10, print_every_hit=True):
        self.hef = hef
        self.thresh_deg_ns = float(stopping_dm_dt_deg_ns)
        self.check_every = int(check_every)
        self.print_every_hit = bool(print_every_hit)
        self.u_prev = None
        self.t_prev = None
        self.last_max_dmdt_deg_ns = float("nan")

    def __call__(self, step, t):
        if self.thresh_deg_ns <= 0.0:
            return False
        if self.check_every > 1 and step % self.check_every != 0:
            return False
        u = self.hef.get_state()
        if self.t_prev is None or t - self.t_prev <= 0.0:
            self.u_prev, self.t_prev = u, t
            return False
        out = _lib.c_dbl()
        call("spx_vec_node_diff_max", ptr(u), ptr(self.u_prev), self.hef.N, C.byref(out), _lib.stream_ptr())
        mx = out.value / (t - self.t_prev)
        self.last_max_dmdt_deg_ns = mx * (180.0 / np.pi) * 1e-9
        if self.print_every_hit:
            print(f"[dmdt] step={step} t={t * 1e9:.6f} ns  max|dm/dt|={self.last_max_dmdt_deg_ns:.6e} deg/ns",
                  flush=True)
        self.u_prev, self.t_prev = u, t
        return self.last_max_dmdt_deg_ns < self.thresh_deg_ns
