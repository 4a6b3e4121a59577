"""FEM/BEM demagnetising field (drop-in for DemagFieldLindholmGPU).

Mirrors ``gpu/fields/Demag_Lindholm_GPU.py``: same constructor option names
(``boundary_backend``, ``ksp_rtol_u1/u2``, ``hmatrix_*``, ``dense_gpu_max_bytes``),
``compute_vec(m_vec, out_vec)`` (:643-670), ``Energy_lumped_gpu`` (:706-724),
``boundary_memory_report`` (:672-704) and the ``last_its_u1/u2`` attributes.
Vectors are CUDA float64 torch tensors of length 3N in AoS order (the layout of
the reference's PETSc CUDA Vec with block size 3) instead of PETSc Vecs.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import call, ptr
from .geometry import as_mesh
from .hmatrix import HMatrixGPUPackedFused


class DemagFieldLindholmGPU:
    def __init__(self, X, tets, Ms, *, ksp_rtol_u1=1e-6, ksp_rtol_u2=1e-6, ksp_atol=1e-12, ksp_maxit_u1=2000,
                 ksp_maxit_u2=12000, incident_policy="skip", volume_scale=1e27, boundary_backend="dense",
                 dense_gpu_max_bytes=512 * 1024 ** 2, hmatrix_epsilon=1e-5, hmatrix_eta=2.0, hmatrix_leaf_size=64,
                 hmatrix_compressor="fullaca", hmatrix_max_rank=None,
                 hmatrix_max_temporary_block_bytes=256 * 1024 ** 2, hmatrix_use_fp32=True, precision="f64",
                 hmatrix_precision=None, warm_start=False, hmatrix_batch_bytes=0, hmatrix_verbose=False,
                 u1_preconditioner="amg", hmatrix_cache_path=None, hmatrix_cache_dir="./hmatrix_cache",
                 cache_tag=None, hmatrix_force_rebuild=False, hmatrix_cache_compressed=False, sample_offsets=None,
                 dense_max_nb=4096, hmatrix_recompress=False, **unused):
        """Options as in the reference, plus:

        precision          'f64' | 'f32' (plain FP32) | 'mixed' (FP64 vectors, FP32 matrices,
                           FP32 CG inside FP64 iterative refinement)
        hmatrix_precision  factor storage 'f64' | 'f32' | 'bf16' (default: 'f64' for
                           precision='f64', 'f32' otherwise)
        warm_start         False: zero start (the reference); True: previous solution;
                           'extrapolate': per-RK-stage quartic extrapolation (time loop);
                           'extrapolate_corrected': the same, stages 2-4 shifted by stage 1's
                           prediction error
        u1_preconditioner  'amg' (smoothed aggregation, as the reference's PC "gamg") or
                           'jacobi'
        hmatrix_recompress SVD-recompress the ACA factors after the build (same tolerance;
                           needed by hmatrix_precision 'f32_f16')
        boundary_backend   also 'ensemble': X / tets is a disjoint union of independent samples
                           (``sample_offsets``: node ranges, see spinfemx_b200.ensemble); each
                           sample gets its own boundary operator, dense when its Nb <=
                           ``dense_max_nb``, an H-matrix otherwise
        hmatrix_cache_path / cache_tag
                           npz cache of the H-matrix in the reference's schema
                           (Demag_Lindholm_GPU.py:353-377 naming in hmatrix_cache_dir or
                           $DEMAG_HMATRIX_CACHE_DIR when only cache_tag is given).  Without either,
                           the H-matrix is built on the GPU and no file is written.
        """
        if str(incident_policy).lower()[:4] != "skip":
            raise ValueError("only incident_policy='skip' (the reference default) is implemented")
        if str(hmatrix_compressor).strip().lower() not in {"fullaca", "aca"}:
            raise ValueError("the GPU builder implements the 'fullaca' compressor")
        X, tets = as_mesh(X, tets)
        self.X, self.tets = X, tets
        self.N = X.shape[0]
        self.local_size = 3 * self.N
        self.Ms = float(Ms)
        self.mu0 = 4.0 * np.pi * 1e-7
        self.volume_scale = float(volume_scale)
        self.precision = precision
        req = str(boundary_backend).strip().lower()
        if req not in {"dense", "hmatrix", "auto", "ensemble"}:
            raise ValueError("boundary_backend must be 'dense', 'hmatrix', 'auto' or 'ensemble'.")
        if (req == "ensemble") != (sample_offsets is not None):
            raise ValueError("boundary_backend='ensemble' and sample_offsets go together")
        if req == "auto":
            Nb = _lib.c_i64()
            call("spx_boundary_sizes", ptr(X), self.N, ptr(tets), tets.shape[0], C.byref(Nb), None)
            req = "dense" if Nb.value * Nb.value * 8 <= int(dense_gpu_max_bytes) else "hmatrix"
        self.boundary_backend = req
        if precision not in ("f64", "f32", "mixed"):
            raise ValueError("precision must be 'f64', 'f32' or 'mixed'")
        hprec = hmatrix_precision or ("f64" if precision == "f64" else "f32")
        if hprec not in ("f64", "f32", "bf16", "f32_f16"):
            raise ValueError("hmatrix_precision must be 'f64', 'f32', 'bf16' or 'f32_f16'")
        if hprec == "f32_f16":
            hmatrix_recompress = True
        self.hmatrix_precision = hprec
        ws = {False: 0, True: 1, 0: 0, 1: 1, 2: 2, 3: 3, "extrapolate": 2, "extrapolate_corrected": 3}.get(warm_start)
        if ws is None:
            raise ValueError("warm_start must be False, True, 'extrapolate' or 'extrapolate_corrected'")
        o = _lib.DemagOptions()
        o.backend = 0 if req == "dense" else 1
        o.precision = _lib.PREC[precision]
        o.rtol_u1, o.rtol_u2, o.atol = float(ksp_rtol_u1), float(ksp_rtol_u2), float(ksp_atol)
        o.maxit_u1, o.maxit_u2 = int(ksp_maxit_u1), int(ksp_maxit_u2)
        self.ksp_rtol_u1, self.ksp_rtol_u2, self.ksp_atol = o.rtol_u1, o.rtol_u2, o.atol
        self.ksp_maxit_u1, self.ksp_maxit_u2 = o.maxit_u1, o.maxit_u2
        o.warm_start = ws
        pcs = {"amg": 0, "gamg": 0, "jacobi": 1}
        if str(u1_preconditioner).lower() not in pcs:
            raise ValueError("u1_preconditioner must be 'amg' or 'jacobi'")
        o.u1_preconditioner = pcs[str(u1_preconditioner).lower()]
        self.u1_preconditioner = str(u1_preconditioner).lower()
        o.hmat = _lib.HmatConfig(epsilon=float(hmatrix_epsilon), eta=float(hmatrix_eta),
                                 leaf_size=int(hmatrix_leaf_size), max_rank=int(hmatrix_max_rank or 0),
                                 max_temporary_block_bytes=int(hmatrix_max_temporary_block_bytes),
                                 precision=_lib.PREC[hprec], flags=1 if hmatrix_recompress else 0,
                                 batch_bytes=int(hmatrix_batch_bytes))
        self._h = C.c_void_p()
        self.hmatrix_cache_path = None
        if req == "hmatrix" and (hmatrix_cache_path is not None or cache_tag is not None):
            import os
            from pathlib import Path
            from .hmatrix import HMatrixBuildConfig, build_or_load_hmatrix
            if hmatrix_cache_path is None:
                root = Path(os.environ.get("DEMAG_HMATRIX_CACHE_DIR", hmatrix_cache_dir))
                eps_tag = f"{float(hmatrix_epsilon):.0e}".replace("+", "")
                eta_tag = f"{float(hmatrix_eta):g}".replace(".", "p")
                comp = str(hmatrix_compressor).strip().lower().replace("-", "_")
                hmatrix_cache_path = root / (f"{cache_tag}_eps{eps_tag}_eta{eta_tag}_leaf{int(hmatrix_leaf_size)}_"
                                             f"{comp}_gpu.npz")
            self.hmatrix_cache_path = str(hmatrix_cache_path)
            cfg = HMatrixBuildConfig(epsilon=float(hmatrix_epsilon), eta=float(hmatrix_eta),
                                     leaf_size=int(hmatrix_leaf_size), max_rank=hmatrix_max_rank,
                                     max_temporary_block_bytes=int(hmatrix_max_temporary_block_bytes),
                                     batch_bytes=int(hmatrix_batch_bytes), recompress=bool(hmatrix_recompress))
            Hc = build_or_load_hmatrix(self.hmatrix_cache_path, X, tets, cfg, precision=hprec,
                                       force_rebuild=bool(hmatrix_force_rebuild), verbose=bool(hmatrix_verbose),
                                       cache_compressed=bool(hmatrix_cache_compressed))
            self.hmatrix_metadata = Hc.metadata
            call("spx_demag_create_with_hmat", ptr(X), self.N, ptr(tets), tets.shape[0], self.Ms, C.byref(o),
                 Hc.handle, C.byref(self._h))
            del Hc  # its data moved into the demag object
        elif req == "ensemble":
            offs = np.ascontiguousarray(np.asarray(sample_offsets, dtype=np.int64).reshape(-1))
            self.sample_offsets = offs
            call("spx_demag_create_ensemble", ptr(X), self.N, ptr(tets), tets.shape[0], self.Ms, C.byref(o),
                 offs.size - 1, ptr(offs), int(dense_max_nb), C.byref(self._h))
        else:
            call("spx_demag_create", ptr(X), self.N, ptr(tets), tets.shape[0], self.Ms, C.byref(o),
                 C.byref(self._h))
        N, Nb, NI, by = _lib.c_i64(), _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
        call("spx_demag_info", self._h, C.byref(N), C.byref(Nb), C.byref(NI), C.byref(by))
        self.Nb, self.NI = Nb.value, NI.value
        self.last_its_u1 = 0
        self.last_its_u2 = 0
        self.B_dense_gpu = None
        self.B_hmatrix_gpu = None
        if req == "ensemble":
            hh = C.c_void_p()
            if _lib.lib().spx_demag_ensemble_hmat(self._h, 0, C.byref(hh)) == 0:  # samples sharing a mesh
                st = np.zeros(16, np.int64)
                call("spx_hmat_stats", hh, ptr(st), None)
                self.B_hmatrix_gpu = HMatrixGPUPackedFused.from_handle(hh, self, {"bf16": "mixed"}.get(hprec, hprec),
                                                                       int(st[14]))
        if req == "hmatrix":
            hh = C.c_void_p()
            call("spx_demag_hmat", self._h, C.byref(hh))
            self.B_hmatrix_gpu = HMatrixGPUPackedFused.from_handle(hh, self, {"bf16": "mixed"}.get(hprec, hprec),
                                                                   self.Nb)
            if hmatrix_verbose:
                st = self.B_hmatrix_gpu.stats()
                print(f"[Demag Lindholm HMatrix b200] built in {st['build_time_seconds']:.2f} s | "
                      f"far={st['n_far']:,} | rank avg/max={st['average_far_rank']:.1f}/"
                      f"{st['max_observed_rank']}", flush=True)

    @property
    def handle(self):
        return self._h

    def _check(self, v, name):
        import torch
        if not (isinstance(v, torch.Tensor) and v.is_cuda and v.dtype == torch.float64):
            raise TypeError(f"{name} must be a CUDA float64 tensor")
        if v.numel() < self.local_size or not v.is_contiguous():
            raise RuntimeError(f"{name} must be contiguous with at least {self.local_size} entries")

    def compute_vec(self, m_vec, out_vec):
        """H_demag(m) into out_vec (AoS, length 3N; entries past 3N are zeroed)."""
        self._check(m_vec, "m_vec")
        self._check(out_vec, "out_vec")
        call("spx_demag_apply", self._h, ptr(m_vec), ptr(out_vec), _lib.stream_ptr())
        if out_vec.numel() > self.local_size:
            out_vec[self.local_size:] = 0.0
        i1, i2, r1, r2 = _lib.c_i64(), _lib.c_i64(), _lib.c_dbl(), _lib.c_dbl()
        call("spx_demag_stats", self._h, C.byref(i1), C.byref(i2), C.byref(r1), C.byref(r2))
        self.last_its_u1, self.last_its_u2 = i1.value, i2.value
        self.last_res_u1, self.last_res_u2 = r1.value, r2.value
        return out_vec

    def compute_vec_transpose(self, w_vec, out_vec):
        """out = D^T w for the linear map D: m -> H_demag (adjoint of compute_vec)."""
        self._check(w_vec, "w_vec")
        self._check(out_vec, "out_vec")
        call("spx_demag_apply_transpose", self._h, ptr(w_vec), ptr(out_vec), _lib.stream_ptr())
        if out_vec.numel() > self.local_size:
            out_vec[self.local_size:] = 0.0
        return out_vec

    def potentials(self):
        import torch
        u1 = torch.empty(self.N, dtype=torch.float64, device="cuda")
        u2 = torch.empty_like(u1)
        call("spx_demag_potentials", self._h, ptr(u1), ptr(u2), _lib.stream_ptr())
        return u1, u2

    def Energy_lumped_gpu(self, m_vec, h_vec):
        self._check(m_vec, "m_vec")
        self._check(h_vec, "h_vec")
        E = _lib.c_dbl()
        call("spx_demag_energy", self._h, ptr(m_vec), ptr(h_vec), C.byref(E), _lib.stream_ptr())
        return float(E.value) * (1e27 / self.volume_scale)

    def set_tolerances(self, *, ksp_rtol_u1=None, ksp_rtol_u2=None, ksp_atol=None, ksp_maxit_u1=None,
                       ksp_maxit_u2=None):
        """Change the Krylov tolerances after construction (KSP.setTolerances in the reference)."""
        self.ksp_rtol_u1 = self.ksp_rtol_u1 if ksp_rtol_u1 is None else float(ksp_rtol_u1)
        self.ksp_rtol_u2 = self.ksp_rtol_u2 if ksp_rtol_u2 is None else float(ksp_rtol_u2)
        self.ksp_atol = self.ksp_atol if ksp_atol is None else float(ksp_atol)
        self.ksp_maxit_u1 = self.ksp_maxit_u1 if ksp_maxit_u1 is None else int(ksp_maxit_u1)
        self.ksp_maxit_u2 = self.ksp_maxit_u2 if ksp_maxit_u2 is None else int(ksp_maxit_u2)
        call("spx_demag_set_tolerances", self._h, self.ksp_rtol_u1, self.ksp_rtol_u2, self.ksp_atol,
             self.ksp_maxit_u1, self.ksp_maxit_u2)

    def solver_counters(self):
        """Totals since construction: inner iterations, refinement steps, solves, and the sums of
        the relative residuals at the starting guess and at return, for the u1 and u2 solves."""
        c1, c2 = (_lib.c_i64 * 4)(), (_lib.c_i64 * 4)()
        r1, r2 = (_lib.c_dbl * 2)(), (_lib.c_dbl * 2)()
        call("spx_demag_counters", self._h, c1, c2)
        call("spx_demag_residuals", self._h, r1, r2)
        out = {}
        for name, c, r in (("u1", c1, r1), ("u2", c2, r2)):
            out[name] = {"iterations": c[0], "refinements": c[1], "solves": c[2],
                         "initial_rel_residual_sum": r[0], "final_rel_residual_sum": r[1]}
        return out

    def amg_levels(self):
        """Rows and nonzeros (A, P, R) per level of the u1 AMG hierarchy ([] without AMG)."""
        out = np.zeros(4 * 16, np.int64)
        nl = _lib.c_i32()
        call("spx_demag_amg_levels", self._h, ptr(out), 16, C.byref(nl))
        return [dict(rows=int(out[4 * l]), nnz_A=int(out[4 * l + 1]), nnz_P=int(out[4 * l + 2]),
                     nnz_R=int(out[4 * l + 3])) for l in range(nl.value)]

    def boundary_memory_report(self):
        N, Nb, NI, by = _lib.c_i64(), _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
        call("spx_demag_info", self._h, C.byref(N), C.byref(Nb), C.byref(NI), C.byref(by))
        if self.boundary_backend == "dense":
            b = Nb.value * Nb.value * 8
            return {"backend": "dense", "Nb": Nb.value, "accounted_gpu_bytes": b,
                    "accounted_gpu_mib": b / 2 ** 20, "total_device_bytes": by.value}
        rep = self.B_hmatrix_gpu.memory_report()
        rep["Nb"] = Nb.value
        rep["total_device_bytes"] = by.value
        return rep

    def print_boundary_memory_report(self):
        for k, v in self.boundary_memory_report().items():
            print(f"[Demag Lindholm b200] {k}: {v}", flush=True)

    def __del__(self):
        try:
            h = getattr(self, "_h", None)
            if h is not None and h.value:
                try:
                    _lib.lib().spx_demag_destroy(h)
                except Exception:
                    pass
                self._h = C.c_void_p()

        except Exception:
            pass