"""ctypes binding of libspx.so (the C ABI declared in include/spx.h).

The library is loaded from this package directory.  A missing library raises
ImportError: there is no CPU fallback for any operation of this package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libspx.so"

SPX_OK, SPX_ERR_INVALID, SPX_ERR_CUDA, SPX_ERR_OOM = 0, 1, 2, 3
SPX_ERR_NOT_CONVERGED, SPX_ERR_TIMEOUT, SPX_ERR_INTERNAL, SPX_ERR_NO_DEVICE = 4, 5, 6, 7
PREC = {"f64": 0, "fp64": 0, "float64": 0, "f32": 1, "fp32": 1, "float32": 1, "mixed": 2, "bf16": 2, "f32_f16": 3}

c_i32, c_i64, c_dbl, c_vp = C.c_int32, C.c_int64, C.c_double, C.c_void_p
P_i32, P_i64, P_dbl = C.POINTER(c_i32), C.POINTER(c_i64), C.POINTER(c_dbl)


class HmatConfig(C.Structure):
    _fields_ = [("epsilon", c_dbl), ("eta", c_dbl), ("leaf_size", c_i32), ("max_rank", c_i32),
                ("max_temporary_block_bytes", c_i64), ("precision", c_i32), ("flags", c_i32),
                ("batch_bytes", c_i64)]


class DemagOptions(C.Structure):
    _fields_ = [("backend", c_i32), ("precision", c_i32), ("rtol_u1", c_dbl), ("rtol_u2", c_dbl),
                ("atol", c_dbl), ("maxit_u1", c_i32), ("maxit_u2", c_i32), ("warm_start", c_i32),
                ("u1_preconditioner", c_i32), ("hmat", HmatConfig)]


class LLGParams(C.Structure):
    _fields_ = [("Ms", c_dbl), ("gamma", c_dbl), ("alpha", c_dbl), ("do_precess", c_dbl), ("Aex", c_dbl),
                ("Ku", c_dbl), ("Ku_nodes", c_vp), ("n_ani", c_vp), ("D_int", c_dbl), ("n_int", c_vp),
                ("H0_nodes", c_vp), ("H0_uniform", c_dbl * 3), ("use_demag", c_i32), ("precision", c_i32),
                ("stt_J", c_dbl), ("stt_P", c_dbl), ("stt_beta", c_dbl), ("stt_dir", c_vp),
                ("sot_Hdl", c_dbl), ("sot_Hfl", c_dbl), ("sot_p", c_vp), ("D_bulk", c_dbl)]


class BdfOpts(C.Structure):
    _fields_ = [("rtol", c_dbl), ("atol", c_dbl), ("snes_rtol", c_dbl), ("snes_atol", c_dbl),
                ("snes_stol", c_dbl), ("snes_divtol", c_dbl), ("ksp_rtol", c_dbl), ("ksp_atol", c_dbl),
                ("ksp_dtol", c_dbl), ("ls_alpha", c_dbl), ("ls_minlambda", c_dbl), ("ls_maxstep", c_dbl),
                ("snes_max_it", c_i32), ("ksp_max_it", c_i32), ("ksp_restart", c_i32), ("ls_max_it", c_i32),
                ("use_pc", c_i32), ("reserved", c_i32)]


class BdfResult(C.Structure):
    _fields_ = [("wlte", c_dbl), ("snes_reason", c_i32), ("order", c_i32), ("restarted", c_i32),
                ("newton_its", c_i32), ("linear_its", c_i32), ("fevals", c_i32)]


# name -> (restype, argtypes)
SIGNATURES = {
    "spx_last_error": (C.c_char_p, []),
    "spx_version": (C.c_int, []),
    "spx_device_count": (C.c_int, [P_i32]),
    "spx_boundary_sizes": (C.c_int, [c_vp, c_i64, c_vp, c_i64, P_i64, P_i64]),
    "spx_boundary_data": (C.c_int, [c_vp, c_i64, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "spx_fem_sizes": (C.c_int, [c_vp, c_i64, c_vp, c_i64, P_i64]),
    "spx_fem_assemble": (C.c_int, [c_vp, c_i64, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "spx_cluster_tree": (C.c_int, [c_vp, c_i64, c_i32, c_vp]),
    "spx_boundary_create": (C.c_int, [c_vp, c_i64, c_vp, c_i64, C.POINTER(c_vp)]),
    "spx_boundary_destroy": (C.c_int, [c_vp]),
    "spx_boundary_info": (C.c_int, [c_vp, P_i64, P_i64, P_i32]),
    "spx_lindholm_pairs": (C.c_int, [c_vp, c_vp, c_vp, c_i64, c_vp, c_vp]),
    "spx_lindholm_fill_block": (C.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, c_vp, c_vp]),
    "spx_dense_b_assemble": (C.c_int, [c_vp, c_vp, c_vp]),
    "spx_dense_b_apply": (C.c_int, [c_vp, c_i64, c_vp, c_vp, c_vp]),
    "spx_hmat_build": (C.c_int, [c_vp, C.POINTER(HmatConfig), C.POINTER(c_vp)]),
    "spx_hmat_stats": (C.c_int, [c_vp, c_vp, P_dbl]),
    "spx_hmat_num_blocks": (C.c_int, [c_vp, P_i64]),
    "spx_hmat_blocks": (C.c_int, [c_vp, c_vp, c_i64]),
    "spx_hmat_perm": (C.c_int, [c_vp, c_vp]),
    "spx_hmat_apply": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_hmat_repack": (C.c_int, [c_vp, c_i32]),
    "spx_hmat_recompress": (C.c_int, [c_vp, c_vp, P_dbl]),
    "spx_hmat_tensor_cores": (C.c_int, [c_vp, c_i32, P_i64]),
    "spx_hmat_tc_status": (C.c_int, [c_vp, P_i32]),
    "spx_hmat_apply_noalloc": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_hmat_apply_transpose": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_hmat_apply_multi": (C.c_int, [c_vp, c_vp, c_vp, c_i32, c_vp]),
    "spx_hmat_far_factors": (C.c_int, [c_vp, c_i64, c_vp, c_vp]),
    "spx_hmat_memory": (C.c_int, [c_vp, P_i64, P_i64, P_i64]),
    "spx_hmat_destroy": (C.c_int, [c_vp]),
    "spx_demag_create": (C.c_int, [c_vp, c_i64, c_vp, c_i64, c_dbl, C.POINTER(DemagOptions), C.POINTER(c_vp)]),
    "spx_demag_apply": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_demag_ensemble_info": (C.c_int, [c_vp, c_vp]),
    "spx_demag_ensemble_hmat": (C.c_int, [c_vp, c_i32, C.POINTER(c_vp)]),
    "spx_debug_barrier_probe": (C.c_int, [c_i32, c_i64, C.POINTER(c_i32), C.POINTER(c_i32)]),
    "spx_debug_fail_alloc": (C.c_int, [c_i64, c_i32]),
    "spx_debug_noalloc_cap": (C.c_int, [c_i64]),
    "spx_debug_barrier_time": (C.c_int, [c_i32, c_i32, c_i32, P_dbl]),
    "spx_debug_pcg_phase_times": (C.c_int, [c_vp, c_vp]),
    "spx_debug_pcg_timing": (C.c_int, [c_i32]),
    "spx_device_l2_persisting": (C.c_int, [P_i64, P_i64]),
    "spx_llg_set_time_field": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_step_time_field": (C.c_int, [c_vp, c_dbl, c_vp, c_vp, c_vp]),
    "spx_llg_rk_attempt": (C.c_int, [c_vp, c_i32, c_dbl, c_dbl, c_dbl, c_vp, c_vp, c_i32, P_dbl, c_vp]),
    "spx_llg_rk_accept": (C.c_int, [c_vp, c_vp]),
    "spx_bdf_default_opts": (C.c_int, [C.POINTER(BdfOpts)]),
    "spx_llg_bdf_attempt": (C.c_int, [c_vp, c_dbl, c_dbl, C.POINTER(BdfOpts), c_vp, c_vp, C.POINTER(BdfResult),
                                      c_vp]),
    "spx_llg_bdf_accept": (C.c_int, [c_vp, c_vp]),
    "spx_llg_bdf_reset": (C.c_int, [c_vp]),
    "spx_vec_node_diff_max": (C.c_int, [c_vp, c_vp, c_i64, P_dbl, c_vp]),
    "spx_demag_create_ensemble": (C.c_int, [c_vp, c_i64, c_vp, c_i64, c_dbl, C.POINTER(DemagOptions), c_i64, c_vp,
                                            c_i64, C.POINTER(c_vp)]),
    "spx_demag_apply_transpose": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_demag_potentials": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_demag_energy": (C.c_int, [c_vp, c_vp, c_vp, P_dbl, c_vp]),
    "spx_demag_stats": (C.c_int, [c_vp, P_i64, P_i64, P_dbl, P_dbl]),
    "spx_demag_info": (C.c_int, [c_vp, P_i64, P_i64, P_i64, P_i64]),
    "spx_demag_hmat": (C.c_int, [c_vp, C.POINTER(c_vp)]),
    "spx_demag_destroy": (C.c_int, [c_vp]),
    "spx_demag_profile_begin": (C.c_int, [c_vp]),
    "spx_demag_profile_end": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_demag_counters": (C.c_int, [c_vp, c_vp, c_vp]),
    "spx_demag_residuals": (C.c_int, [c_vp, c_vp, c_vp]),
    "spx_demag_amg_levels": (C.c_int, [c_vp, c_vp, C.c_int32, c_vp]),
    "spx_demag_create_with_hmat": (C.c_int, [c_vp, c_i64, c_vp, c_i64, c_dbl, C.POINTER(DemagOptions), c_vp,
                                             C.POINTER(c_vp)]),
    "spx_hmat_export_sizes": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "spx_hmat_export": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "spx_hmat_import": (C.c_int, [c_vp, C.POINTER(HmatConfig), c_vp, c_vp, c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp,
                                  c_vp, C.POINTER(c_vp)]),
    "spx_demag_set_tolerances": (C.c_int, [c_vp, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_int32]),
    "spx_llg_create": (C.c_int, [c_vp, c_vp, c_i64, c_vp, c_i64, C.POINTER(LLGParams), C.POINTER(c_vp)]),
    "spx_llg_heff": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_hjac": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_rhs": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_update_jac_state": (C.c_int, [c_vp, c_vp, c_vp]),
    "spx_llg_jv": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_pc_build": (C.c_int, [c_vp, c_dbl, c_i32, c_i32, c_vp]),
    "spx_llg_pc_apply": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_set_state": (C.c_int, [c_vp, c_vp, c_vp]),
    "spx_llg_get_state": (C.c_int, [c_vp, c_vp, c_vp]),
    "spx_llg_step": (C.c_int, [c_vp, c_dbl, c_i64, c_vp]),
    "spx_llg_zhang_li": (C.c_int, [c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_set_sot": (C.c_int, [c_vp, c_dbl, c_dbl, c_vp]),
    "spx_llg_min_eval": (C.c_int, [c_vp, c_vp, c_vp, c_i32, c_vp, c_vp]),
    "spx_llg_min_trial": (C.c_int, [c_vp, c_vp, c_vp, c_dbl, c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_set_graph": (C.c_int, [c_vp, c_i32]),
    "spx_llg_graph_stats": (C.c_int, [c_vp, P_i64, P_i32]),
    "spx_llg_set_anisotropy_map": (C.c_int, [c_vp, c_vp]),
    "spx_llg_rhs_vjp": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_step_vjp": (C.c_int, [c_vp, c_vp, c_dbl, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "spx_llg_step_jvp": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_dbl, c_vp, c_vp, c_vp]),
    "spx_llg_run_host": (C.c_int, [c_vp, c_vp, c_vp, c_dbl, c_i64]),
    "spx_llg_set_uniform_field": (C.c_int, [c_vp, c_dbl, c_dbl, c_dbl]),
    "spx_llg_stats": (C.c_int, [c_vp, P_i64, P_i64, P_i64]),
    "spx_llg_destroy": (C.c_int, [c_vp]),
}

_lib = None


def lib():
    """Load libspx.so once; raise ImportError if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with fenicsx-micromagnetics_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class SpxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[spx status {code}] {msg}")
        self.code = code


class SpxTimeout(SpxError):
    pass


def check(code: int):
    if code == SPX_OK:
        return
    msg = lib().spx_last_error().decode(errors="replace")
    if code == SPX_ERR_INVALID:
        raise ValueError(msg)
    if code == SPX_ERR_OOM:
        raise MemoryError(msg)
    if code == SPX_ERR_TIMEOUT:
        raise SpxTimeout(code, msg)
    raise SpxError(code, msg)


def call(name, *args):
    check(getattr(lib(), name)(*args))


def ptr(t):
    """Raw address of a torch tensor or numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return t.ctypes.data_as(C.c_void_p)


def stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return C.c_void_p(s.cuda_stream)


def device_count() -> int:
    n = c_i32(0)
    lib().spx_device_count(C.byref(n))
    return int(n.value)
