#!/usr/bin/env python
"""LLG steps/s on the 0.48M-node film with the FEM/BEM (H-matrix) demag field.

Workload (one "step" = one fixed-dt RK4 step = 4 effective-field/RHS evaluations):
  film 1000 x 1000 x 5 nm, 400 x 400 x 2 cubes of 2.5 nm, 6 tets per cube
  (1.92M tets, 482,403 nodes, 323,202 boundary nodes); Ms 8e5 A/m, A 1.3e-11 J/m,
  alpha 0.02, uniform 25 mT at 170 deg in plane; m0 = x + N(0, 0.05^2) renormalised
  (seeded); dt 50 fs.  Demag: u1 / u2 Poisson solves and the Lindholm double layer as
  an H-matrix (ACA 1e-5, leaf 64, eta 2) built on the GPU in FP64.  The Krylov
  tolerance (default rtol 1e-8) is the one at which the demag field of the run stays
  within 1e-5 of a tightly converged FP64 evaluation; the line reports that error.
  Synthetic mesh and magnetisation (no dataset is involved).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

At N = 1 the line also carries "batched": the same mesh as 8 films (seeded m0 each)
integrated together in the mixed + batched form (one H-matrix applied to all films with the
far field on the tensor cores, the u1 hierarchy shared), its film-steps/s, its ratio to the
single film of the same run, and film 0's demag error against FP64 (--batched 0 turns it off).

Multi-GPU: the film does not shard (one boundary operator couples every boundary
node), so N GPUs run N independent replicas ("replicas only"); value = N x steps/s.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
for _p in (str(ROOT), str(ROOT / "fenicsx-micromagnetics_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "LLG steps/s at 0.48M nodes, demag err<=1e-5 (film 400x400x2 @2.5nm, H-matrix ACA 1e-5, RK4 dt 50 fs)"
MU0 = 4e-7 * math.pi


# DRAM bytes (read + write) per launch over algorithmic bytes, from one ncu capture of the
# boundary apply (k_hgather + k_far_z + k_rows) on the 150 x 150 x 2 film:
# profiles/boundary_apply_traffic_film150x150.md (635.9 MB measured / 610.4 MB algorithmic).
TRAFFIC_PER_ALGORITHMIC_BYTE = {"boundary_apply": 635.9 / 610.4}


def l2_persisting():
    """(set-aside bytes, device maximum) of the L2 persisting carve-out of this context."""
    import ctypes as C_
    from spinfemx_b200 import _lib
    cur, mx = C_.c_int64(), C_.c_int64()
    _lib.call("spx_device_l2_persisting", C_.byref(cur), C_.byref(mx))
    return {"set_aside_bytes": cur.value, "max_bytes": mx.value}


def workload(nx, ny, nz, h, seed):
    from spinfemx_b200.geometry import kuhn_box
    X, T = kuhn_box(nx, ny, nz, h)
    N = X.shape[0]
    rng = np.random.default_rng(seed)
    m = np.tile([1.0, 0.0, 0.0], (N, 1)) + rng.normal(0.0, 0.05, (N, 3))
    m /= np.linalg.norm(m, axis=1)[:, None]
    th = math.radians(170.0)
    H0 = (0.025 / MU0) * np.array([math.cos(th), math.sin(th), 0.0])
    return X, T, m.ravel(), H0


def c2_row_vectors(Xb):
    """The three boundary vectors of the reference-rows fixture (tests/golden/c2_rows.npz):
    seeded standard normal; cos(2 pi x / 1000) cos(2 pi y / 1000); z - mean(z) + 0.1 x
    seeded noise (boundary order, Nb x 3)."""
    Nb = Xb.shape[0]
    rng = np.random.default_rng(3101)
    x = np.empty((Nb, 3))
    x[:, 0] = rng.standard_normal(Nb)
    x[:, 1] = np.cos(2 * math.pi * Xb[:, 0] / 1000.0) * np.cos(2 * math.pi * Xb[:, 1] / 1000.0)
    x[:, 2] = (Xb[:, 2] - Xb[:, 2].mean()) + 0.1 * rng.standard_normal(Nb)
    return x


def rows_err_vs_reference(spx, X, T, H):
    """Relative L2 error of H x against the reference's dense rows B[rows] x over the
    fixture's 4,096 rows (max over its three vectors); None when the mesh is not the
    fixture's."""
    import torch
    f = ROOT / "tests" / "golden" / "c2_rows.npz"
    if not f.exists():
        return None
    g = np.load(f)
    bd = spx.boundary_data(X, T)
    if bd["Xb"].shape[0] != int(g["nb"]):
        return None
    x = c2_row_vectors(bd["Xb"])
    if not np.allclose(x.sum(0), g["x_sum"], rtol=1e-12, atol=1e-9):
        return None
    rows = g["rows"]
    errs = []
    for k in range(3):
        y = H.matvec(torch.as_tensor(x[:, k].copy(), device="cuda")).cpu().numpy()[rows]
        errs.append(float(np.linalg.norm(y - g["y"][:, k]) / np.linalg.norm(g["y"][:, k])))
    return max(errs)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(n_gpus, timeout_s=300):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE); NCCL on GPUs, gloo on a
    host without one (the CPU tests of the multi-rank logic)."""
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=timeout_s),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, ws, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(x, ws):
    """Max over ranks (device times are reported as the slowest rank's)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, ms_max, ws):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return ws * units_per_rank / (ms_max * 1e-3)


def amg_iter_bytes(levels, n0, nnz0):
    """Algorithmic bytes of one AMG-preconditioned PCG iteration (k_pcg_amg): every V-cycle
    phase reads its matrix once (FP32 value + int32 column per nonzero) and its FP32 level
    vectors; the coarsest level is a dense FP32 GEMV; the PCG phases read the FP32 unscaled
    matrix and FP64 vectors (u gather, p, q, r, y, diagonal scalings)."""
    total = 0.0
    for l in range(len(levels) - 1):
        n, a, p, r = levels[l]["rows"], levels[l]["nnz_A"], levels[l]["nnz_P"], levels[l]["nnz_R"]
        nc = levels[l + 1]["rows"]
        total += (8 * a + 20 * n) + (8 * a + 16 * n) + (8 * r + 4 * n + 20 * nc)  # pre-smooth, residual, restrict
        total += (8 * p + 4 * nc + 8 * n) + (8 * a + 24 * n) + (8 * a + 20 * n)  # prolong, post-smooth x2
    ncs = levels[-1]["rows"]
    total += 4 * ncs * ncs + 8 * ncs
    total += 24 * n0  # top level: u (FP64) write, r (FP64) read, D^-1/2 read
    total += 8 * nnz0 + 60 * n0  # A z in difference form + p, q updates
    total += 68 * n0  # y, r updates, level-0 right-hand side
    return total


def bytes_model(st, nnz, N, Nb, NI, nnzI, counters, H, amg_levels=None):
    """Algorithmic bytes per launch for each kernel group (FP32 working precision)."""
    wv, wm = 4, 4
    # Jacobi refinement solves: per inner iteration one SELL SpMV + 7 vector passes
    # (nnz (w_m + 4) + 4 (N+1) + 7 N w_v); per refinement step an FP64 residual SpMV.
    def cg_bytes(c, n, z):
        if c[2] == 0:
            return 0.0
        inner = c[0] * (z * (wm + 4) + 4 * (n + 1) + 7 * n * wv)
        outer = c[1] * (z * (8 + 4) + 4 * (n + 1) + 3 * n * 8)
        return (inner + outer) / c[2]

    def amg_bytes(c, n, z):
        if c[2] == 0:
            return 0.0
        outer = c[1] * (z * (8 + 4) + 4 * (n + 1) + 3 * n * 8 + 8 * n)
        return (c[0] * amg_iter_bytes(amg_levels, n, z) + outer) / c[2]
    return {
        "u1_solve": amg_bytes(counters[0], N, nnz) if amg_levels else cg_bytes(counters[0], N, nnz),
        "u2_solve": cg_bytes(counters[1], NI, nnzI),
        # far factors + near tiles + x gather (Nb w_v) + scatter of phi and g (2 Nb w_v)
        "boundary_apply": H["far_bytes"] + H["near_bytes"] + 4 * Nb * wv,
        # Div: nnz (3 w_m + 4) + 3N w_v + N w_v
        "div": nnz * (3 * wm + 4) + 4 * N * wv,
        # fused stage: nnz (w_m exchange + 3 w_m G + 4 index) + m gather (3N) + phi (N)
        #             + acc/mn/out (3 x 3N read/write)
        "stage": nnz * (4 * wm + 4) + 4 * N * wv + 12 * N * wv,
    }


def run_ours(a):
    import torch
    import spinfemx_b200 as spx
    from spinfemx_b200 import _lib

    rank, ws, local = dist_init(a.gpus)
    dev = torch.cuda.current_device()
    X, T, m0, H0 = workload(a.nx, a.ny, a.nz, a.h, 2000 + rank)
    N = X.shape[0]
    t0 = time.time()
    hef = spx.EffectiveField(
        X, T, 8e5, Aex=1.3e-11, alpha=0.02, gamma=2.211e5, H0_static=H0, use_demag=True,
        precision=a.precision,
        demag_kwargs=dict(boundary_backend="hmatrix", hmatrix_epsilon=a.hmatrix_epsilon, hmatrix_eta=2.0,
                          hmatrix_leaf_size=a.hmatrix_leaf, ksp_rtol_u1=a.rtol_u1, ksp_rtol_u2=a.rtol_u2,
                          precision=a.precision,
                          hmatrix_precision=a.hmatrix_precision, hmatrix_recompress=bool(a.hmatrix_recompress),
                          warm_start={0: False, 1: True, 2: "extrapolate", 3: "extrapolate_corrected"}[a.warm_start]))
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    dm = hef.demag_field
    Hst = dm.B_hmatrix_gpu.stats()
    Hmem = dm.B_hmatrix_gpu.memory_report()
    m = torch.as_tensor(m0, device="cuda")
    hef.set_state(m)
    # warm-up
    hef.step(a.dt, a.warmup)
    torch.cuda.synchronize()
    c_before = counters(dm)
    sampler = ClockSampler(dev) if rank == 0 else None
    barrier(ws)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    _lib.call("spx_demag_profile_begin", dm.handle)
    st0 = hef.stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    hef.step(a.dt, a.steps)
    ev1.record()
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_cat = np.zeros(8)
    nl_cat = np.zeros(8, np.int64)
    ng_cat = np.zeros(8, np.int64)
    _lib.call("spx_demag_profile_end", dm.handle, _lib.ptr(ms_cat), _lib.ptr(nl_cat), _lib.ptr(ng_cat))
    barrier(ws)
    clocks = sampler.stop() if sampler else None
    st1 = hef.stats()
    c_after = counters(dm)
    ms_max = allmax(ms, ws)
    # accuracy: the final state's demag field against an FP64 evaluation, the H-matrix
    # against the reference's dense rows, and the trajectory against an FP64 trajectory
    mfin = hef.get_state().clone()
    err = rows_err = drift = hmat_arrays = hef64 = None
    want_batch = rank == 0 and ws == 1 and a.batched > 1
    if rank == 0 and a.check_error:
        rows_err = rows_err_vs_reference(spx, X, T, dm.B_hmatrix_gpu)
        err, drift, hmat_arrays, hef64 = accuracy_vs_f64(spx, X, T, H0, m0, mfin, hef, a,
                                                         export=bool(a.cpu_baseline and ws == 1), keep=want_batch)
        hef.set_state(mfin)
    # the mixed + batched form: films of this mesh integrated together (one GPU)
    batched = None
    if want_batch:
        batched = batched_film_steps(spx, a, X, T, H0, a.batched,
                                     hef64.demag_field if hef64 is not None else None)
        del hef64
        torch.cuda.empty_cache()
    # end-to-end through the host-buffer entry point (pinned), one step per call
    e2e = None
    if not a.no_e2e:
        hin = torch.empty(3 * N, dtype=torch.float64).pin_memory()
        hout = torch.empty(3 * N, dtype=torch.float64).pin_memory()
        hin.copy_(mfin.cpu())
        ke = max(1, min(a.steps, a.e2e_steps))
        # warm: the accuracy check above ran other trajectories through the same solvers, and
        # each RK stage's Krylov start extrapolates from its last five solutions
        for _ in range(max(a.warmup, 5)):
            hef.run_host(hin, a.dt, 1, out=hout)
            hin, hout = hout, hin
        barrier(ws)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        for _ in range(ke):
            hef.run_host(hin, a.dt, 1, out=hout)
            hin, hout = hout, hin
        torch.cuda.synchronize()
        el = allmax(time.perf_counter() - t1, ws)
        e2e = {"value": job_rate(ke, el * 1e3, ws), "unit": "steps/s", "h2d_bytes_per_step": 3 * N * 8,
               "d2h_bytes_per_step": 3 * N * 8, "steps": ke}
    if rank != 0:
        finish(ws)
        return
    # roofline of the dominant kernel group
    cats = ["div", "u1_solve", "boundary_apply", "u2_rhs", "u2_solve", "phi", "stage"]
    dc = [c_after[0][k] - c_before[0][k] for k in range(3)], [c_after[1][k] - c_before[1][k] for k in range(3)]
    nnz, nnzI = fem_nnz(spx, X, T, dm)
    levels = dm.amg_levels()
    bm = bytes_model(Hst, nnz, N, dm.Nb, dm.NI, nnzI, dc, Hmem, levels)
    per = {}
    for k, name in enumerate(cats):
        if ng_cat[k] == 0:
            continue
        avg_ms = ms_cat[k] / ng_cat[k]
        b = bm.get(name)
        per[name] = {"ms_total": round(float(ms_cat[k]), 3), "executions": int(ng_cat[k]),
                     "kernel_launches": int(nl_cat[k]),
                     "avg_ms": round(float(avg_ms), 4), "share": round(float(ms_cat[k] / ms), 4)}
        if b:
            per[name]["algorithmic_bytes"] = float(b)
            per[name]["achieved_GBps"] = round(b / (avg_ms * 1e-3) / 1e9, 1)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    dom = max((k for k in per if "achieved_GBps" in per[k]), key=lambda k: per[k]["ms_total"])
    traffic = None
    if a.traffic:
        traffic = a.traffic.get(dom)
    elif dom in TRAFFIC_PER_ALGORITHMIC_BYTE and "algorithmic_bytes" in per[dom]:
        # measured DRAM bytes per launch on a smaller film, scaled by this launch's
        # algorithmic bytes (both grow with the H-matrix's factor bytes)
        traffic = round(TRAFFIC_PER_ALGORITHMIC_BYTE[dom] * per[dom]["algorithmic_bytes"])
    roof = {"bound": "hbm", "kernel": dom, "achieved": per[dom]["achieved_GBps"], "peak": peak,
            "peak_source": peak_src, "unit": "GB/s", "frac": round(per[dom]["achieved_GBps"] / peak, 4),
            "traffic": traffic, "traffic_unit": "bytes per launch"}
    launches = int(sum(int(x) for x in nl_cat[:7]))
    line = {
        "metric": METRIC, "value": round(job_rate(a.steps, ms_max, ws), 4), "unit": "steps/s", "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": round(ms_max / a.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": {"f32": "fp32", "f64": "fp64", "mixed": "fp64 vectors / fp32 operators"}[a.precision],
        "data": "synthetic (seeded Kuhn-box film and magnetisation)",
        "config": {"workload": f"film {a.nx}x{a.ny}x{a.nz} cubes @{a.h}nm, N={N}, Nb={dm.Nb}, H-matrix ACA "
                               f"{a.hmatrix_epsilon:g} leaf {a.hmatrix_leaf} eta 2, RK4 dt {a.dt:g}s, {a.precision} "
                               f"(H factors {dm.hmatrix_precision}"
                               f"{', SVD-recompressed' if a.hmatrix_recompress else ''})",
                   "nodes": N, "boundary_nodes": dm.Nb, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (H-matrix factors %.1f GB per apply)" % (
                       (Hmem["far_bytes"] + Hmem["near_bytes"]) / 1e9),
                   "l2_persisting": l2_persisting(),
                   "cg_start": {0: "zero", 1: "previous", 2: "extrapolated per RK stage",
                                3: "extrapolated per RK stage, corrected by stage 1"}[a.warm_start],
                   "rtol_u1": a.rtol_u1, "rtol_u2": a.rtol_u2,
                   "demag_rel_err_vs_fp64": err},
        "hmatrix_rows_err_vs_reference": rows_err,
        "m_drift_vs_f64": drift,
        "e2e": e2e,
        "roofline": roof,
        "kernels": per,
        "hmatrix": {"build_s": round(Hst["build_time_seconds"], 2), "n_far": Hst["n_far"], "n_near": Hst["n_near"],
                    "avg_rank": round(Hst["average_far_rank"], 2), "max_rank": Hst["max_observed_rank"],
                    "far_entries": Hst["far_entries"], "near_entries": Hst["near_entries"]},
        "amg_levels": [[lv["rows"], lv["nnz_A"]] for lv in levels],
        "cg": {"u1_iters_per_solve": round(dc[0][0] / max(dc[0][2], 1), 1),
               "u1_refinements_per_solve": round(dc[0][1] / max(dc[0][2], 1), 2),
               "u2_iters_per_solve": round(dc[1][0] / max(dc[1][2], 1), 1),
               "u2_refinements_per_solve": round(dc[1][1] / max(dc[1][2], 1), 2),
               "u1_start_rel_residual": float("%.3g" % ((c_after[2][0] - c_before[2][0]) / max(dc[0][2], 1))),
               "u1_final_rel_residual": float("%.3g" % ((c_after[2][1] - c_before[2][1]) / max(dc[0][2], 1))),
               "u2_start_rel_residual": float("%.3g" % ((c_after[3][0] - c_before[3][0]) / max(dc[1][2], 1))),
               "u2_final_rel_residual": float("%.3g" % ((c_after[3][1] - c_before[3][1]) / max(dc[1][2], 1)))},
        "setup_s": round(setup_s, 1),
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if batched is not None:
        batched["vs_single_film"] = round(batched["value"] / line["value"], 3)
        line["batched"] = batched
    if a.cpu_baseline and ws == 1:
        line["cpu_baseline"] = cpu_baseline(a, hmat_arrays if hmat_arrays is not None else film_hmatrix_arrays(a))
        del hmat_arrays
    print(json.dumps(line), flush=True)
    finish(ws)


def batched_film_steps(spx, a, X, T, H0, R, ref_demag=None):
    """The mixed + batched form on one GPU: R films of this mesh (one seeded m0 each, the
    seeds of `--batch R`) integrated together as one ensemble: ONE H-matrix applied to all
    films per stage (far field on the tensor cores for batches of 8), the u1 hierarchy shared
    by the identical diagonal blocks.  Film-steps/s over a.batched_steps RK4 steps, and film
    0's demag field at the final state against the FP64 field `ref_demag`."""
    import ctypes as C_
    import torch
    from spinfemx_b200 import _lib
    N = X.shape[0]
    m0s = [workload(a.nx, a.ny, a.nz, a.h, 2000 + j)[2] for j in range(R)]
    dk = dict(hmatrix_epsilon=a.hmatrix_epsilon, hmatrix_eta=2.0, hmatrix_leaf_size=a.hmatrix_leaf,
              ksp_rtol_u1=a.rtol_u1, ksp_rtol_u2=a.rtol_u2, hmatrix_precision=a.hmatrix_precision,
              hmatrix_recompress=bool(a.hmatrix_recompress),
              warm_start={0: False, 1: True, 2: "extrapolate", 3: "extrapolate_corrected"}[a.warm_start])
    t0 = time.time()
    ens = spx.LLGEnsemble([(X, T)] * R, 8e5, Aex=1.3e-11, alpha=0.02, H0=[H0] * R, dense_max_nb=0,
                          precision=a.precision, demag_kwargs=dk)
    dm = ens.hef.demag_field
    tc_bytes = None
    if R == 8:
        hh = C_.c_void_p()
        _lib.call("spx_demag_ensemble_hmat", dm.handle, 0, C_.byref(hh))
        nb = C_.c_int64()
        _lib.call("spx_hmat_tensor_cores", hh, 1, C_.byref(nb))
        tc_bytes = nb.value
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    ens.set_state(m0s)
    ens.step(a.dt, max(a.warmup, 5))  # the Krylov starts extrapolate from five solutions per stage
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.step(a.dt, a.batched_steps)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    err = None
    if ref_demag is not None:
        mall = ens.get_state()
        Hall = torch.empty_like(mall)
        dm.compute_vec(mall, Hall)
        m_0 = mall[: 3 * N].contiguous()
        Hr = torch.empty_like(m_0)
        ref_demag.compute_vec(m_0, Hr)
        err = float(torch.linalg.norm(Hall[: 3 * N] - Hr) / torch.linalg.norm(Hr))
    del ens
    torch.cuda.empty_cache()
    return {"films": R, "value": round(1000.0 * R * a.batched_steps / ms, 4), "unit": "film-steps/s",
            "ms_per_step": round(ms / a.batched_steps, 4), "steps": a.batched_steps,
            "tensor_cores": tc_bytes is not None, "tensor_core_plan_bytes": tc_bytes,
            "demag_rel_err_vs_fp64_film0": err, "setup_s": round(setup_s, 1)}


def ku_fourier_map(X, seed, mean=2e5, std=5e4, modes=16):
    """Seeded smooth nodal Ku map: sum of `modes` in-plane cosine modes (wave numbers 1-4 per
    axis over the film), normalised to the given mean and standard deviation."""
    rng = np.random.default_rng(seed)
    lo, hi = X.min(axis=0), X.max(axis=0)
    L = np.where(hi - lo > 0, hi - lo, 1.0)
    f = np.zeros(X.shape[0])
    for _ in range(modes):
        k = rng.integers(-4, 5, size=2)
        while not k.any():
            k = rng.integers(-4, 5, size=2)
        ph = rng.uniform(0.0, 2 * math.pi)
        f += rng.normal() / np.linalg.norm(k) * np.cos(2 * math.pi * (k[0] * (X[:, 0] - lo[0]) / L[0]
                                                                   + k[1] * (X[:, 1] - lo[1]) / L[1]) + ph)
    f = (f - f.mean()) / f.std()
    return mean + std * f


def run_adjoint(a):
    """Gradient of a trajectory loss through the hand-written adjoint (film 100x100x2 @2 nm).

    Loss ||m(T) - m_target||^2 after 400 RK4 steps of 25 fs; m_target is the trajectory from
    a second seeded Ku map.  Gradient with respect to the nodal Ku map and the uniform
    applied field (autograd Function, checkpoints every 20 steps), checked against central
    differences (h = 1e-4 relative) of the same pipeline on 32 seeded directions and against
    the forward-mode tangent on 4 of them."""
    import torch
    import spinfemx_b200 as spx
    rank, ws, local = dist_init(a.gpus)
    nx, ny, nz, h = 100, 100, 2, 2.0
    X, T = spx.kuhn_box(nx, ny, nz, h)
    N = X.shape[0]
    rng = np.random.default_rng(5000 + rank)
    m0 = np.tile([1.0, 0.0, 0.0], (N, 1)) + rng.normal(0.0, 0.05, (N, 3))
    m0 = (m0 / np.linalg.norm(m0, axis=1)[:, None]).ravel()
    Ku = ku_fourier_map(X, 5001 + rank)
    Ku_t = ku_fourier_map(X, 5002 + rank)
    H0 = np.array([0.0, 0.05 / MU0, 0.0])
    nsteps, dt, every = a.adj_steps, 25e-15, 20
    t0 = time.time()
    hef = spx.EffectiveField(
        X, T, 8e5, Aex=1.3e-11, alpha=0.1, Ku=0.0, Ku_nodes=Ku, n_ani_vec=np.tile([0.0, 0.0, 1.0], N),
        H0_static=H0, use_demag=True, precision="mixed",
        demag_kwargs=dict(boundary_backend="hmatrix", hmatrix_epsilon=1e-5, hmatrix_eta=2.0, hmatrix_leaf_size=64,
                          hmatrix_precision="f32", ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10, ksp_atol=0.0,
                          ksp_maxit_u1=20000, ksp_maxit_u2=20000, precision="mixed",
                          warm_start="extrapolate_corrected"))
    torch.cuda.synchronize()
    setup_s = time.time() - t0

    def run(Ku_map, H):
        hef.set_anisotropy_map(Ku_map)
        hef.set_uniform_field(*H)
        hef.set_state(torch.as_tensor(m0, device="cuda"))
        hef.step(dt, nsteps)
        return hef.get_state()

    mt = run(Ku_t, H0).clone()

    def loss_of(Ku_map, H):
        return float(torch.sum((run(Ku_map, H) - mt) ** 2).item())

    # warm-up of both passes
    for _ in range(max(1, a.warmup)):
        Kt = torch.as_tensor(Ku, device="cuda").requires_grad_(True)
        Ht = torch.as_tensor(H0, device="cuda").requires_grad_(True)
        mT = spx.llg_trajectory(hef, torch.as_tensor(m0, device="cuda"), dt, min(nsteps, 2 * every), Ku=Kt, H0=Ht,
                                checkpoint_every=every)
        torch.sum((mT - mt) ** 2).backward()
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    if sampler:
        sampler.start()
    Kt = torch.as_tensor(Ku, device="cuda").requires_grad_(True)
    Ht = torch.as_tensor(H0, device="cuda").requires_grad_(True)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record()
    mT = spx.llg_trajectory(hef, torch.as_tensor(m0, device="cuda"), dt, nsteps, Ku=Kt, H0=Ht,
                            checkpoint_every=every)
    loss = torch.sum((mT - mt) ** 2)
    e1.record()
    loss.backward()
    e2.record()
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    fwd_ms, bwd_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    gKu, gH = Kt.grad.cpu().numpy(), Ht.grad.cpu().numpy()
    L0 = float(loss.item())
    # central differences on seeded directions (Ku map and field together)
    drng = np.random.default_rng(6000)
    hrel = 1e-4
    errs, tan_errs = [], []
    t1 = time.time()
    for k in range(a.fd_dirs):
        dK = drng.normal(size=N) * 5e4
        dH = drng.normal(size=3) * np.linalg.norm(H0)
        Lp = loss_of(Ku + hrel * dK, H0 + hrel * dH)
        Lm = loss_of(Ku - hrel * dK, H0 - hrel * dH)
        fd = (Lp - Lm) / (2 * hrel)
        g = float(gKu @ dK + gH @ dH)
        errs.append(abs(g - fd) / max(abs(fd), 1e-300))
        if k < a.tangent_dirs:
            mT2, dmT = spx.trajectory_tangent(hef, m0, dt, nsteps, dKu=dK, dH0=dH, Ku=Ku, H0=H0)
            tan = float(torch.sum(2.0 * (mT2 - mt) * dmT).item())
            tan_errs.append(abs(tan - g) / max(abs(g), 1e-300))
    fd_s = time.time() - t1
    if rank != 0:
        finish(ws)
        return
    tot_ms = fwd_ms + bwd_ms
    line = {
        "metric": "trajectory-loss gradient wrt nodal Ku map + applied field, film 100x100x2 @2nm, 400 RK4 steps",
        "value": round(tot_ms / 1e3, 3), "unit": "s per gradient (forward + backward)", "n_gpus": ws,
        "steps": nsteps, "warmup": a.warmup, "ms_per_step": round(tot_ms / nsteps, 4), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp64 vectors / fp32 operators (H factors f32)",
        "data": "synthetic (seeded Kuhn-box film, seeded 16-mode Fourier Ku maps)",
        "config": {"workload": f"film {nx}x{ny}x{nz} cubes @{h}nm, N={N}, Nb={hef.demag_field.Nb}, H-matrix ACA 1e-5 "
                               f"f32, alpha 0.1, Ku(x) mean 2e5 std 5e4 along z, B 50 mT along y, dt 25 fs",
                   "checkpoint_every": every, "rtol": 1e-10, "parallelism": f"replicas x{ws}"},
        "forward_ms": round(fwd_ms, 1), "backward_ms": round(bwd_ms, 1),
        "backward_over_forward": round(bwd_ms / fwd_ms, 2),
        "loss": L0,
        "fd_check": {"directions": a.fd_dirs, "h_rel": hrel, "max_rel_err": float(max(errs)) if errs else None,
                     "median_rel_err": float(np.median(errs)) if errs else None, "seconds": round(fd_s, 1)},
        "tangent_check": {"directions": len(tan_errs), "max_rel_err": float(max(tan_errs)) if tan_errs else None},
        "grad_norms": {"Ku": float(np.linalg.norm(gKu)), "H0": float(np.linalg.norm(gH))},
        "setup_s": round(setup_s, 1),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    finish(ws)


def run_film_batch(a):
    """LLG film-steps/s for a batch of films of the same 0.48M-node mesh (different seeded m0)
    integrated together: one ensemble (block-diagonal FEM and Poisson systems) whose boundary
    operator is ONE H-matrix applied to all films at once (spx_hmat_apply_multi)."""
    import torch
    import spinfemx_b200 as spx
    from spinfemx_b200 import _lib
    rank, ws, local = dist_init(a.gpus)
    R = a.batch
    X, T, _, H0 = workload(a.nx, a.ny, a.nz, a.h, 2000)
    N = X.shape[0]
    m0s = [workload(a.nx, a.ny, a.nz, a.h, 2000 + 100 * rank + j)[2] for j in range(R)]
    t0 = time.time()
    dk = dict(hmatrix_epsilon=1e-5, hmatrix_eta=2.0, hmatrix_leaf_size=64, ksp_rtol_u1=a.rtol_u1,
              ksp_rtol_u2=a.rtol_u2, hmatrix_precision=a.hmatrix_precision,
              hmatrix_recompress=bool(a.hmatrix_recompress),
              warm_start={0: False, 1: True, 2: "extrapolate", 3: "extrapolate_corrected"}[a.warm_start])
    ens = spx.LLGEnsemble([(X, T)] * R, 8e5, Aex=1.3e-11, alpha=0.02, H0=[H0] * R, dense_max_nb=0,
                          precision=a.precision, demag_kwargs=dk)
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    dm = ens.hef.demag_field
    tc_bytes = None
    if a.tensor_cores:  # far field of the shared H-matrix on the tensor cores (batches of 8)
        import ctypes as C_
        hh = C_.c_void_p()
        _lib.call("spx_demag_ensemble_hmat", dm.handle, 0, C_.byref(hh))
        nb = C_.c_int64()
        _lib.call("spx_hmat_tensor_cores", hh, 1, C_.byref(nb))
        tc_bytes = nb.value
    ens.set_state(m0s)
    ens.step(a.dt, a.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    barrier(ws)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.step(a.dt, a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = allmax(e0.elapsed_time(e1), ws)
    clocks = sampler.stop() if sampler else None
    c_before = counters(dm)
    _lib.call("spx_demag_profile_begin", dm.handle)
    ens.step(a.dt, min(a.steps, 10))
    ms_cat = np.zeros(8)
    nl_cat = np.zeros(8, np.int64)
    ng_cat = np.zeros(8, np.int64)
    _lib.call("spx_demag_profile_end", dm.handle, _lib.ptr(ms_cat), _lib.ptr(nl_cat), _lib.ptr(ng_cat))
    c_after = counters(dm)
    dc = [[c_after[j][k] - c_before[j][k] for k in range(3)] for j in range(2)]
    nprof = min(a.steps, 10)
    cats = ["div", "u1_solve", "boundary_apply", "u2_rhs", "u2_solve", "phi", "stage"]
    phases = {c: round(float(ms_cat[k]) / nprof, 4) for k, c in enumerate(cats) if ng_cat[k]}
    err = None
    if rank == 0 and a.check_error:  # film 0 of the batch against an FP64 evaluation of its state
        mall = ens.get_state()
        Hall = torch.empty_like(mall)
        dm.compute_vec(mall, Hall)
        m_0 = mall[: 3 * N].contiguous()
        ref = spx.DemagFieldLindholmGPU(X, T, 8e5, boundary_backend="hmatrix", hmatrix_epsilon=1e-5,
                                        precision="f64", ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10,
                                        ksp_maxit_u1=50000, ksp_maxit_u2=50000, ksp_atol=0.0,
                                        hmatrix_precision="f64")
        Hr = torch.empty_like(m_0)
        ref.compute_vec(m_0, Hr)
        err = float(torch.linalg.norm(Hall[: 3 * N] - Hr) / torch.linalg.norm(Hr))
        del ref
    single = None
    if rank == 0 and a.compare_single:
        # the same film alone (same precision, H-matrix settings and solver tolerances), timed
        # over the same number of steps: the batched form's gain over one film at a time
        hef1 = spx.EffectiveField(X, T, 8e5, Aex=1.3e-11, alpha=0.02, H0_static=H0, use_demag=True,
                                  precision=a.precision,
                                  demag_kwargs=dict(dk, precision=a.precision, boundary_backend="hmatrix"))
        hef1.set_state(torch.as_tensor(m0s[0], device="cuda"))
        hef1.step(a.dt, a.warmup)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record()
        hef1.step(a.dt, a.steps)
        f1.record()
        torch.cuda.synchronize()
        rate1 = 1000.0 * a.steps / f0.elapsed_time(f1)
        single = {"steps_per_s": round(rate1, 4), "precision": a.precision,
                  "h_factors": hef1.demag_field.hmatrix_precision}
        del hef1
        torch.cuda.empty_cache()
    if rank != 0:
        finish(ws)
        return
    Hmem = dm.B_hmatrix_gpu.memory_report() if dm.B_hmatrix_gpu is not None else {}
    line = {
        "metric": f"LLG film-steps/s at 0.48M nodes, batch of {R} films sharing one H-matrix",
        "value": round(job_rate(R * a.steps, ms, ws), 4), "unit": "film-steps/s", "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": {"f32": "fp32", "f64": "fp64", "mixed": "fp64 vectors / fp32 operators"}[a.precision],
        "data": "synthetic (seeded Kuhn-box film, one seeded magnetisation per film)",
        "config": {"workload": f"{R} x film {a.nx}x{a.ny}x{a.nz} cubes @{a.h}nm, N={N} each, Nb={dm.Nb // R} "
                               f"each, one H-matrix ACA 1e-5 leaf 64 eta 2 (factors {dm.hmatrix_precision}) "
                               f"applied to all films, RK4 dt {a.dt:g}s",
                   "batch": R, "rtol_u1": a.rtol_u1, "rtol_u2": a.rtol_u2,
                   "tensor_cores": bool(a.tensor_cores), "tensor_core_plan_bytes": tc_bytes,
                   "hmatrix_factor_gb": round((Hmem.get("far_bytes", 0) + Hmem.get("near_bytes", 0)) / 1e9, 2),
                   "demag_rel_err_vs_fp64_film0": err},
        "phases_ms_per_step": phases,
        "single_film": single,
        "vs_single_film": (round(job_rate(R * a.steps, ms, ws) / single["steps_per_s"], 3) if single else None),
        "cg": {"u1_iters_per_solve": round(dc[0][0] / max(dc[0][2], 1), 1),
               "u1_refinements_per_solve": round(dc[0][1] / max(dc[0][2], 1), 2),
               "u2_iters_per_solve": round(dc[1][0] / max(dc[1][2], 1), 1),
               "u2_refinements_per_solve": round(dc[1][1] / max(dc[1][2], 1), 2)},
        "amg_levels": [[lv["rows"], lv["nnz_A"]] for lv in dm.amg_levels()],
        "l2_persisting": l2_persisting(),
        "setup_s": round(setup_s, 1),
        "gpu_launches": int(sum(int(x) for x in nl_cat[:7])) * a.steps // max(nprof, 1),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    finish(ws)


def ensemble_boxes(n, seed):
    """Ensemble box shapes: lateral sides U[20, 120] nm and thickness in {4, 6, 8, 10} nm,
    snapped to 2 nm cubes (Kuhn split)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nx, ny = (int(round(rng.uniform(20.0, 120.0) / 2.0)) for _ in range(2))
        nz = int(rng.choice([4, 6, 8, 10])) // 2
        out.append((max(nx, 1), max(ny, 1), nz))
    return out


def run_ensemble(a):
    """Sample-steps/s of a batched ensemble of 64 independent boxes (sides U[20, 120] nm,
    thickness 4-10 nm, 2 nm cubes)."""
    import torch
    import spinfemx_b200 as spx
    from spinfemx_b200.ensemble import ShardedEnsemble
    rank, ws, local = dist_init(a.gpus)
    # one ensemble of a.samples boxes (the same draw on every rank), split by sample across
    # the ranks with balanced cost; no exchange until the final gather
    boxes = ensemble_boxes(a.samples, 7000)
    meshes = [spx.kuhn_box(nx, ny, nz, 2.0) for nx, ny, nz in boxes]
    rng = np.random.default_rng(7100)
    Bz = rng.uniform(-0.5, 0.5, size=len(meshes))
    m0_all = []
    for X, _ in meshes:
        m = rng.normal(size=(X.shape[0], 3))
        m0_all.append((m / np.linalg.norm(m, axis=1)[:, None]).ravel())
    mat = dict(Aex=1.6e-11, Ku=8e5, D_int=3e-3, alpha=0.3)
    dk = dict(hmatrix_epsilon=1e-5, hmatrix_eta=2.0, hmatrix_leaf_size=64, ksp_rtol_u1=a.rtol_u1,
              ksp_rtol_u2=a.rtol_u2, warm_start={0: False, 1: True, 2: "extrapolate", 3: "extrapolate_corrected"}[
                  a.warm_start])
    t0 = time.time()
    sh = ShardedEnsemble(meshes, 1.1e6, rank=rank, world_size=ws, H0=[[0.0, 0.0, b / MU0] for b in Bz],
                         dense_max_nb=4096, precision=a.precision, demag_kwargs=dk, graph=bool(a.graph), **mat)
    ens = sh.local
    all_meshes = meshes
    meshes = [all_meshes[i] for i in sh.mine]
    Bz_all, Bz = Bz, Bz[sh.mine]
    m0 = [m0_all[i] for i in sh.mine]
    torch.cuda.synchronize()
    setup_s = time.time() - t0
    dm = ens.hef.demag_field
    dt = 20e-15
    ens.set_state(m0)
    ens.step(dt, a.warmup)
    torch.cuda.synchronize()
    sampler = ClockSampler(torch.cuda.current_device()) if rank == 0 else None
    barrier(ws)
    torch.cuda.synchronize()
    if sampler:
        sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ens.step(dt, a.steps)
    e1.record()
    torch.cuda.synchronize()
    ms = allmax(e0.elapsed_time(e1), ws)
    clocks = sampler.stop() if sampler else None
    # per-phase breakdown on a separate (profiled) run of the same number of steps
    from spinfemx_b200 import _lib
    _lib.call("spx_demag_profile_begin", dm.handle)
    ens.step(dt, a.steps)
    ms_cat = np.zeros(8)
    nl_cat = np.zeros(8, np.int64)
    ng_cat = np.zeros(8, np.int64)
    _lib.call("spx_demag_profile_end", dm.handle, _lib.ptr(ms_cat), _lib.ptr(nl_cat), _lib.ptr(ng_cat))
    cats = ["div", "u1_solve", "boundary_apply", "u2_rhs", "u2_solve", "phi", "stage"]
    phases = {c: {"ms_per_step": round(float(ms_cat[k]) / a.steps, 4), "launches_per_step":
                  round(float(nl_cat[k]) / a.steps, 1)} for k, c in enumerate(cats) if ng_cat[k]}
    launches = int(nl_cat[:7].sum())
    info = np.zeros(6, np.int64)
    _lib.call("spx_demag_ensemble_info", dm.handle, _lib.ptr(info))
    c_a = counters(dm)
    wm = 8 if a.precision == "f64" else 4
    wv = 4 if a.precision == "f32" else 8
    bnd_bytes = float(info[2] * wm + info[4] + info[5] + 6 * dm.Nb * wv)
    if "boundary_apply" in phases:
        per_apply = phases["boundary_apply"]["ms_per_step"] / 4.0
        phases["boundary_apply"]["algorithmic_bytes_per_apply"] = bnd_bytes
        phases["boundary_apply"]["achieved_GBps"] = round(bnd_bytes / (per_apply * 1e-3) / 1e9, 1)
    # the same samples one by one (separate field objects, same options), a few of them timed
    seq = None
    if a.ens_compare and rank == 0:
        per = []
        nchk = min(a.ens_compare, len(meshes))
        idx = np.linspace(0, len(meshes) - 1, nchk).astype(int)
        for k in idx:
            X, T = meshes[k]
            kw = dict(dk, boundary_backend="dense" if dm_nb(spx, X, T) <= 4096 else "hmatrix", precision=a.precision)
            hef = spx.EffectiveField(X, T, 1.1e6, n_ani_vec=[0.0, 0.0, 1.0], n0_int_vec=[0.0, 0.0, 1.0],
                                     H0_static=[0.0, 0.0, Bz[k] / MU0], use_demag=True, demag_kwargs=kw, **mat)
            hef.set_state(torch.as_tensor(m0[k], device="cuda"))
            hef.step(dt, a.warmup)
            torch.cuda.synchronize()
            f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            f0.record()
            hef.step(dt, a.steps)
            f1.record()
            torch.cuda.synchronize()
            per.append((int(k), f0.elapsed_time(f1) / a.steps, int(X.shape[0])))
        # sequential time for all samples: per-node cost interpolated from the timed samples
        tn = np.array([p[1] for p in per])
        nn = np.array([p[2] for p in per], dtype=np.float64)
        coef = np.polyfit(nn, tn, 1) if len(per) > 1 else np.array([0.0, tn[0]])
        est = float(sum(max(np.polyval(coef, X.shape[0]), tn.min()) for X, _ in all_meshes))
        seq = {"timed_samples": [{"sample": p[0], "nodes": p[2], "ms_per_step": round(p[1], 4)} for p in per],
               "est_ms_per_ensemble_step": round(est, 3),
               "est_sample_steps_per_s": round(len(all_meshes) * 1e3 / est, 1)}
    sh.set_state(m0_all)
    sh.step(dt, 1)
    gathered = sh.gather(dst=0)  # the only exchange: final states to rank 0 (untimed)
    if rank != 0:
        finish(ws)
        return
    gathered_ok = gathered is not None and len(gathered) == len(all_meshes) and all(
        bool(np.isfinite(g).all()) for g in gathered)
    nodes = int(sum(X.shape[0] for X, _ in all_meshes))
    blk = {"dense": int(sum(1 for X, T in all_meshes if dm_nb(spx, X, T) <= 4096))}
    blk["hmatrix"] = len(all_meshes) - blk["dense"]
    line = {
        "metric": "ensemble sample-steps/s: 64 independent boxes (sides U[20,120] nm, thickness 4-10 nm @2 nm), one launch per phase",  # noqa: E501
        "value": round(len(all_meshes) * a.steps / (ms * 1e-3), 2), "unit": "sample-steps/s", "n_gpus": ws,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None,
        "dtype": {"f32": "fp32", "f64": "fp64", "mixed": "fp64 vectors / fp32 operators"}[a.precision],
        "data": "synthetic (seeded box sizes, fields and magnetisations)",
        "config": {"workload": f"{len(all_meshes)} boxes, sides U[20,120] nm, thickness {{4,6,8,10}} nm @2 nm, "
                               f"{nodes} nodes in total, Ms 1.1e6, A 1.6e-11, Ku 8e5 z, D_int 3e-3, alpha 0.3, "
                               f"Bz U[-0.5,0.5] T, RK4 dt 20 fs",
                   "nodes": nodes, "boundary_nodes_rank0": int(dm.Nb), "boundary_blocks": blk,
                   "rtol_u1": a.rtol_u1, "rtol_u2": a.rtol_u2,
                   "parallelism": f"one ensemble split by sample over {ws} rank(s) (cost-balanced), final gather",
                   "rank0_samples": len(sh.mine), "gathered_all_samples": gathered_ok},
        "phases": phases,
        "graph": ens.hef.graph_stats(),
        "boundary": {"dense_samples": int(info[1]), "dense_entries": int(info[2]), "hmatrix_rows": int(info[3]),
                     "hmatrix_far_bytes": int(info[4]), "hmatrix_near_bytes": int(info[5])},
        "cg": {"u1_iters_per_solve": round(c_a[0][0] / max(c_a[0][2], 1), 1),
               "u2_iters_per_solve": round(c_a[1][0] / max(c_a[1][2], 1), 1)},
        "gpu_launches_per_step": round(launches / a.steps, 1),
        "unbatched": seq,
        "setup_s": round(setup_s, 1),
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    finish(ws)


def dm_nb(spx, X, T):
    return int(spx.boundary_data(X, T)["bverts"].shape[0])


def counters(dm):
    from spinfemx_b200 import _lib
    c1 = np.zeros(4, np.int64)
    c2 = np.zeros(4, np.int64)
    r1 = np.zeros(2)
    r2 = np.zeros(2)
    _lib.call("spx_demag_counters", dm.handle, _lib.ptr(c1), _lib.ptr(c2))
    _lib.call("spx_demag_residuals", dm.handle, _lib.ptr(r1), _lib.ptr(r2))
    return c1.tolist(), c2.tolist(), r1.tolist(), r2.tolist()


def fem_nnz(spx, X, T, dm):
    f = spx.fem_assemble(X, T)
    nnz = int(f["rowptr"][-1])
    bd = np.zeros(X.shape[0], bool)
    bd[spx.boundary_data(X, T)["bverts"]] = True
    rows = np.repeat(np.arange(X.shape[0]), np.diff(f["rowptr"]))
    nnzI = int(np.count_nonzero(~bd[rows] & ~bd[f["col"]]))
    return nnz, nnzI


def accuracy_vs_f64(spx, X, T, H0, m0, mfin, hef, a, export=False, keep=False):
    """Against an all-FP64 field (FP64 vectors, operators and H-matrix factors, rtol 1e-10):
    (1) the relative L2 error of the working-precision demag field at the final state;
    (2) max |m - m_f64| after a.drift_steps RK4 steps from m0 (both runs from the same
    state, same dt); (3) with `export`, the FP64 H-matrix in the reference's cache schema
    (for the CPU baseline); (4) with `keep`, the FP64 effective field itself (else None)."""
    import torch
    hef64 = spx.EffectiveField(
        X, T, 8e5, Aex=1.3e-11, alpha=0.02, gamma=2.211e5, H0_static=H0, use_demag=True, precision="f64",
        demag_kwargs=dict(boundary_backend="hmatrix", hmatrix_epsilon=a.hmatrix_epsilon, hmatrix_eta=2.0,
                          hmatrix_leaf_size=a.hmatrix_leaf, ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10,
                          ksp_maxit_u1=50000, ksp_maxit_u2=50000, ksp_atol=0.0, precision="f64",
                          hmatrix_precision="f64", warm_start="extrapolate_corrected"))
    Hr = torch.empty_like(mfin)
    hef64.demag_field.compute_vec(mfin, Hr)
    Hw = torch.empty_like(mfin)
    hef.demag_field.compute_vec(mfin, Hw)
    e = float(torch.linalg.norm(Hw - Hr) / torch.linalg.norm(Hr))
    drift = None
    if a.drift_steps > 0:
        m0t = torch.as_tensor(m0, device="cuda")
        hef64.set_state(m0t)
        hef64.step(a.dt, a.drift_steps)
        hef.set_state(m0t)
        hef.step(a.dt, a.drift_steps)
        d = float((hef.get_state() - hef64.get_state()).abs().max().item())
        drift = {"steps": a.drift_steps, "max_abs_dm": d, "bar": 1e-5}
    arrays = hef64.demag_field.B_hmatrix_gpu.cache_arrays() if export else None
    if keep:
        return e, drift, arrays, hef64
    del hef64
    torch.cuda.synchronize()
    return e, drift, arrays, None


def finish(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------- CPU (oracle)
def boundary_operator_cpu(arrays):
    """The CPU H-matrix apply (oracle.hmatrix.PackedCPU: HMatrixCPUData.matvec_cpu restated
    over the reference's cache arrays, on all host threads)."""
    from oracle import hmatrix as ohm
    H = ohm.PackedCPU(arrays)
    return H.matvec, ("the oracle's restatement of HMatrixCPUData.matvec_cpu (storage.py:60-75) on "
                      f"{H.threads} threads")


def _numba_spmv():
    """Row-parallel CSR SpMV on all host threads (numba prange)."""
    from numba import njit, prange

    @njit(parallel=True, cache=False)
    def spmv(indptr, indices, data, x, y):
        for i in prange(indptr.size - 1):
            acc = 0.0
            for k in range(indptr[i], indptr[i + 1]):
                acc += data[k] * x[indices[k]]
            y[i] = acc
    return spmv


class OracleCPU:
    """The FP64 CPU pipeline of one LLG right-hand side on the film (test infrastructure):
    Div m, the u1 Neumann solve, the boundary double layer B (the reference's own CPU
    H-matrix apply, HMatrixCPUData.matvec_cpu, on the film's H-matrix), the u2 Dirichlet
    solve, H = G (u1 + u2) / V, exchange, Zeeman and the LLG RHS.  The P1 operators and
    solves are the oracle's restatement of the reference's DOLFINx / PETSc forms
    (Demag_Lindholm_GPU.py:188-281, 554-670): sparse SpMVs on all host threads (numba),
    u1 / u2 by SuperLU factorised once (single-threaded triangular solves).  The
    H-matrix is the one the GPU built (ACA 1e-5, leaf 64, eta 2, FP64 factors), handed
    over in the reference's cache schema during set-up: the reference's own CPU builder
    needs hours at Nb = 323k.  The reference's Python package cannot travel with the
    benchmark, so every part is the oracle's restatement ("port")."""

    def __init__(self, a, hmat_arrays, seed=2000):
        import scipy.sparse.linalg as spla
        from oracle import fem, lindholm, llg, mesh
        X, T = mesh.kuhn_box(a.nx, a.ny, a.nz, a.h)
        self.N = N = X.shape[0]
        rng = np.random.default_rng(seed)
        m = np.tile([1.0, 0.0, 0.0], (N, 1)) + rng.normal(0.0, 0.05, (N, 3))
        m /= np.linalg.norm(m, axis=1)[:, None]
        self.m = m.ravel()
        th = math.radians(170.0)
        self.H0 = np.tile((0.025 / MU0) * np.array([math.cos(th), math.sin(th), 0.0]), N)
        tris, _ = lindholm.boundary_facets(X, T)
        bv = np.unique(tris.ravel())
        A = fem.stiffness(X, T).tocsr()
        self.vol = fem.lumped_volume(X, T)
        inter = np.ones(N, bool)
        inter[bv] = False
        self.I = np.nonzero(inter)[0]
        self.lu1 = spla.splu(A[1:, 1:].tocsc())
        self.lu2 = spla.splu(A[self.I][:, self.I].tocsc())
        self.ops = {"Div": fem.divergence(X, T, 8e5).tocsr(), "G": fem.gradient_op(X, T).tocsr(),
                    "K": fem.exchange_matrix(X, T, 1.3e-11, 8e5, self.vol).tocsr(),
                    "AIB": A[self.I][:, bv].tocsr()}
        self.spmv = _numba_spmv()
        self.bv = bv
        self.B, self.b_label = boundary_operator_cpu(hmat_arrays)
        self.pref, self.stab = llg.constants(8e5, 2.211e5, 0.02)
        self.llg = llg
        self.threads = int(os.environ.get("NUMBA_NUM_THREADS", os.cpu_count() or 1))

    def mv(self, name, x):
        M = self.ops[name]
        y = np.empty(M.shape[0])
        self.spmv(M.indptr, M.indices, M.data, np.ascontiguousarray(x), y)
        return y

    def rhs(self, m):
        b = self.mv("Div", m)
        b -= b.mean()
        u = np.zeros(self.N)
        u[1:] = self.lu1.solve(b[1:])
        u -= u.mean()
        g = self.B(u[self.bv])                     # boundary double layer (the reference's apply)
        u2 = np.zeros(self.N)
        u2[self.bv] = g
        u2[self.I] = self.lu2.solve(-self.mv("AIB", g))
        H = (self.mv("G", u + u2)).reshape(-1, 3) / self.vol[:, None]
        H = H.ravel() + self.mv("K", m) + self.H0
        return self.llg.rhs(m, H, self.pref, 0.02, 1.0, self.stab)

    def step(self, dt):
        self.m = self.llg.rk4_step(self.rhs, self.m, dt)


def time_cpu_evals(o, n_evals=None, seconds=None):
    """Seconds per right-hand-side evaluation over n_evals evaluations (or as many as fit in
    `seconds`) on the film state; the first evaluation is untimed (numba compile)."""
    m = o.m
    o.rhs(m)
    t = time.perf_counter()
    n = 0
    while True:
        m = m + 1e-3 * o.rhs(m) * 1e-14
        n += 1
        el = time.perf_counter() - t
        if (n_evals is not None and n >= n_evals) or (seconds is not None and el > seconds):
            break
    return el / n, n, el


def cpu_sample_text(o, n, el):
    return (f"{n} right-hand-side evaluation(s) of the FP64 CPU pipeline on the full film (4 per RK4 step; "
            f"steps/s = 1 / (4 x seconds per evaluation)), {el:.1f} s: boundary double layer by {o.b_label}, "
            f"P1 SpMVs on {o.threads} threads (numba), u1/u2 by SuperLU triangular solves (1 thread)")


def cpu_baseline(a, hmat_arrays):
    o = OracleCPU(a, hmat_arrays)
    per, n, el = time_cpu_evals(o, seconds=a.cpu_seconds)
    return {"value": round(1.0 / (4.0 * per), 5), "unit": "steps/s", "cores": o.threads, "kind": "port",
            "sample": cpu_sample_text(o, n, el)}


def run_reference(a):
    """The reference arm: the reference's CPU algorithm for the path (the oracle's FP64
    restatement, with the boundary double layer applied as HMatrixCPUData.matvec_cpu does)
    on the film, on all host threads.
    Set-up (untimed) builds the film's H-matrix on the GPU and hands it over in the
    reference's cache schema.  Each timed step is one right-hand-side evaluation (a
    quarter of an RK4 step); the value is 1 / (4 x seconds per evaluation)."""
    rank = int(os.environ.get("RANK", "0"))
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    os.environ.setdefault("NUMBA_NUM_THREADS", str(os.cpu_count() or 1))
    t0 = time.time()
    arrays = film_hmatrix_arrays(a)
    o = OracleCPU(a, arrays)
    del arrays
    setup_s = time.time() - t0
    if a.warmup:
        time_cpu_evals(o, n_evals=a.warmup)
    per, n, el = time_cpu_evals(o, n_evals=a.steps)
    v = 1.0 / (4.0 * per)
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 5), "unit": "steps/s", "n_gpus": ws,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(4e3 * per, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
            "data": "synthetic (seeded Kuhn-box film and magnetisation)",
            "config": {"workload": f"film {a.nx}x{a.ny}x{a.nz} cubes @{a.h}nm, FP64 CPU pipeline (oracle port) with "
                                   f"the HMatrixCPUData.matvec_cpu boundary apply (H-matrix ACA "
                                   f"{a.hmatrix_epsilon:g} leaf {a.hmatrix_leaf} eta 2), RK4 dt {a.dt:g}s",
                       "parallelism": f"cpu, {o.threads} threads", "setup_s": round(setup_s, 1)},
            "cpu_baseline": {"value": round(v, 5), "unit": "steps/s", "cores": o.threads, "kind": "port",
                             "sample": cpu_sample_text(o, n, el)},
            "e2e": {"value": round(v, 5), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def film_hmatrix_arrays(a):
    """The film's H-matrix (ACA, FP64 factors) in the reference's cache schema: built on the
    GPU when there is one; on a host without a GPU (small films only) by the oracle's
    restatement of the reference's CPU builder (builder.py:186-419)."""
    import torch
    if torch.cuda.is_available():
        import spinfemx_b200 as spx
        torch.cuda.set_device(0)
        X, T = spx.kuhn_box(a.nx, a.ny, a.nz, a.h)
        geom = spx.BoundaryGeometry(X, T)
        H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=a.hmatrix_epsilon, eta=2.0,
                                                                   leaf_size=a.hmatrix_leaf), precision="f64")
        arrays = H.cache_arrays()
        del H, geom
        return arrays
    from oracle import hmatrix as ohm
    from oracle import lindholm, mesh
    X, T = mesh.kuhn_box(a.nx, a.ny, a.nz, a.h)
    bd = lindholm.boundary_data(X, T)
    h = ohm.build(bd, epsilon=a.hmatrix_epsilon, eta=2.0, leaf_size=a.hmatrix_leaf)
    far, perm, diag, near = h.far, h.perm, h.diag_jump, h.near
    meta = np.zeros(len(far), dtype=[("row_start", np.int64), ("row_stop", np.int64), ("col_start", np.int64),
                                     ("col_stop", np.int64), ("rank", np.int64), ("u_offset", np.int64),
                                     ("u_size", np.int64), ("v_offset", np.int64), ("v_size", np.int64),
                                     ("relative_residual", np.float64)])
    uo = vo = 0
    for i, (rs, re, cs, ce, U, V, rel) in enumerate(far):
        meta[i] = (rs, re, cs, ce, U.shape[1], uo, U.size, vo, V.size, rel)
        uo += U.size
        vo += V.size
    return dict(perm=np.asarray(perm, np.int32), diag_jump=np.asarray(diag, np.float64),
                near_data=near.data, near_indices=near.indices.astype(np.int32),
                near_indptr=near.indptr.astype(np.int32), near_shape=np.array(near.shape, np.int64), far_meta=meta,
                far_U_flat=np.concatenate([np.ascontiguousarray(f[4]).ravel() for f in far]) if far else np.zeros(0),
                far_V_flat=np.concatenate([np.ascontiguousarray(f[5]).ravel() for f in far]) if far else np.zeros(0))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["f32", "f64", "mixed"])
    ap.add_argument("--hmatrix-precision", default=None, choices=["f64", "f32", "bf16", "f32_f16"])
    ap.add_argument("--hmatrix-recompress", type=int, default=1,
                    help="SVD-recompress the ACA factors after the build (same tolerance)")
    ap.add_argument("--hmatrix-epsilon", type=float, default=1e-5,
                    help="film: ACA tolerance (the metric is quoted at 1e-5; larger values only for small "
                         "profiling captures of the solver kernels)")
    ap.add_argument("--hmatrix-leaf", type=int, default=64, help="film: H-matrix leaf size (metric: 64)")
    ap.add_argument("--nx", type=int, default=400)
    ap.add_argument("--ny", type=int, default=400)
    ap.add_argument("--nz", type=int, default=2)
    ap.add_argument("--h", type=float, default=2.5)
    ap.add_argument("--dt", type=float, default=5e-14)
    ap.add_argument("--rtol-u1", type=float, default=1e-8)
    ap.add_argument("--rtol-u2", type=float, default=1e-8)
    ap.add_argument("--warm-start", type=int, default=3, help="0 zero, 1 previous, 2 extrapolated per RK stage, 3 extrapolated and corrected")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--check-error", type=int, default=1)
    ap.add_argument("--drift-steps", type=int, default=200, help="film: RK4 steps of the FP64 trajectory check")
    ap.add_argument("--cpu-baseline", type=int, default=1)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--traffic", type=json.loads, default=None,
                    help='per-group DRAM bytes per launch from an ncu capture, e.g. {"u1_solve": 1.2e9}')
    ap.add_argument("--samples", type=int, default=64)
    ap.add_argument("--graph", type=int, default=1, help="ensemble: replay RK4 steps from CUDA graphs")
    ap.add_argument("--ens-compare", type=int, default=6, help="ensemble: samples also timed one by one")
    ap.add_argument("--batch", type=int, default=1, help="film: films of the same mesh integrated together")
    ap.add_argument("--tensor-cores", type=int, default=0, help="batch: far field of the shared H-matrix on tcgen05")
    ap.add_argument("--compare-single", type=int, default=1, help="batch: also time the film alone")
    ap.add_argument("--batched", type=int, default=8,
                    help="film (N=1): also time this many films of the mesh integrated together (0: off)")
    ap.add_argument("--batched-steps", type=int, default=10)
    ap.add_argument("--workload", default="film", choices=["film", "adjoint", "ensemble"],
                    help="film: LLG steps/s on the 0.48M-node film (the headline); adjoint: trajectory gradient "
                         "on the 100x100x2 film")
    ap.add_argument("--adj-steps", type=int, default=400)
    ap.add_argument("--fd-dirs", type=int, default=32)
    ap.add_argument("--tangent-dirs", type=int, default=4)
    a = ap.parse_args()
    if a.warmup < 0 or a.steps < 1:
        ap.error("steps >= 1 and warmup >= 0")
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "adjoint":
        run_adjoint(a)
    elif a.workload == "ensemble":
        run_ensemble(a)
    elif a.batch > 1:
        run_film_batch(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
