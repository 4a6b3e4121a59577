"""H-matrix of the Lindholm double-layer operator on the GPU.

Mirrors the reference package ``gpu/fields/lindholm_hmatrix_gpu``:

* ``HMatrixBuildConfig``      builder.py:24-95 (same fields, same validation)
* ``build_or_load_hmatrix``   builder.py:814-927 (GPU construction; npz cache in the
  reference's ``HMatrixCPUData.save/load`` schema, storage.py:72-209, with the same
  geometry-hash / build-config / provider-signature validation)
* ``HMatrixGPUPackedFused``   backend_fused.py:341-646 (``matvec``, ``matvec_numpy``,
  ``benchmark``, ``benchmark_roundtrip``, ``memory_report``)

Construction (tree, partition, fill, full-pivot ACA) and the apply run in
libspx; see csrc/hbuild.cu and csrc/hmat.cu.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import asdict, dataclass
from hashlib import sha256
from pathlib import Path
from time import perf_counter

import numpy as np

from . import _lib
from ._lib import call, ptr
from .geometry import BoundaryGeometry, boundary_data

HMATRIX_CONSTRUCTION_VERSION = "lindholm-hmatrix-build-v2-b200"
# cache signature of the device entry provider (the reference's providers report theirs,
# entry_provider.py:177-185, entry_provider_gpu.py:473-486)
PROVIDER_SIGNATURE = {"provider": "LindholmEntryProviderB200", "kernel_version": "lindholm-tiles-sm100a-v1",
                      "incident_policy": 0}
FAR_META_DTYPE = np.dtype([("row_start", np.int64), ("row_stop", np.int64), ("col_start", np.int64),
                           ("col_stop", np.int64), ("rank", np.int64), ("u_offset", np.int64), ("u_size", np.int64),
                           ("v_offset", np.int64), ("v_size", np.int64), ("relative_residual", np.float64)])


def geometry_hash(Xb, tri_lid=None) -> str:
    """sha256 of the boundary points (and triangles), as builder.py:98-103."""
    digest = sha256()
    digest.update(np.ascontiguousarray(Xb, dtype=np.float64).view(np.uint8))
    if tri_lid is not None:
        digest.update(np.ascontiguousarray(tri_lid, dtype=np.int32).view(np.uint8))
    return digest.hexdigest()

STAT_NAMES = ("dense_blocks", "low_rank_blocks", "rejected_low_rank_blocks", "forced_subdivisions_memory",
              "compression_tolerance_subdivisions", "max_observed_rank", "sum_observed_rank",
              "block_entry_evaluations", "near_entries", "far_entries", "n_far", "n_near", "aca_steps", "waves")


@dataclass
class HMatrixBuildConfig:
    """The reference's build configuration (builder.py:24-95): same fields, defaults and
    validation messages, except that this library builds on the GPU only.

    * ``build_backend``: "gpu" (the default here) and "auto" build on the current CUDA device;
      "cpu" (the reference's default, its numba builder) is refused with ValueError.
    * ``gpu_device_id`` must name the current CUDA device: the H-matrix is built and applied
      where the caller's tensors live.
    * ``gpu_memory_fraction`` bounds the build's device workspace to that fraction of the
      free device memory (at most 6 GiB); ``batch_bytes`` > 0 sets it directly.
    * ``gpu_fallback_to_cpu``: there is no CPU builder to fall back to.  On an allocation
      failure the build retries with half the workspace (down to 64 MiB) and raises
      MemoryError only when that fails too.
    * the randomized-SVD and progress fields are accepted and validated; the compressor is
      full-pivot ACA.
    * ``recompress`` (this library's): SVD-recompress the ACA factors after the build to the
      smallest ranks that keep every block within epsilon; required by the 'f32_f16' packing.
    """
    epsilon: float = 1e-6
    eta: float = 2.0
    leaf_size: int = 64
    compressor: str = "fullaca"
    max_rank: int | None = None
    max_temporary_block_bytes: int = 256 * 1024 * 1024
    low_rank_storage_factor: float = 0.95
    build_backend: str = "gpu"
    gpu_device_id: int | None = None
    gpu_memory_fraction: float = 0.75
    gpu_fallback_to_cpu: bool = True
    gpu_aca_residual_check_interval: int = 1
    gpu_rsvd_initial_rank: int = 16
    gpu_rsvd_oversampling: int = 8
    gpu_rsvd_power_iterations: int = 1
    gpu_progress_interval_seconds: float = 5.0
    batch_bytes: int = 0
    recompress: bool = False

    def __post_init__(self):
        if self.epsilon <= 0.0:
            raise ValueError("epsilon must be positive.")
        if self.eta <= 0.0:
            raise ValueError("eta must be positive.")
        if self.leaf_size < 1:
            raise ValueError("leaf_size must be positive.")
        if self.max_temporary_block_bytes < 8:
            raise ValueError("max_temporary_block_bytes is too small.")
        if not (0.0 < self.low_rank_storage_factor <= 1.0):
            raise ValueError("low_rank_storage_factor must be in (0, 1].")
        if self.low_rank_storage_factor != 0.95:
            raise ValueError("only low_rank_storage_factor=0.95 (the reference default) is supported")
        c = str(self.compressor).strip().lower()
        if c == "aca":
            c = "fullaca"
        if c != "fullaca":
            raise ValueError("the GPU builder implements the 'fullaca' compressor")
        self.compressor = c
        b = str(self.build_backend).strip().lower()
        if b not in {"gpu", "auto", "cpu"}:
            raise ValueError("build_backend must be 'cpu', 'gpu', or 'auto'.")
        if b == "cpu":
            raise ValueError("build_backend='cpu' (the reference's numba builder) is not part of this library; "
                             "use 'gpu' or 'auto'")
        self.build_backend = b
        if self.gpu_device_id is not None:
            self.gpu_device_id = int(self.gpu_device_id)
            if self.gpu_device_id < 0:
                raise ValueError("gpu_device_id must be non-negative.")
        if not (0.0 < float(self.gpu_memory_fraction) <= 1.0):
            raise ValueError("gpu_memory_fraction must be in (0, 1].")
        if self.gpu_aca_residual_check_interval < 1:
            raise ValueError("gpu_aca_residual_check_interval must be positive.")
        if self.gpu_rsvd_initial_rank < 1:
            raise ValueError("gpu_rsvd_initial_rank must be positive.")
        if self.gpu_rsvd_oversampling < 0:
            raise ValueError("gpu_rsvd_oversampling must be non-negative.")
        if self.gpu_rsvd_power_iterations < 0:
            raise ValueError("gpu_rsvd_power_iterations must be non-negative.")
        if self.gpu_progress_interval_seconds < 0.0:
            raise ValueError("gpu_progress_interval_seconds must be non-negative.")

    def workspace_bytes(self):
        """Device workspace of one fill/ACA batch: batch_bytes if set, else gpu_memory_fraction
        of the free device memory, at most 6 GiB."""
        if self.batch_bytes > 0:
            return int(self.batch_bytes)
        try:
            import torch
            free = torch.cuda.mem_get_info()[0] if torch.cuda.is_available() else 0
        except Exception:
            free = 0
        cap = 6 * 1024 ** 3
        return int(min(cap, self.gpu_memory_fraction * free)) if free else 0

    def check_device(self):
        if self.gpu_device_id is None:
            return
        import torch
        cur = torch.cuda.current_device()
        if self.gpu_device_id != cur:
            raise ValueError(f"gpu_device_id={self.gpu_device_id} differs from the current CUDA device {cur}; "
                             "the H-matrix is built and applied on the current device")

    def to_c(self, precision="f64", batch_bytes=None):
        bb = self.batch_bytes if batch_bytes is None else batch_bytes
        return _lib.HmatConfig(epsilon=self.epsilon, eta=self.eta, leaf_size=int(self.leaf_size),
                               max_rank=int(self.max_rank or 0),
                               max_temporary_block_bytes=int(self.max_temporary_block_bytes),
                               precision=_lib.PREC[precision],
                               flags=1 if (self.recompress or precision == "f32_f16") else 0, batch_bytes=int(bb))


MIN_WORKSPACE = 64 * 1024 ** 2


def build_with_retry(geometry, cfg, precision):
    """spx_hmat_build with the workspace of cfg; on an allocation failure the build is
    repeated with half the workspace, down to 64 MiB (the reference instead subdivides the
    block or falls back to its CPU builder, builder.py:597-662, 880-901)."""
    ws = cfg.workspace_bytes()
    while True:
        h = C.c_void_p()
        c = cfg.to_c(precision, batch_bytes=ws)
        try:
            call("spx_hmat_build", geometry.handle, C.byref(c), C.byref(h))
            return h
        except MemoryError:
            cur = ws if ws > 0 else 6 * 1024 ** 3
            if cur // 2 < MIN_WORKSPACE:
                raise
            ws = cur // 2


def _precision_name(use_fp32=True, precision=None):
    if precision is not None:
        if precision not in _lib.PREC:
            raise ValueError(f"unknown precision {precision!r}")
        return precision
    return "f32" if use_fp32 else "f64"


class HMatrixGPUPackedFused:
    """Packed GPU H-matrix (y = H x in the original boundary ordering).

    ``HMatrixGPUPackedFused(geometry, config, use_fp32=True, precision=None)`` builds
    the matrix on the device; ``from_handle`` wraps one owned by a demag object.
    ``use_fp32`` stores factors and near tiles in FP32 (``precision='f64'`` keeps
    everything in FP64, ``'mixed'`` uses BF16 far factors and FP32 near tiles).
    """

    backend_name = "packed_fused_b200"

    def __init__(self, geometry: BoundaryGeometry | None = None, config: HMatrixBuildConfig | None = None,
                 threads_per_block=128, use_fp32=True, precision=None, _handle=None, _owner=None, _size=None):
        if threads_per_block < 32 or threads_per_block > 1024:
            raise ValueError("threads_per_block must be between 32 and 1024.")
        self.precision = _precision_name(use_fp32, precision)
        self._owner = _owner
        self.metadata = {}
        if _handle is not None:
            self._h = _handle
            self._owned = False
        else:
            if geometry is None:
                raise ValueError("a BoundaryGeometry is required")
            self._geometry = geometry
            cfg = config or HMatrixBuildConfig()
            cfg.check_device()
            self._h = build_with_retry(geometry, cfg, self.precision)
            self._owned = True
        n = _lib.c_i64()
        call("spx_hmat_num_blocks", self._h, C.byref(n))
        self._nblocks = n.value
        st = self.stats()
        self.size = int(_size if _size is not None else geometry.Nb)
        self.n_far_blocks = st["n_far"]
        self.max_rank = st["max_observed_rank"]

    @classmethod
    def from_handle(cls, handle, owner, precision, size):
        return cls(_handle=handle, _owner=owner, precision=precision, _size=size)

    @property
    def handle(self):
        return self._h

    # --------------------------------------------------------------- info
    def stats(self):
        v = np.zeros(16, np.int64)
        secs = _lib.c_dbl()
        call("spx_hmat_stats", self._h, ptr(v), C.byref(secs))
        d = {k: int(v[i]) for i, k in enumerate(STAT_NAMES)}
        d["build_time_seconds"] = float(secs.value)
        d["average_far_rank"] = d["sum_observed_rank"] / max(d["low_rank_blocks"], 1)
        return d

    def blocks(self):
        out = np.zeros((self._nblocks, 6), np.int64)
        call("spx_hmat_blocks", self._h, ptr(out), self._nblocks)
        return out

    def partition(self):
        b = self.blocks()
        return sorted(tuple(int(v) for v in r[:5]) for r in b)

    def far_factors(self, index):
        b = self.blocks()[index]
        m, n, k = int(b[1] - b[0]), int(b[3] - b[2]), int(b[5])
        Ut = np.empty((k, m))
        V = np.empty((k, n))
        call("spx_hmat_far_factors", self._h, int(index), ptr(Ut), ptr(V))
        return Ut.T.copy(), V

    @property
    def perm(self):
        p = np.empty(self.size, np.int32)
        call("spx_hmat_perm", self._h, ptr(p))
        return p

    def enable_tensor_cores(self, enable=True):
        """Run the far field of matmat on the tensor cores for batches of 8 states (builds the
        packed factors once); enable="auto" times the CUDA-core path and two tensor-core tile
        lengths and keeps the fastest.  Returns the plan's device bytes (0: CUDA cores)."""
        b = _lib.c_i64()
        mode = 2 if enable == "auto" else (1 if enable else 0)
        call("spx_hmat_tensor_cores", self._h, mode, C.byref(b))
        return b.value

    def tensor_core_status(self):
        """0, or the timeout code of a tensor-core kernel since the last call."""
        st = _lib.c_i32()
        call("spx_hmat_tc_status", self._h, C.byref(st))
        return st.value

    def recompress(self):
        """SVD recompression of the far factors (same tolerance); returns entries before /
        after, blocks rewritten and the largest block truncation error (relative)."""
        out = np.zeros(3, np.int64)
        e = _lib.c_dbl()
        call("spx_hmat_recompress", self._h, ptr(out), C.byref(e))
        return {"entries_before": int(out[0]), "entries_after": int(out[1]), "rewritten": int(out[2]),
                "max_rel_truncation": e.value}

    def repack(self, precision):
        call("spx_hmat_repack", self._h, _lib.PREC[precision])
        self.precision = precision

    # --------------------------------------------------------------- apply
    def matvec(self, x_gpu, out=None):
        import torch
        if x_gpu.dtype != torch.float64 or not x_gpu.is_cuda:
            raise TypeError("matvec expects a CUDA float64 tensor")
        x = x_gpu.contiguous()
        if out is None:
            out = torch.empty_like(x)
        call("spx_hmat_apply", self._h, ptr(x), ptr(out), _lib.stream_ptr())
        return out

    def matmat(self, X_gpu, out=None):
        """Y = H X for a CUDA float64 tensor of shape (R, Nb) (R vectors, one per row) in one pass."""
        import torch
        if X_gpu.dtype != torch.float64 or not X_gpu.is_cuda or X_gpu.dim() != 2 or X_gpu.shape[1] != self.size:
            raise TypeError("matmat expects a CUDA float64 tensor of shape (R, Nb)")
        X = X_gpu.contiguous()
        if out is None:
            out = torch.empty_like(X)
        call("spx_hmat_apply_multi", self._h, ptr(X), ptr(out), int(X.shape[0]), _lib.stream_ptr())
        return out

    def rmatvec(self, x_gpu, out=None):
        """y = H^T x (transposed apply; the transposed H-matrix is packed on the first call)."""
        import torch
        if x_gpu.dtype != torch.float64 or not x_gpu.is_cuda:
            raise TypeError("rmatvec expects a CUDA float64 tensor")
        x = x_gpu.contiguous()
        if out is None:
            out = torch.empty_like(x)
        call("spx_hmat_apply_transpose", self._h, ptr(x), ptr(out), _lib.stream_ptr())
        return out

    def matvec_noalloc(self, x_gpu, out):
        """y = H x through spx_hmat_apply_noalloc: no device allocation inside the call
        (the scratch is the library's fixed 32 MiB device array, shared by every call, so
        calls must not overlap on the GPU).  ``out`` must be a preallocated CUDA float64
        tensor of length Nb."""
        import torch
        if x_gpu.dtype != torch.float64 or not x_gpu.is_cuda or not x_gpu.is_contiguous():
            raise TypeError("matvec_noalloc expects a contiguous CUDA float64 tensor")
        if out.dtype != torch.float64 or not out.is_cuda or not out.is_contiguous() or out.numel() != self.size:
            raise TypeError("out must be a contiguous CUDA float64 tensor of length Nb")
        call("spx_hmat_apply_noalloc", self._h, ptr(x_gpu), ptr(out), _lib.stream_ptr())
        return out

    def matvec_numpy(self, x):
        import torch
        xt = torch.as_tensor(np.asarray(x, dtype=np.float64), device="cuda")
        return self.matvec(xt).cpu().numpy()

    def benchmark(self, x, repeats=20, warmup=3):
        import torch
        xt = torch.as_tensor(np.asarray(x, dtype=np.float64), device="cuda")
        out = torch.empty_like(xt)
        for _ in range(warmup):
            self.matvec(xt, out=out)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(repeats):
            self.matvec(xt, out=out)
        e.record()
        e.synchronize()
        sec = s.elapsed_time(e) * 1e-3
        return {"timer": "cuda_events", "repeats": int(repeats), "total_seconds": sec,
                "average_seconds": sec / repeats}

    def benchmark_roundtrip(self, x, repeats=20, warmup=3):
        import torch
        for _ in range(warmup):
            self.matvec_numpy(x)
        torch.cuda.synchronize()
        t0 = perf_counter()
        for _ in range(repeats):
            self.matvec_numpy(x)
        torch.cuda.synchronize()
        el = perf_counter() - t0
        return {"timer": "perf_counter_roundtrip", "repeats": int(repeats), "total_seconds": el,
                "average_seconds": el / repeats}

    # --------------------------------------------------------------- cache
    def cache_arrays(self):
        """The reference's HMatrixCPUData arrays (storage.py:72-149) of this H-matrix."""
        nf, nu, nv, nz = (_lib.c_i64() for _ in range(4))
        call("spx_hmat_export_sizes", self._h, C.byref(nf), C.byref(nu), C.byref(nv), C.byref(nz))
        nf, nu, nv, nz = nf.value, nu.value, nv.value, nz.value
        perm = np.empty(self.size, np.int32)
        diag = np.empty(self.size)
        meta5 = np.empty((nf, 5), np.int64)
        relres = np.empty(nf)
        U = np.empty(nu)
        V = np.empty(nv)
        indptr = np.empty(self.size + 1, np.int32)
        indices = np.empty(nz, np.int32)
        data = np.empty(nz)
        call("spx_hmat_export", self._h, ptr(perm), ptr(diag), ptr(meta5), ptr(relres), ptr(U), ptr(V), ptr(indptr),
             ptr(indices), ptr(data))
        m = meta5[:, 1] - meta5[:, 0]
        n = meta5[:, 3] - meta5[:, 2]
        k = meta5[:, 4]
        far_meta = np.zeros(nf, FAR_META_DTYPE)
        for i, name in enumerate(("row_start", "row_stop", "col_start", "col_stop", "rank")):
            far_meta[name] = meta5[:, i]
        far_meta["u_size"] = m * k
        far_meta["v_size"] = k * n
        far_meta["u_offset"] = np.concatenate([[0], np.cumsum(m * k)[:-1]]) if nf else []
        far_meta["v_offset"] = np.concatenate([[0], np.cumsum(k * n)[:-1]]) if nf else []
        far_meta["relative_residual"] = relres
        return dict(perm=perm, diag_jump=diag, near_data=data, near_indices=indices, near_indptr=indptr,
                    near_shape=np.array([self.size, self.size], np.int64), far_meta=far_meta, far_U_flat=U,
                    far_V_flat=V)

    def save(self, path, *, compressed=True, metadata=None):
        """Write the reference's npz cache (HMatrixCPUData.save, storage.py:72-149)."""
        path = Path(path)
        path.parent.mkdir(parents=True, exist_ok=True)
        arrays = self.cache_arrays()
        arrays["metadata_json"] = np.asarray(json.dumps(metadata or {}))
        with path.open("wb") as f:
            (np.savez_compressed if compressed else np.savez)(f, **arrays)

    @classmethod
    def load(cls, path, geometry: BoundaryGeometry, config: HMatrixBuildConfig | None = None, precision="f32"):
        """Read an npz cache in the reference's schema (HMatrixCPUData.load, storage.py:151-209)
        onto the device.  The cluster tree is rebuilt from ``geometry`` and must reproduce the
        cached permutation.  Returns (H, metadata)."""
        a = np.load(Path(path), allow_pickle=False)
        perm = np.ascontiguousarray(a["perm"], dtype=np.int32)
        if perm.size != geometry.Nb:
            raise ValueError(f"cache has {perm.size} boundary nodes, the geometry {geometry.Nb}")
        fm = a["far_meta"]
        meta5 = np.ascontiguousarray(np.stack([fm[k] for k in ("row_start", "row_stop", "col_start", "col_stop",
                                                               "rank")], 1).astype(np.int64)).reshape(-1, 5)
        U_all = np.asarray(a["far_U_flat"], dtype=np.float64)
        V_all = np.asarray(a["far_V_flat"], dtype=np.float64)
        # factors in block order, contiguous (the offsets of the file may have any order)
        if fm.size:
            U = np.concatenate([U_all[o:o + z] for o, z in zip(fm["u_offset"], fm["u_size"])])
            V = np.concatenate([V_all[o:o + z] for o, z in zip(fm["v_offset"], fm["v_size"])])
        else:
            U = V = np.empty(0)
        relres = np.ascontiguousarray(fm["relative_residual"], dtype=np.float64) if fm.size else np.empty(0)
        indptr = np.ascontiguousarray(a["near_indptr"], dtype=np.int32)
        indices = np.ascontiguousarray(a["near_indices"], dtype=np.int32)
        data = np.ascontiguousarray(a["near_data"], dtype=np.float64)
        diag = np.ascontiguousarray(a["diag_jump"], dtype=np.float64)
        raw = str(np.asarray(a["metadata_json"]).item())
        metadata = json.loads(raw) if raw else {}
        cfg = config or HMatrixBuildConfig(leaf_size=int(metadata.get("build_config", {}).get("leaf_size", 64)))
        c = cfg.to_c(precision)
        h = C.c_void_p()
        call("spx_hmat_import", geometry.handle, C.byref(c), ptr(perm), ptr(diag), meta5.shape[0], ptr(meta5),
             ptr(relres), ptr(U), ptr(V), ptr(indptr), ptr(indices), ptr(data), C.byref(h))
        H = cls(_handle=h, _owner=None, precision=precision, _size=geometry.Nb)
        H._owned = True
        H._geometry = geometry
        return H, metadata

    def memory_report(self):
        f, n, t = _lib.c_i64(), _lib.c_i64(), _lib.c_i64()
        call("spx_hmat_memory", self._h, C.byref(f), C.byref(n), C.byref(t))
        st = self.stats()
        return {"backend": self.backend_name, "n_far_blocks": st["n_far"], "max_rank": st["max_observed_rank"],
                "precision": self.precision, "far_bytes": f.value, "near_bytes": n.value,
                "accounted_gpu_bytes": t.value, "accounted_gpu_human": f"{t.value / 2**20:.3f} MiB"}

    def print_memory_report(self, prefix="[HMatrixGPUPackedFused]"):
        for k, v in self.memory_report().items():
            print(f"{prefix} {k:28s}: {v}", flush=True)

    def __del__(self):
        try:
            h = getattr(self, "_h", None)
            if getattr(self, "_owned", False) and h is not None and h.value:
                try:
                    _lib.lib().spx_hmat_destroy(h)
                except Exception:
                    pass
                self._h = C.c_void_p()
        except Exception:
            pass


def _cache_build_config(config: HMatrixBuildConfig) -> dict:
    value = asdict(config)
    value["resolved_build_backend"] = "gpu"
    value["construction_version"] = HMATRIX_CONSTRUCTION_VERSION
    return json.loads(json.dumps(value, sort_keys=True))


def build_or_load_hmatrix(cache_path, X, tets, config: HMatrixBuildConfig | None = None, *,
                          precision="f32", force_rebuild=False, verbose=False, geometry=None, cache_compressed=True):
    """Build the H-matrix of the mesh boundary on the GPU, or load it from an npz cache
    (builder.py:814-927).  A cache is used when its metadata carries the same geometry hash
    (boundary points and triangles), build configuration and provider signature; else the
    matrix is built and the cache (re)written.  ``cache_path=None`` builds without a file.
    The returned object carries ``metadata`` (cache_loaded, cache_file_bytes, ...)."""
    geom = geometry or BoundaryGeometry(X, tets)
    cfg = config or HMatrixBuildConfig()
    bd = boundary_data(X, tets)
    expected = {"geometry_hash": geometry_hash(bd["Xb"], bd["tri_lid"]), "build_config": _cache_build_config(cfg),
                "provider_signature": dict(PROVIDER_SIGNATURE)}
    path = Path(cache_path) if cache_path is not None else None
    if path is not None and path.exists() and not force_rebuild:
        try:
            H, meta = HMatrixGPUPackedFused.load(path, geom, cfg, precision=precision)
        except (ValueError, KeyError, RuntimeError, OSError) as exc:
            H, meta = None, {"load_error": str(exc)}
        if H is not None and all(meta.get(k) == v for k, v in expected.items()):
            meta["cache_loaded"] = True
            meta["cache_file_bytes"] = int(path.stat().st_size)
            H.metadata = meta
            if verbose:
                print(f"[HMatrix b200] loaded cache: {path}", flush=True)
            return H
        if verbose:
            print("[HMatrix b200] cache metadata changed; rebuilding.", flush=True)
        del H
    H = HMatrixGPUPackedFused(geom, cfg, precision=precision)
    st = H.stats()
    meta = {"Nb": geom.Nb, **expected, "build_time_seconds": st["build_time_seconds"],
            "average_far_rank": st["average_far_rank"], "resolved_build_backend": "gpu",
            "construction_version": HMATRIX_CONSTRUCTION_VERSION,
            **{k: st[k] for k in STAT_NAMES}, "cache_compressed": bool(cache_compressed), "cache_loaded": False}
    if path is not None:
        t0 = perf_counter()
        H.save(path, compressed=cache_compressed, metadata=meta)
        meta["cache_write_seconds"] = perf_counter() - t0
        meta["cache_file_bytes"] = int(path.stat().st_size)
    H.metadata = meta
    if verbose:
        print(f"[HMatrix b200] built in {st['build_time_seconds']:.2f} s | far={st['n_far']} near={st['n_near']} "
              f"| rank avg/max={st['average_far_rank']:.1f}/{st['max_observed_rank']}", flush=True)
    return H
