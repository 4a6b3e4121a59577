"""Mesh input, boundary geometry and host-side set-up calls of libspx.

The reference takes its meshes from DOLFINx (``gpu/io_utils/mesh.py:6-30``) and
builds the boundary data in Python (``gpu/fields/Demag_Lindholm.py:177-285``).
Here a mesh is two arrays: ``X`` [N, 3] float64 coordinates in nm and ``tets``
[E, 4] int32 vertex ids (for a DOLFINx P1 space: the dof coordinates and the
cell->dof map).  ``kuhn_box`` builds the synthetic boxes used by the benchmarks.
"""
from __future__ import annotations

import ctypes as C
import itertools

import numpy as np

from . import _lib
from ._lib import call, ptr


def as_mesh(X, tets):
    X = np.ascontiguousarray(X, dtype=np.float64)
    tets = np.ascontiguousarray(tets, dtype=np.int32)
    if X.ndim != 2 or X.shape[1] != 3:
        raise ValueError("X must have shape (N, 3)")
    if tets.ndim != 2 or tets.shape[1] != 4:
        raise ValueError("tets must have shape (E, 4)")
    return X, tets


def kuhn_box(nx: int, ny: int, nz: int, h: float):
    """Box of nx*ny*nz cubes of side h (nm), 6 tets per cube around the 000->111 diagonal.

    Vertex (i, j, k) has index i + (nx+1)*(j + (ny+1)*k).
    """
    nx, ny, nz = int(nx), int(ny), int(nz)
    k, j, i = np.meshgrid(np.arange(nz + 1), np.arange(ny + 1), np.arange(nx + 1), indexing="ij")
    X = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) * float(h)
    ck, cj, ci = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()

    def vid(a, b, c):
        return a + (nx + 1) * (b + (ny + 1) * c)

    tets = np.empty((ci.size, 6, 4), dtype=np.int64)
    for p, (a, b, _) in enumerate(itertools.permutations(range(3))):
        o1 = np.zeros(3, dtype=np.int64)
        o1[a] = 1
        o2 = o1.copy()
        o2[b] = 1
        for q, o in enumerate((np.zeros(3, dtype=np.int64), o1, o2, np.ones(3, dtype=np.int64))):
            tets[:, p, q] = vid(ci + o[0], cj + o[1], ck + o[2])
    return X, tets.reshape(-1, 4).astype(np.int32)


def boundary_data(X, tets):
    """Host boundary data: dict(bverts, tri_lid, Xb, ntri, area, omega_sum)."""
    X, tets = as_mesh(X, tets)
    Nb, Nt = _lib.c_i64(), _lib.c_i64()
    call("spx_boundary_sizes", ptr(X), X.shape[0], ptr(tets), tets.shape[0], C.byref(Nb), C.byref(Nt))
    Nb, Nt = Nb.value, Nt.value
    out = dict(bverts=np.empty(Nb, np.int32), tri_lid=np.empty((Nt, 3), np.int32), Xb=np.empty((Nb, 3)),
               ntri=np.empty((Nt, 3)), area=np.empty(Nt), omega_sum=np.empty(Nb))
    call("spx_boundary_data", ptr(X), X.shape[0], ptr(tets), tets.shape[0], ptr(out["bverts"]),
         ptr(out["tri_lid"]), ptr(out["Xb"]), ptr(out["ntri"]), ptr(out["area"]), ptr(out["omega_sum"]))
    return out


def fem_assemble(X, tets):
    """Host P1 operators on the scalar pattern: dict(rowptr, col, A, Div, G, vol)."""
    X, tets = as_mesh(X, tets)
    nnz = _lib.c_i64()
    call("spx_fem_sizes", ptr(X), X.shape[0], ptr(tets), tets.shape[0], C.byref(nnz))
    N, nnz = X.shape[0], nnz.value
    out = dict(rowptr=np.empty(N + 1, np.int64), col=np.empty(nnz, np.int32), A=np.empty(nnz),
               Div=np.empty((nnz, 3)), G=np.empty((nnz, 3)), vol=np.empty(N))
    call("spx_fem_assemble", ptr(X), N, ptr(tets), tets.shape[0], ptr(out["rowptr"]), ptr(out["col"]),
         ptr(out["A"]), ptr(out["Div"]), ptr(out["G"]), ptr(out["vol"]))
    return out


def cluster_tree_perm(points, leaf_size=64):
    """Permutation of build_cluster_tree (lindholm_hmatrix_gpu/tree.py:41-96)."""
    pts = np.ascontiguousarray(points, dtype=np.float64)
    perm = np.empty(pts.shape[0], np.int32)
    call("spx_cluster_tree", ptr(pts), pts.shape[0], int(leaf_size), ptr(perm))
    return perm


class BoundaryGeometry:
    """Boundary geometry resident on the current CUDA device (opaque spx_boundary)."""

    def __init__(self, X, tets):
        X, tets = as_mesh(X, tets)
        self._h = C.c_void_p()
        call("spx_boundary_create", ptr(X), X.shape[0], ptr(tets), tets.shape[0], C.byref(self._h))
        Nb, Nt, mi = _lib.c_i64(), _lib.c_i64(), _lib.c_i32()
        call("spx_boundary_info", self._h, C.byref(Nb), C.byref(Nt), C.byref(mi))
        self.Nb, self.Nt, self.max_incident = Nb.value, Nt.value, mi.value

    @property
    def handle(self):
        return self._h

    def lindholm_pairs(self, x0, tri):
        """Weights [P, 3] of targets x0 [P, 3] (cuda float64) against triangles tri [P] (cuda int32)."""
        import torch
        w = torch.empty((x0.shape[0], 3), dtype=torch.float64, device=x0.device)
        call("spx_lindholm_pairs", self._h, ptr(x0.contiguous()), ptr(tri.contiguous()), x0.shape[0], ptr(w),
             _lib.stream_ptr())
        return w

    def fill_block(self, rows, cols):
        """B[rows, cols] without the diagonal jump (rows, cols: cuda int32)."""
        import torch
        out = torch.empty((rows.numel(), cols.numel()), dtype=torch.float64, device=rows.device)
        call("spx_lindholm_fill_block", self._h, ptr(rows.contiguous()), rows.numel(), ptr(cols.contiguous()),
             cols.numel(), ptr(out), _lib.stream_ptr())
        return out

    def dense_B(self, device="cuda"):
        import torch
        B = torch.empty((self.Nb, self.Nb), dtype=torch.float64, device=device)
        call("spx_dense_b_assemble", self._h, ptr(B), _lib.stream_ptr())
        return B

    def __del__(self):
        try:
            h = getattr(self, "_h", None)
            if h is not None and h.value:
                try:
                    _lib.lib().spx_boundary_destroy(h)
                except Exception:
                    pass
                self._h = C.c_void_p()
        except Exception:
            pass


def dense_b_apply(B, x, out=None):
    import torch
    if out is None:
        out = torch.empty_like(x)
    call("spx_dense_b_apply", ptr(B), B.shape[0], ptr(x), ptr(out), _lib.stream_ptr())
    return out
