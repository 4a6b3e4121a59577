"""Cluster tree, block partition, full-pivot ACA and H-matrix matvec (oracle).

Restates:

* ``build_cluster_tree``  gpu/fields/lindholm_hmatrix_gpu/tree.py:41-96
  (median split on the longest bbox axis, stable mergesort, mid = size//2)
* ``bbox_distance``, ``admissible``  tree.py:99-115
* ``fullaca_dense``  compressors.py:35-99 (argmax |R|, first index on ties)
* ``HMatrixBuilder._build_block`` / ``_subdivide`` / ``build``
  builder.py:229-419 (accept rule :322-370, forced memory split :338-341,
  larger-diameter node subdivided first :260-275)
* ``HMatrixStorageBuilder.finalize`` and ``HMatrixCPUData.matvec_cpu``
  storage.py:175-190, :333-390
* ``PackedCPU``: the same matvec (x~ = x[perm]; diag jump + near CSR + sum_b U_b (V_b x~))
  over the arrays of the reference's npz cache schema (``HMatrixCPUData.save``,
  storage.py:77-149), row- and block-parallel on all host threads (numba); per-thread
  partial sums of the far field are added at the end.  Used as the timed CPU baseline.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from . import lindholm


@dataclass
class Node:
    start: int
    stop: int
    bmin: np.ndarray
    bmax: np.ndarray
    left: "Node | None" = None
    right: "Node | None" = None

    @property
    def size(self):
        return self.stop - self.start

    @property
    def is_leaf(self):
        return self.left is None and self.right is None

    @property
    def diameter(self):
        return float(np.linalg.norm(self.bmax - self.bmin))


def cluster_tree(points, leaf_size=64):
    points = np.ascontiguousarray(points, dtype=np.float64)
    order = []

    def rec(idx):
        lp = points[idx]
        bmin, bmax = lp.min(axis=0), lp.max(axis=0)
        if idx.size <= leaf_size:
            s = len(order)
            order.extend(idx.tolist())
            return Node(s, len(order), bmin, bmax)
        axis = int(np.argmax(bmax - bmin))
        srt = idx[np.argsort(lp[:, axis], kind="mergesort")]
        mid = srt.size // 2
        if mid == 0 or mid == srt.size:
            mid = max(1, srt.size // 2)
        L = rec(srt[:mid])
        R = rec(srt[mid:])
        return Node(L.start, R.stop, bmin, bmax, L, R)

    root = rec(np.arange(points.shape[0], dtype=np.int32))
    return np.asarray(order, dtype=np.int32), root


def bbox_distance(a, b):
    gap = np.maximum(np.maximum(a.bmin - b.bmax, b.bmin - a.bmax), 0.0)
    return float(np.linalg.norm(gap))


def admissible(a, b, eta):
    d = bbox_distance(a, b)
    if d <= 0.0:
        return False
    return max(a.diameter, b.diameter) <= float(eta) * d


def fullaca(A, rtol, max_rank=None):
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    kmax = min(m, n) if max_rank is None else min(max(int(max_rank), 0), m, n)
    normA = float(np.linalg.norm(A))
    if normA == 0.0 or kmax == 0:
        return np.zeros((m, 0)), np.zeros((0, n)), 0.0
    R = A.copy()
    U, V = [], []
    rel = 1.0
    eps = np.finfo(np.float64).eps
    for _ in range(kmax):
        p = int(np.argmax(np.abs(R)))
        i, j = divmod(p, n)
        piv = R[i, j]
        if abs(piv) <= eps * normA:
            break
        u = R[:, j].copy()
        v = R[i, :].copy() / piv
        U.append(u)
        V.append(v)
        R -= np.outer(u, v)
        rel = float(np.linalg.norm(R) / normA)
        if rel <= rtol:
            break
    if not U:
        return np.zeros((m, 0)), np.zeros((0, n)), rel
    return np.column_stack(U), np.vstack(V), rel


@dataclass
class HOracle:
    perm: np.ndarray
    diag_jump: np.ndarray
    near: sp.csr_matrix
    far: list = field(default_factory=list)       # (rs, re, cs, ce, U, V, rel)
    dense_blocks: list = field(default_factory=list)  # (rs, re, cs, ce)
    stats: dict = field(default_factory=dict)

    def matvec(self, x):
        xp = x[self.perm]
        yp = self.diag_jump[self.perm] * xp + self.near @ xp
        for rs, re, cs, ce, U, V, _ in self.far:
            yp[rs:re] += U @ (V @ xp[cs:ce])
        y = np.empty_like(x)
        y[self.perm] = yp
        return y

    def partition(self):
        """Sorted list of (rs, re, cs, ce, is_far) describing the block partition."""
        out = [(b[0], b[1], b[2], b[3], 1) for b in self.far]
        out += [(b[0], b[1], b[2], b[3], 0) for b in self.dense_blocks]
        return sorted(out)


def build(bd, epsilon=1e-5, eta=2.0, leaf_size=64, max_rank=None,
          max_temporary_block_bytes=256 * 1024 ** 2, low_rank_storage_factor=0.95):
    Xb = bd["Xb"]
    Nb = Xb.shape[0]
    perm, root = cluster_tree(Xb, leaf_size)
    margin = 1.0 + 64.0 * np.finfo(np.float64).eps
    rows_l, cols_l, data_l = [], [], []
    far, dense = [], []
    stats = dict(dense_blocks=0, low_rank_blocks=0, rejected_low_rank_blocks=0,
                 forced_subdivisions_memory=0, compression_tolerance_subdivisions=0,
                 max_observed_rank=0, sum_observed_rank=0)

    def fill(r, c):
        return lindholm.fill_block(bd, perm[r.start:r.stop], perm[c.start:c.stop])

    def add_dense(r, c, A=None):
        if A is None:
            A = fill(r, c)
        lr, lc = np.nonzero(A)
        rows_l.append(lr + r.start)
        cols_l.append(lc + c.start)
        data_l.append(A[lr, lc])
        dense.append((r.start, r.stop, c.start, c.stop))
        stats["dense_blocks"] += 1

    def subdivide(r, c):
        rs, cs = not r.is_leaf, not c.is_leaf
        if not rs and not cs:
            add_dense(r, c)
            return
        if rs and (not cs or r.diameter >= c.diameter):
            block(r.left, c)
            block(r.right, c)
        else:
            block(r, c.left)
            block(r, c.right)

    def block(r, c):
        dense_bytes = r.size * c.size * 8
        adm = admissible(r, c, eta)
        if adm and dense_bytes > max_temporary_block_bytes:
            stats["forced_subdivisions_memory"] += 1
            subdivide(r, c)
            return
        if adm:
            A = fill(r, c)
            U, V, rel = fullaca(A, epsilon, max_rank)
            k = U.shape[1]
            ok = np.isfinite(rel) and rel <= epsilon * margin
            if k > 0 and ok and (U.size + V.size) < low_rank_storage_factor * A.size:
                far.append((r.start, r.stop, c.start, c.stop, U, V, rel))
                stats["low_rank_blocks"] += 1
                stats["max_observed_rank"] = max(stats["max_observed_rank"], k)
                stats["sum_observed_rank"] += k
                return
            if not ok and (not r.is_leaf or not c.is_leaf):
                stats["compression_tolerance_subdivisions"] += 1
                subdivide(r, c)
                return
            add_dense(r, c, A)
            stats["rejected_low_rank_blocks"] += 1
            return
        if r.is_leaf and c.is_leaf:
            add_dense(r, c)
            return
        subdivide(r, c)

    block(root, root)
    if rows_l:
        near = sp.coo_matrix((np.concatenate(data_l), (np.concatenate(rows_l), np.concatenate(cols_l))),
                             shape=(Nb, Nb)).tocsr()
        near.sum_duplicates()
    else:
        near = sp.csr_matrix((Nb, Nb))
    return HOracle(perm=perm, diag_jump=lindholm.diag_jump(bd), near=near, far=far,
                   dense_blocks=dense, stats=stats)


def _packed_kernels():
    from numba import njit, prange

    @njit(parallel=True, cache=False)
    def near_part(indptr, indices, data, diag, xp, y):
        for i in prange(indptr.size - 1):
            acc = diag[i] * xp[i]
            for k in range(indptr[i], indptr[i + 1]):
                acc += data[k] * xp[indices[k]]
            y[i] = acc

    @njit(parallel=True, cache=False)
    def far_part(meta, U, V, xp, ybuf, chunk_start):
        nth = ybuf.shape[0]
        for t in prange(nth):
            zt = np.empty(256)
            for b in range(chunk_start[t], chunk_start[t + 1]):
                rs, re, cs, ce, k = meta[b, 0], meta[b, 1], meta[b, 2], meta[b, 3], meta[b, 4]
                uo, vo = meta[b, 5], meta[b, 6]
                n = ce - cs
                if k > zt.size:
                    zt = np.empty(k)
                for q in range(k):                    # z = V x~[cs:ce], V is k x n row-major
                    acc = 0.0
                    base = vo + q * n
                    for c in range(n):
                        acc += V[base + c] * xp[cs + c]
                    zt[q] = acc
                for r in range(re - rs):              # y += U z, U is m x k row-major
                    acc = 0.0
                    base = uo + r * k
                    for q in range(k):
                        acc += U[base + q] * zt[q]
                    ybuf[t, rs + r] += acc

    return near_part, far_part


class PackedCPU:
    """H-matrix apply over the reference's cache arrays on all host threads (see header)."""

    def __init__(self, arrays, threads=None):
        import os
        import numba
        self.perm = np.asarray(arrays["perm"], np.int64)
        self.diag = np.asarray(arrays["diag_jump"], np.float64)[self.perm]
        self.indptr = np.asarray(arrays["near_indptr"], np.int64)
        self.indices = np.asarray(arrays["near_indices"], np.int32)
        self.data = np.asarray(arrays["near_data"], np.float64)
        fm = arrays["far_meta"]
        self.meta = np.stack([fm["row_start"], fm["row_stop"], fm["col_start"], fm["col_stop"], fm["rank"],
                              fm["u_offset"], fm["v_offset"]], axis=1).astype(np.int64) if len(fm) else \
            np.zeros((0, 7), np.int64)
        self.U = np.asarray(arrays["far_U_flat"], np.float64)
        self.V = np.asarray(arrays["far_V_flat"], np.float64)
        self.threads = int(threads or numba.get_num_threads() or os.cpu_count() or 1)
        # blocks dealt to threads in contiguous runs of about equal factor entries
        w = (self.meta[:, 1] - self.meta[:, 0] + self.meta[:, 3] - self.meta[:, 2]) * self.meta[:, 4]
        cw = np.concatenate([[0], np.cumsum(w)])
        targets = cw[-1] * np.arange(self.threads + 1) / self.threads
        self.chunk = np.searchsorted(cw, targets).astype(np.int64)
        self.chunk[0], self.chunk[-1] = 0, self.meta.shape[0]
        self.near_k, self.far_k = _packed_kernels()
        self.ybuf = np.zeros((self.threads, self.perm.size))

    def matvec(self, x):
        x = np.asarray(x, dtype=np.float64)
        xp = x[self.perm]
        yp = np.empty_like(xp)
        self.near_k(self.indptr, self.indices, self.data, self.diag, xp, yp)
        self.ybuf[:] = 0.0
        self.far_k(self.meta, self.U, self.V, xp, self.ybuf, self.chunk)
        yp += self.ybuf.sum(axis=0)
        y = np.empty_like(x)
        y[self.perm] = yp
        return y
