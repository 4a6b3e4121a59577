"""Lindholm double-layer weights, boundary geometry and dense B (oracle).

Restates, in vectorised numpy FP64:

* ``solid_angle_with_atan2``   gpu/fields/Lindholm_kernel.py:30-48
* ``_P_log1p``                 gpu/fields/Lindholm_kernel.py:51-63
* ``lindholm_weights_precomp`` gpu/fields/Lindholm_kernel.py:66-125
  (opposite-edge convention at :118-123)
* ``build_boundary_data_serial`` gpu/fields/Demag_Lindholm.py:177-285
* ``assemble_B_rows_owned``    gpu/fields/Demag_Lindholm.py:51-116
  (diagonal Omega/4pi - 1, incident triangles skipped)

Boundary facet order.  DOLFINx numbers exterior facets itself
(``exterior_facet_indices``); that numbering is not reproducible without
DOLFINx, so the oracle and the product both use one canonical order: boundary
facets sorted lexicographically by their ascending vertex triple, each facet
starting from that ascending triple (DOLFINx's facet->vertex order) and then
oriented outward by the rule of Demag_Lindholm.py:205-217 (swap v1, v2 when
the normal points towards the adjacent cell centroid).
"""
from __future__ import annotations

import math

import numpy as np

TINY = 1e-300
_FACE_LOCAL = np.array([[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]], dtype=np.int64)


def solid_angle(x0, p0, p1, p2):
    """Signed solid angle of triangle (p0,p1,p2) seen from x0; arrays [...,3]."""
    r0 = p0 - x0
    r1 = p1 - x0
    r2 = p2 - x0
    n0 = np.sqrt(np.sum(r0 * r0, axis=-1)) + TINY
    n1 = np.sqrt(np.sum(r1 * r1, axis=-1)) + TINY
    n2 = np.sqrt(np.sum(r2 * r2, axis=-1)) + TINY
    det = (r0[..., 0] * (r1[..., 1] * r2[..., 2] - r1[..., 2] * r2[..., 1])
           - r0[..., 1] * (r1[..., 0] * r2[..., 2] - r1[..., 2] * r2[..., 0])
           + r0[..., 2] * (r1[..., 0] * r2[..., 1] - r1[..., 1] * r2[..., 0]))
    d01 = np.sum(r0 * r1, axis=-1)
    d12 = np.sum(r1 * r2, axis=-1)
    d20 = np.sum(r2 * r0, axis=-1)
    denom = n0 * n1 * n2 + d01 * n2 + d12 * n0 + d20 * n1
    return 2.0 * np.arctan2(det, denom)


def _p_log1p(ri, rj, s):
    denom = ri + rj - s
    denom = np.where(denom < TINY, TINY, denom)
    return np.log1p((2.0 * s) / denom)


def lindholm_weights(x0, p0, p1, p2, n_unit, area, s_edge, eta, gamma):
    """(w0, w1, w2) for targets x0 [P,3] and per-pair triangle data.

    Shapes: p* [P,3], n_unit [P,3], area [P], s_edge [P,3], eta [P,3,3],
    gamma [P,3,3].  Follows Lindholm_kernel.py:66-125 term by term.
    """
    rho0 = p0 - x0
    rho1 = p1 - x0
    rho2 = p2 - x0
    r0 = np.sqrt(np.sum(rho0 * rho0, axis=-1)) + TINY
    r1 = np.sqrt(np.sum(rho1 * rho1, axis=-1)) + TINY
    r2 = np.sqrt(np.sum(rho2 * rho2, axis=-1)) + TINY
    h = np.sum(n_unit * rho0, axis=-1)
    eta0 = np.sum(eta[:, 0] * rho0, axis=-1)
    eta1 = np.sum(eta[:, 1] * rho1, axis=-1)
    eta2 = np.sum(eta[:, 2] * rho2, axis=-1)
    s0, s1, s2 = s_edge[:, 0], s_edge[:, 1], s_edge[:, 2]
    P0 = _p_log1p(r0, r1, s0)
    P1 = _p_log1p(r1, r2, s1)
    P2 = _p_log1p(r2, r0, s2)
    omega = solid_angle(x0, p0, p1, p2)
    gP0 = gamma[:, 0, 0] * P0 + gamma[:, 0, 1] * P1 + gamma[:, 0, 2] * P2
    gP1 = gamma[:, 1, 0] * P0 + gamma[:, 1, 1] * P1 + gamma[:, 1, 2] * P2
    gP2 = gamma[:, 2, 0] * P0 + gamma[:, 2, 1] * P1 + gamma[:, 2, 2] * P2
    c = 1.0 / (8.0 * math.pi * (area + TINY))
    w0 = s1 * c * (eta1 * omega - h * gP0)
    w1 = s2 * c * (eta2 * omega - h * gP1)
    w2 = s0 * c * (eta0 * omega - h * gP2)
    return w0, w1, w2


def boundary_facets(X, tets):
    """Outward boundary triangles in the canonical order (global vertex ids)."""
    tets = np.asarray(tets, dtype=np.int64)
    faces = np.sort(tets[:, _FACE_LOCAL], axis=2).reshape(-1, 3)
    uniq, first, counts = np.unique(faces, axis=0, return_index=True, return_counts=True)
    sel = counts == 1
    tris = uniq[sel].copy()
    cells = first[sel] // 4
    p0, p1, p2 = X[tris[:, 0]], X[tris[:, 1]], X[tris[:, 2]]
    n = np.cross(p1 - p0, p2 - p0)
    nn = np.linalg.norm(n, axis=1)
    keep = nn != 0.0
    tris, cells, n, nn = tris[keep], cells[keep], n[keep], nn[keep]
    p0, p1, p2 = p0[keep], p1[keep], p2[keep]
    n = n / nn[:, None]
    cc = X[tets[cells]].mean(axis=1)
    fc = (p0 + p1 + p2) / 3.0
    flip = np.sum((fc - cc) * n, axis=1) < 0.0
    tris[flip, 1], tris[flip, 2] = tris[flip, 2].copy(), tris[flip, 1].copy()
    p1, p2 = X[tris[:, 1]], X[tris[:, 2]]
    nf = np.cross(p1 - p0, p2 - p0)
    nf = nf / (np.linalg.norm(nf, axis=1) + 1e-30)[:, None]
    n = np.where(flip[:, None], nf, n)
    return tris, n


def boundary_data(X, tets):
    """Restatement of build_boundary_data_serial (Demag_Lindholm.py:177-285).

    Returns a dict with Xb, tri_lid, tri_pts, ntri, area, s_edge, eta, gamma,
    omega_sum plus bverts (global vertex id of each boundary row).
    """
    X = np.asarray(X, dtype=np.float64)
    tets = np.asarray(tets, dtype=np.int64)
    tris, ntri = boundary_facets(X, tets)
    bverts = np.unique(tris.ravel())
    Nb = bverts.size
    Xb = X[bverts].astype(np.float64)
    bmap = -np.ones(X.shape[0], dtype=np.int64)
    bmap[bverts] = np.arange(Nb)
    tri_lid = bmap[tris].astype(np.int32)
    tri_pts = X[tris].astype(np.float64)
    cross = np.cross(tri_pts[:, 1] - tri_pts[:, 0], tri_pts[:, 2] - tri_pts[:, 0])
    area = 0.5 * np.linalg.norm(cross, axis=1)
    e0 = tri_pts[:, 1] - tri_pts[:, 0]
    e1 = tri_pts[:, 2] - tri_pts[:, 1]
    e2 = tri_pts[:, 0] - tri_pts[:, 2]
    s0 = np.linalg.norm(e0, axis=1) + 1e-30
    s1 = np.linalg.norm(e1, axis=1) + 1e-30
    s2 = np.linalg.norm(e2, axis=1) + 1e-30
    s_edge = np.stack([s0, s1, s2], axis=1)
    xi = np.stack([e0 / s0[:, None], e1 / s1[:, None], e2 / s2[:, None]], axis=1)
    eta = np.stack([np.cross(ntri, xi[:, i]) for i in range(3)], axis=1)
    gamma = np.empty((xi.shape[0], 3, 3))
    for i in range(3):
        for j in range(3):
            gamma[:, i, j] = np.sum(xi[:, (i + 1) % 3] * xi[:, j], axis=1)
    # omega_sum: sum over cells of |solid angle| at each boundary vertex
    # (Demag_Lindholm.py:265-283)
    omega_sum = np.zeros(Nb)
    pts = X[tets]
    for j in range(4):
        lid = bmap[tets[:, j]]
        sel = lid >= 0
        P = pts[sel, j]
        T1 = pts[sel, (j + 1) % 4]
        T2 = pts[sel, (j + 2) % 4]
        T3 = pts[sel, (j + 3) % 4]
        np.add.at(omega_sum, lid[sel], np.abs(solid_angle(P, T1, T2, T3)))
    return dict(Xb=Xb, tri_lid=tri_lid, tri_pts=tri_pts, ntri=ntri, area=area,
                s_edge=s_edge, eta=eta, gamma=gamma, omega_sum=omega_sum,
                bverts=bverts.astype(np.int32), tris=tris.astype(np.int32))


def _pair_weights(bd, rows, tri):
    """Weights for all pairs (rows[k], tri[k])."""
    return lindholm_weights(bd["Xb"][rows], bd["tri_pts"][tri, 0], bd["tri_pts"][tri, 1],
                            bd["tri_pts"][tri, 2], bd["ntri"][tri], bd["area"][tri],
                            bd["s_edge"][tri], bd["eta"][tri], bd["gamma"][tri])


def dense_rows(bd, rows, incident_skip=True, chunk=4_000_000, with_diag=True):
    """Rows of the dense double-layer matrix B (assemble_B_rows_owned).

    B[i, i] = omega_sum_i / 4pi - 1 (Demag_Lindholm.py:72-76); off-diagonal
    entries are sums of Lindholm weights over all triangles, skipping the
    triangles incident to the row vertex (:87-96).
    """
    rows = np.asarray(rows, dtype=np.int64)
    Nb = bd["Xb"].shape[0]
    Nt = bd["tri_lid"].shape[0]
    out = np.zeros(rows.size * Nb)
    tl = bd["tri_lid"].astype(np.int64)
    per = max(1, chunk // max(Nt, 1))
    for r0 in range(0, rows.size, per):
        rr = rows[r0:r0 + per]
        R = np.repeat(np.arange(r0, r0 + rr.size), Nt)
        T = np.tile(np.arange(Nt), rr.size)
        g = rows[R]
        if incident_skip:
            keep = (tl[T, 0] != g) & (tl[T, 1] != g) & (tl[T, 2] != g)
            R, T, g = R[keep], T[keep], g[keep]
        w0, w1, w2 = _pair_weights(bd, g, T)
        base = R * Nb
        out += np.bincount(base + tl[T, 0], weights=w0, minlength=out.size)
        out += np.bincount(base + tl[T, 1], weights=w1, minlength=out.size)
        out += np.bincount(base + tl[T, 2], weights=w2, minlength=out.size)
    out = out.reshape(rows.size, Nb)
    if with_diag:
        out[np.arange(rows.size), rows] += bd["omega_sum"][rows] / (4.0 * math.pi) - 1.0
    return out


def dense_B(bd, incident_skip=True):
    Nb = bd["Xb"].shape[0]
    return dense_rows(bd, np.arange(Nb), incident_skip=incident_skip)


def diag_jump(bd):
    """diag_jump = omega_sum/4pi - 1 (Demag_Lindholm_GPU.py:326-328)."""
    return bd["omega_sum"] / (4.0 * math.pi) - 1.0


def fill_block(bd, rows, cols, incident_skip=True):
    """Block B[rows, cols] without the diagonal jump (entry_provider.py:41-117).

    Only triangles incident to at least one block column contribute; each is
    evaluated once per row and scattered to its in-block columns.
    """
    rows = np.asarray(rows, dtype=np.int64)
    cols = np.asarray(cols, dtype=np.int64)
    Nb = bd["Xb"].shape[0]
    col_of = -np.ones(Nb, dtype=np.int64)
    col_of[cols] = np.arange(cols.size)
    tl = bd["tri_lid"].astype(np.int64)
    rel = np.nonzero((col_of[tl] >= 0).any(axis=1))[0]
    rc = col_of[tl[rel]]
    out = np.zeros(rows.size * cols.size)
    if rel.size == 0 or rows.size == 0:
        return out.reshape(rows.size, cols.size)
    R = np.repeat(np.arange(rows.size), rel.size)
    Ti = np.tile(np.arange(rel.size), rows.size)
    g = rows[R]
    T = rel[Ti]
    if incident_skip:
        keep = (tl[T, 0] != g) & (tl[T, 1] != g) & (tl[T, 2] != g)
        R, Ti, T, g = R[keep], Ti[keep], T[keep], g[keep]
    w = _pair_weights(bd, g, T)
    for k in range(3):
        c = rc[Ti, k]
        ok = c >= 0
        out += np.bincount(R[ok] * cols.size + c[ok], weights=w[k][ok], minlength=out.size)
    return out.reshape(rows.size, cols.size)
