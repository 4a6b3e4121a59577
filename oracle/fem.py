"""P1 finite-element operators on a tetrahedral mesh (oracle).

DOLFINx is absent here, so the UFL forms of the reference are restated as
explicit P1 element formulas (mesh coordinates in nm):

* stiffness  a(u,v) = int grad u . grad v         Demag_Lindholm_GPU.py:188-190, :247-251
* Div        Ms int grad v . m                    Demag_Lindholm_GPU.py:199-205
* G          int v . (-grad phi)                  Demag_Lindholm_GPU.py:554-560
* lumped VolN = int v . (1,1,1)                   llg_module_GPU.py:469-484
* exchange K = diag(-2A/(mu0 Ms V_i) 1e18) * vector stiffness   Exchange_GPU.py:53-68
* interfacial DMI K (volume + half boundary term), row-scaled by
  -2D/(mu0 Ms)/1e-9/V_i                           DMI_Interfacial_GPU.py:140-172

Matrices are scipy CSR; vectors are AoS (node-major, 3 components).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

MU0 = 4.0 * math.pi * 1e-7


def tet_geometry(X, tets):
    """Per-tet volume [E] and barycentric gradients [E,4,3] (1/nm)."""
    X = np.asarray(X, dtype=np.float64)
    P = X[np.asarray(tets, dtype=np.int64)]
    M = np.stack([P[:, 1] - P[:, 0], P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]], axis=1)
    det = np.linalg.det(M)
    Minv = np.linalg.inv(M)          # grad lambda_k (k=1..3) = column k-1 of inv(M)
    g = np.empty((P.shape[0], 4, 3))
    g[:, 1:, :] = np.transpose(Minv, (0, 2, 1))
    g[:, 0, :] = -g[:, 1:, :].sum(axis=1)
    return np.abs(det) / 6.0, g


def stiffness(X, tets):
    tets = np.asarray(tets, dtype=np.int64)
    N = X.shape[0]
    vol, g = tet_geometry(X, tets)
    K = vol[:, None, None] * np.einsum("eac,ebc->eab", g, g)
    rows = np.repeat(tets, 4, axis=1).ravel()
    cols = np.tile(tets, (1, 4)).ravel()
    return sp.csr_matrix((K.ravel(), (rows, cols)), shape=(N, N))


def lumped_volume(X, tets):
    """Scalar nodal volume V_i = int phi_i (nm^3)."""
    vol, _ = tet_geometry(X, tets)
    return np.bincount(np.asarray(tets, dtype=np.int64).ravel(),
                       weights=np.repeat(vol / 4.0, 4), minlength=X.shape[0])


def divergence(X, tets, Ms):
    """Div [N, 3N]: Div[i, 3j+c] = Ms sum_e vol_e/4 d_c lambda_i."""
    tets = np.asarray(tets, dtype=np.int64)
    N = X.shape[0]
    vol, g = tet_geometry(X, tets)
    E = tets.shape[0]
    vals = (Ms * vol / 4.0)[:, None, None, None] * g[:, :, None, :] * np.ones((E, 4, 4, 3))
    rows = np.broadcast_to(tets[:, :, None, None], (E, 4, 4, 3)).ravel()
    cols = (3 * np.broadcast_to(tets[:, None, :, None], (E, 4, 4, 3))
            + np.arange(3)[None, None, None, :]).ravel()
    return sp.csr_matrix((vals.ravel(), (rows, cols)), shape=(N, 3 * N))


def gradient_op(X, tets):
    """G [3N, N]: G[3i+c, j] = -sum_e vol_e/4 d_c lambda_j."""
    tets = np.asarray(tets, dtype=np.int64)
    N = X.shape[0]
    vol, g = tet_geometry(X, tets)
    E = tets.shape[0]
    vals = -(vol / 4.0)[:, None, None, None] * np.broadcast_to(g[:, None, :, :], (E, 4, 4, 3))
    vals = np.transpose(vals, (0, 1, 3, 2))            # [e, a(row node), c, b(col node)]
    rows = (3 * np.broadcast_to(tets[:, :, None, None], (E, 4, 3, 4))
            + np.arange(3)[None, None, :, None]).ravel()
    cols = np.broadcast_to(tets[:, None, None, :], (E, 4, 3, 4)).ravel()
    return sp.csr_matrix((vals.ravel(), (rows, cols)), shape=(3 * N, N))


def vector_block(Ks):
    """Scalar [N,N] -> block-diagonal vector operator [3N,3N] (AoS)."""
    return sp.kron(Ks, sp.identity(3), format="csr")


def exchange_matrix(X, tets, A, Ms, vol=None):
    if vol is None:
        vol = lumped_volume(X, tets)
    pref = -2.0 * A / (MU0 * Ms) / vol / 1e-18
    return sp.diags(np.repeat(pref, 3)) @ vector_block(stiffness(X, tets))


def _facet_triple_mass(area, a, b, k):
    """int_T phi_a phi_b phi_k over a triangle (local ids), exact."""
    cnt = np.zeros(3, dtype=int)
    for i in (a, b, k):
        cnt[i] += 1
    num = math.factorial(cnt[0]) * math.factorial(cnt[1]) * math.factorial(cnt[2])
    return 2.0 * area * num / math.factorial(2 + cnt.sum())


def dmi_interfacial_matrix(X, tets, D, Ms, n_nodes, bd_tris, bd_normals, vol=None):
    """Interfacial DMI operator, restating DMI_Interfacial_GPU.py:140-172.

    Volume form int (div(u) n - grad(n.u)) . v with n a P1 field, plus
    0.5 int_ds ((n x nu) x u) . v on the boundary (nu outward normal), all
    row-scaled by -2D/(mu0 Ms)/1e-9/V_i.
    """
    tets = np.asarray(tets, dtype=np.int64)
    N = X.shape[0]
    if vol is None:
        vol = lumped_volume(X, tets)
    nN = np.asarray(n_nodes, dtype=np.float64).reshape(N, 3)
    tv, g = tet_geometry(X, tets)
    E = tets.shape[0]
    Mloc = (tv / 20.0)[:, None, None] * (np.ones((4, 4)) + np.eye(4))[None]   # int phi_a phi_b
    nE = nN[tets]                                     # [E,4,3]
    Mn = np.einsum("eak,ekc->eac", Mloc, nE)          # sum_k M_ak n_{k,c}
    dn = np.einsum("ekd,ekc->ecd", nE, g)             # d_c n_d  [E,c,d]
    # K[a c, b d] = g_b,d Mn_a,c - dn_c,d M_ab - g_b,c Mn_a,d
    Kl = (np.einsum("ebd,eac->eacbd", g, Mn)
          - np.einsum("ecd,eab->eacbd", dn, Mloc)
          - np.einsum("ebc,ead->eacbd", g, Mn))
    rows = (3 * np.broadcast_to(tets[:, :, None, None, None], (E, 4, 3, 4, 3))
            + np.arange(3)[None, None, :, None, None])
    cols = (3 * np.broadcast_to(tets[:, None, None, :, None], (E, 4, 3, 4, 3))
            + np.arange(3)[None, None, None, None, :])
    K = sp.csr_matrix((Kl.ravel(), (rows.ravel(), cols.ravel())), shape=(3 * N, 3 * N))
    # boundary term 0.5 int phi_a phi_b (nu_c n_d - n_c nu_d)
    tris = np.asarray(bd_tris, dtype=np.int64)
    nu = np.asarray(bd_normals, dtype=np.float64)
    P = X[tris]
    area = 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    nT = nN[tris]                                     # [F,3(k),3]
    F = tris.shape[0]
    Bl = np.zeros((F, 3, 3, 3, 3))                    # [f, a, c, b, d]
    for a in range(3):
        for b in range(3):
            # int phi_a phi_b n  (vector) over the facet
            w = np.stack([_facet_triple_mass(1.0, a, b, k) for k in range(3)])  # per unit area
            nab = area[:, None] * np.einsum("k,fkd->fd", w, nT)                 # [F,3]
            Bl[:, a, :, b, :] = 0.5 * (nu[:, :, None] * nab[:, None, :] - nab[:, :, None] * nu[:, None, :])
    rows = (3 * np.broadcast_to(tris[:, :, None, None, None], (F, 3, 3, 3, 3))
            + np.arange(3)[None, None, :, None, None])
    cols = (3 * np.broadcast_to(tris[:, None, None, :, None], (F, 3, 3, 3, 3))
            + np.arange(3)[None, None, None, None, :])
    K = K + sp.csr_matrix((Bl.ravel(), (rows.ravel(), cols.ravel())), shape=(3 * N, 3 * N))
    pref = -2.0 * D / (MU0 * Ms) / 1e-9 / vol
    return (sp.diags(np.repeat(pref, 3)) @ K).tocsr()


def dmi_bulk_matrix(X, tets, D, Ms, bd_tris, bd_normals, vol=None):
    """Bulk DMI operator, restating DMI_Bulk_GPU.py:52-66: the form
    -int curl(u) . v dx + 0.5 int_ds (nu x u) . v (nu outward normal), row-scaled by
    2D/(mu0 Ms) * 1e9 / V_i (mesh in nm)."""
    tets = np.asarray(tets, dtype=np.int64)
    N = X.shape[0]
    if vol is None:
        vol = lumped_volume(X, tets)
    tv, g = tet_geometry(X, tets)
    E = tets.shape[0]
    eps = np.zeros((3, 3, 3))
    eps[0, 1, 2] = eps[1, 2, 0] = eps[2, 0, 1] = 1.0
    eps[0, 2, 1] = eps[2, 1, 0] = eps[1, 0, 2] = -1.0
    # curl(phi_b e_d)_c = eps_{c k d} d_k phi_b ; int phi_a = vol / 4
    C = np.einsum("ckd,ebk->ebcd", eps, g)                         # [E, b, c, d]
    Kl = -(tv / 4.0)[:, None, None, None, None] * np.broadcast_to(C[:, None], (E, 4, 4, 3, 3))
    Kl = np.transpose(Kl, (0, 1, 3, 2, 4))                           # [E, a, c, b, d]
    rows = (3 * np.broadcast_to(tets[:, :, None, None, None], (E, 4, 3, 4, 3))
            + np.arange(3)[None, None, :, None, None])
    cols = (3 * np.broadcast_to(tets[:, None, None, :, None], (E, 4, 3, 4, 3))
            + np.arange(3)[None, None, None, None, :])
    K = sp.csr_matrix((Kl.ravel(), (rows.ravel(), cols.ravel())), shape=(3 * N, 3 * N))
    tris = np.asarray(bd_tris, dtype=np.int64)
    nu = np.asarray(bd_normals, dtype=np.float64)
    P = X[tris]
    area = 0.5 * np.linalg.norm(np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0]), axis=1)
    F = tris.shape[0]
    Cn = np.einsum("ckd,fk->fcd", eps, nu)                           # (nu x e_d)_c
    mab = (np.ones((3, 3)) + np.eye(3)) / 12.0                       # int_F phi_a phi_b / area
    Bl = 0.5 * area[:, None, None, None, None] * mab[None, :, None, :, None] * Cn[:, None, :, None, :]
    rows = (3 * np.broadcast_to(tris[:, :, None, None, None], (F, 3, 3, 3, 3))
            + np.arange(3)[None, None, :, None, None])
    cols = (3 * np.broadcast_to(tris[:, None, None, :, None], (F, 3, 3, 3, 3))
            + np.arange(3)[None, None, None, None, :])
    K = K + sp.csr_matrix((Bl.ravel(), (rows.ravel(), cols.ravel())), shape=(3 * N, 3 * N))
    pref = 2.0 * D / (MU0 * Ms) * 1e9 / vol
    return (sp.diags(np.repeat(pref, 3)) @ K).tocsr()


def anisotropy_field(m, n_axis, Ku, Ms):
    """Nodal uniaxial field H = 2Ku/(mu0 Ms) (m.n) n (Anisotropy_GPU.py:317-330).

    ``Ku`` may be a scalar or a per-node array (spatial Ku(x) extension).
    """
    m = np.asarray(m).reshape(-1, 3)
    n = np.asarray(n_axis).reshape(-1, 3)
    pref = 2.0 * np.asarray(Ku, dtype=np.float64) / (MU0 * Ms)
    c = pref * np.sum(m * n, axis=1)
    return (c[:, None] * n).ravel()


def anisotropy_diag(n_axis, Ku, Ms):
    n = np.asarray(n_axis).reshape(-1, 3)
    pref = 2.0 * np.asarray(Ku, dtype=np.float64) / (MU0 * Ms)
    return (np.atleast_1d(pref)[:, None] * n * n if np.ndim(pref) else pref * n * n).ravel()
