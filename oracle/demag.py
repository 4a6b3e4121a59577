"""FEM/BEM demagnetising field with exact FP64 solves (oracle).

Restates DemagFieldLindholmGPU.compute_vec (gpu/fields/Demag_Lindholm_GPU.py:643-670):

1. u1:  A u1 = Div m with the constant null space removed from the RHS and
   from the solution (:569-582).  The reference uses CG+GAMG to rtol 1e-6;
   the oracle solves exactly (sparse LU on the system with one vertex
   pinned, then projected), as the reference CPU path does below 60k dofs
   (cpu/fields/Demag/Demag_Lindholm.py:669-680).
2. g = B u1|_boundary scattered to the boundary vertices (:585-616).
3. u2:  Dirichlet Laplace problem, u2 = g on the boundary (:618-640).
4. H = G (u1 + u2) / V_i per node (:659-670).
Energy_lumped: E = -1/2 mu0 Ms sum_i V_i m_i.H_i / 1e27 (:706-724).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from . import fem, lindholm

MU0 = 4.0 * math.pi * 1e-7


class DemagOracle:
    def __init__(self, X, tets, Ms, bd=None, B_apply=None, volume_scale=1e27):
        self.X = np.asarray(X, dtype=np.float64)
        self.tets = np.asarray(tets, dtype=np.int64)
        self.Ms = float(Ms)
        self.N = self.X.shape[0]
        self.volume_scale = float(volume_scale)
        self.bd = lindholm.boundary_data(self.X, self.tets) if bd is None else bd
        self.A = fem.stiffness(self.X, self.tets).tocsr()
        self.Div = fem.divergence(self.X, self.tets, self.Ms).tocsr()
        self.G = fem.gradient_op(self.X, self.tets).tocsr()
        self.vol = fem.lumped_volume(self.X, self.tets)
        self.bverts = self.bd["bverts"].astype(np.int64)
        if B_apply is None:
            self.B = lindholm.dense_B(self.bd)
            self.B_apply = lambda x: self.B @ x
        else:
            self.B = None
            self.B_apply = B_apply
        # u1: pin vertex 0 (system is singular with the constants as kernel)
        self._lu1 = spla.splu(self.A[1:, 1:].tocsc())
        interior = np.ones(self.N, dtype=bool)
        interior[self.bverts] = False
        self.interior = np.nonzero(interior)[0]
        self.A_II = self.A[self.interior][:, self.interior].tocsc()
        self.A_IB = self.A[self.interior][:, self.bverts].tocsr()
        self._lu2 = spla.splu(self.A_II) if self.interior.size else None

    def solve_u1(self, m):
        b = self.Div @ np.asarray(m, dtype=np.float64)
        b = b - b.mean()
        u = np.zeros(self.N)
        u[1:] = self._lu1.solve(b[1:])
        return u - u.mean()

    def boundary_data_g(self, u1):
        y = self.B_apply(u1[self.bverts])
        g = np.zeros(self.N)
        g[self.bverts] = y
        return g

    def solve_u2(self, g):
        u2 = g.copy()
        if self._lu2 is not None:
            u2[self.interior] = self._lu2.solve(-(self.A_IB @ g[self.bverts]))
        return u2

    def compute(self, m, return_parts=False):
        u1 = self.solve_u1(m)
        g = self.boundary_data_g(u1)
        u2 = self.solve_u2(g)
        H = (self.G @ (u1 + u2)).reshape(-1, 3) / self.vol[:, None]
        H = H.ravel()
        if return_parts:
            return H, u1, u2, g
        return H

    def energy(self, m, H):
        m = np.asarray(m).reshape(-1, 3)
        H = np.asarray(H).reshape(-1, 3)
        return -0.5 * MU0 * self.Ms * float(np.sum(self.vol * np.sum(m * H, axis=1))) / self.volume_scale
