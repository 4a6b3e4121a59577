"""Synthetic Kuhn-split box meshes (oracle side).

The reference reads DOLFINx meshes (``gpu/io_utils/mesh.py:6-30``); this
container has no DOLFINx, so every parity case runs on a synthetic box that
the oracle and the product build from the same integer recipe:

* vertex (i, j, k) has index ``i + (nx+1)*(j + (ny+1)*k)`` (i fastest) and
  coordinates ``(i*h, j*h, k*h)`` in nm (the reference's mesh unit, see
  ``gpu/fields/Exchange_GPU.py:62`` where the 1e-18 factor assumes nm);
* every cube is cut into 6 tetrahedra around its 000->111 diagonal, one per
  permutation (a, b, c) of the axes: [v000, v000+e_a, v000+e_a+e_b, v111].
"""
from __future__ import annotations

import itertools

import numpy as np

_PERMS = list(itertools.permutations(range(3)))


def kuhn_box(nx: int, ny: int, nz: int, h: float):
    """Return (X [N,3] float64 nm, tets [E,4] int32) for an nx*ny*nz cube box."""
    nx, ny, nz = int(nx), int(ny), int(nz)
    ii, jj, kk = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1),
                             np.arange(nz + 1), indexing="ij")
    # i fastest: flatten in (k, j, i) order
    X = np.stack([ii.transpose(2, 1, 0).ravel(), jj.transpose(2, 1, 0).ravel(),
                  kk.transpose(2, 1, 0).ravel()], axis=1).astype(np.float64) * float(h)

    def vid(i, j, k):
        return i + (nx + 1) * (j + (ny + 1) * k)

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci = ci.transpose(2, 1, 0).ravel()
    cj = cj.transpose(2, 1, 0).ravel()
    ck = ck.transpose(2, 1, 0).ravel()
    tets = np.empty((ci.size, 6, 4), dtype=np.int64)
    for p, (a, b, _c) in enumerate(_PERMS):
        o0 = np.zeros(3, dtype=np.int64)
        o1 = o0.copy(); o1[a] = 1
        o2 = o1.copy(); o2[b] = 1
        o3 = np.ones(3, dtype=np.int64)
        for q, o in enumerate((o0, o1, o2, o3)):
            tets[:, p, q] = vid(ci + o[0], cj + o[1], ck + o[2])
    return X, tets.reshape(-1, 4).astype(np.int32)


def box_counts(nx, ny, nz):
    """Closed-form (N, E) of a Kuhn box, used by tests as a known answer."""
    return (nx + 1) * (ny + 1) * (nz + 1), 6 * nx * ny * nz
