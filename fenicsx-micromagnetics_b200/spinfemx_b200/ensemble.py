"""Ensembles of independent samples integrated together (no counterpart in the reference,
which builds one field object per mesh).

The samples' meshes are concatenated into one disjoint-union mesh: every pipeline phase
(FEM SpMVs, the two Poisson solves, the boundary operator, the fused field/RHS/RK4 stage
kernel) is then one launch for all samples, whatever their sizes.  The boundary operator is
block diagonal (``DemagFieldLindholmGPU(boundary_backend="ensemble")``): each sample's
Lindholm operator over its own boundary, dense for small samples (all applied by one batched
launch) and an H-matrix for large ones.  Samples share the material constants; the applied
field (and the initial magnetisation) is per sample.
"""
from __future__ import annotations

import numpy as np

from .geometry import as_mesh
from .llg import EffectiveField


def ensemble_mesh(meshes):
    """(X, tets, offsets) of the disjoint union of [(X_s, tets_s), ...]; sample s owns nodes
    offsets[s]:offsets[s+1]."""
    Xs, Ts, offs = [], [], [0]
    for X, T in meshes:
        X, T = as_mesh(X, T)
        Xs.append(X)
        Ts.append(T.astype(np.int64) + offs[-1])
        offs.append(offs[-1] + X.shape[0])
    X = np.ascontiguousarray(np.concatenate(Xs), dtype=np.float64)
    T = np.ascontiguousarray(np.concatenate(Ts), dtype=np.int32)
    return X, T, np.asarray(offs, dtype=np.int64)


class LLGEnsemble:
    """RK4 integration of independent samples in one set of launches per stage."""

    def __init__(self, meshes, Ms, *, Aex=0.0, Ku=0.0, n_ani=(0.0, 0.0, 1.0), D_int=0.0, n_int=(0.0, 0.0, 1.0),
                 alpha=0.5, gamma=2.211e5, H0=None, use_demag=True, dense_max_nb=4096, precision="mixed",
                 demag_kwargs=None, graph=False):
        self.X, self.tets, self.offsets = ensemble_mesh(meshes)
        self.nsamples = len(self.offsets) - 1
        N = self.X.shape[0]
        self.N = N
        counts = np.diff(self.offsets)
        H0n = None
        if H0 is not None:
            h = np.asarray(H0, dtype=np.float64)
            h = np.tile(h.reshape(1, 3), (self.nsamples, 1)) if h.size == 3 else h.reshape(self.nsamples, 3)
            H0n = np.repeat(h, counts, axis=0).ravel()
        dk = dict(demag_kwargs or {})
        dk.update(boundary_backend="ensemble", sample_offsets=self.offsets, dense_max_nb=int(dense_max_nb))
        dk.setdefault("precision", precision)
        self.hef = EffectiveField(self.X, self.tets, Ms, Aex=Aex, Ku=Ku,
                                  n_ani_vec=n_ani if Ku != 0.0 else None, D_int=D_int,
                                  n0_int_vec=n_int if D_int != 0.0 else None, alpha=alpha, gamma=gamma,
                                  use_demag=use_demag, demag_kwargs=dk, H0_static=H0n, precision=precision)
        if graph:
            self.hef.set_graph(True)

    def join(self, ms):
        """Union state (3N) from per-sample states [(3 N_s), ...]."""
        return np.concatenate([np.asarray(m, dtype=np.float64).ravel() for m in ms])

    def split(self, m):
        """Per-sample views of a union state (numpy or torch, length 3N)."""
        return [m[3 * a:3 * b] for a, b in zip(self.offsets[:-1], self.offsets[1:])]

    def set_state(self, m):
        import torch
        if isinstance(m, (list, tuple)):
            m = self.join(m)
        self.hef.set_state(torch.as_tensor(np.asarray(m) if not isinstance(m, torch.Tensor) else m,
                                           dtype=torch.float64, device="cuda").contiguous())

    def step(self, dt, nsteps=1):
        self.hef.step(dt, nsteps)

    def get_state(self):
        return self.hef.get_state()
