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


# ---------------------------------------------------------------- one ensemble over several ranks
def sample_cost(X, tets, dense_max_nb=4096):
    """Work estimate of one sample per step: N (FEM and Poisson solves) + Nb^2 for a dense
    boundary operator, or + 64 Nb (about the factor entries per row) for an H-matrix."""
    from .geometry import boundary_data
    N = int(np.asarray(X).shape[0])
    Nb = int(boundary_data(X, tets)["bverts"].shape[0])
    return float(N + (Nb * Nb if Nb <= dense_max_nb else 64 * Nb))


def partition_samples(costs, world_size):
    """Samples dealt to ranks with balanced total cost (largest first, each to the least loaded
    rank; ties to the lower rank).  Returns, per rank, its sample indices in increasing order."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * int(world_size)
    parts = [[] for _ in range(int(world_size))]
    for i in order:
        r = min(range(int(world_size)), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


class ShardedEnsemble:
    """One ensemble split by sample across the ranks of a torch.distributed process group.

    Each rank integrates its own samples (an LLGEnsemble of them, or what
    ``integrator_factory(meshes, Ms, H0=..., **kw)`` builds); the only exchange is the final
    gather of every sample's state to one rank (``gather``), in the ensemble's sample order.
    Per-sample arguments (H0, initial states) are given for the whole ensemble on every rank."""

    def __init__(self, meshes, Ms, *, rank=None, world_size=None, H0=None, costs=None, dense_max_nb=4096,
                 integrator_factory=None, **kw):
        import torch.distributed as dist
        self.ws = int(world_size if world_size is not None else (dist.get_world_size() if dist.is_initialized()
                                                                 else 1))
        self.rank = int(rank if rank is not None else (dist.get_rank() if dist.is_initialized() else 0))
        self.nsamples = len(meshes)
        if costs is None:
            costs = [sample_cost(X, T, dense_max_nb) for X, T in meshes]
        self.parts = partition_samples(costs, self.ws)
        self.mine = self.parts[self.rank]
        h = None
        if H0 is not None:
            h = np.asarray(H0, dtype=np.float64)
            h = np.tile(h.reshape(1, 3), (self.nsamples, 1)) if h.size == 3 else h.reshape(self.nsamples, 3)
        factory = integrator_factory or (lambda ms, Ms_, **k: LLGEnsemble(ms, Ms_, dense_max_nb=dense_max_nb, **k))
        self.local = factory([meshes[i] for i in self.mine], Ms,
                             H0=None if h is None else h[self.mine], **kw) if self.mine else None

    def set_state(self, ms):
        """ms: the initial states of all samples (list of 3 N_s arrays)."""
        if self.local is not None:
            self.local.set_state([ms[i] for i in self.mine])

    def step(self, dt, nsteps=1):
        if self.local is not None:
            self.local.step(dt, nsteps)

    def local_states(self):
        """{sample index: state (numpy, 3 N_s)} of this rank's samples."""
        if self.local is None:
            return {}
        m = self.local.get_state()
        m = m.cpu().numpy() if hasattr(m, "cpu") else np.asarray(m)
        return {i: np.array(v, copy=True) for i, v in zip(self.mine, self.local.split(m))}

    def gather(self, dst=0):
        """The states of all samples (list in sample order) on rank dst; None elsewhere."""
        import torch.distributed as dist
        mine = self.local_states()
        if self.ws == 1 or not dist.is_initialized():
            return [mine[i] for i in range(self.nsamples)]
        out = [None] * self.ws if self.rank == dst else None
        dist.gather_object(mine, out, dst=dst)
        if self.rank != dst:
            return None
        allst = {}
        for d in out:
            allst.update(d)
        return [allst[i] for i in range(self.nsamples)]
