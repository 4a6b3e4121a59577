"""One ensemble split by sample across two gloo ranks on CPU: the partition balances the
samples' cost, and the states gathered on rank 0 after the run equal the single-rank run bit
for bit.  The per-sample integrator is the oracle's RK4 (each sample integrates on its own),
standing in for LLGEnsemble, whose device run needs a GPU."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
torch = pytest.importorskip("torch")


class OracleEnsemble:
    """Independent samples, each an oracle LLG field (exchange + uniform field) stepped by RK4."""

    def __init__(self, meshes, Ms, H0=None, Aex=1.3e-11, alpha=0.5):
        from oracle import llg as ollg
        self.fields = [ollg.EffectiveFieldOracle(X, T, Ms, Aex=Aex, alpha=alpha,
                                                 H0=np.tile(H0[k], X.shape[0]) if H0 is not None else None)
                       for k, (X, T) in enumerate(meshes)]
        self.sizes = [3 * X.shape[0] for X, _ in meshes]
        self.m = None

    def set_state(self, ms):
        self.m = [np.asarray(m, dtype=np.float64).copy() for m in ms]

    def step(self, dt, n):
        from oracle import llg as ollg
        for _ in range(n):
            self.m = [ollg.rk4_step(f.llg_rhs, m, dt) for f, m in zip(self.fields, self.m)]

    def get_state(self):
        return np.concatenate(self.m)

    def split(self, m):
        out, a = [], 0
        for s in self.sizes:
            out.append(m[a:a + s])
            a += s
        return out


def _problem():
    from oracle import mesh as omesh
    rng = np.random.default_rng(71)
    meshes, m0 = [], []
    for k in range(7):
        nx, ny = int(rng.integers(2, 6)), int(rng.integers(2, 6))
        X, T = omesh.kuhn_box(nx, ny, 2, 2.0)
        meshes.append((X, T))
        m = rng.normal(size=(X.shape[0], 3))
        m0.append((m / np.linalg.norm(m, axis=1)[:, None]).ravel())
    H0 = rng.uniform(-1e5, 1e5, size=(7, 3))
    costs = [float(X.shape[0]) for X, _ in meshes]
    return meshes, m0, H0, costs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      CUDA_VISIBLE_DEVICES="")
    for p in (str(ROOT), str(ROOT / "fenicsx-micromagnetics_b200")):
        sys.path.insert(0, p)
    import datetime
    import torch.distributed as dist
    from spinfemx_b200.ensemble import ShardedEnsemble
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    meshes, m0, H0, costs = _problem()
    ens = ShardedEnsemble(meshes, 8e5, H0=H0, costs=costs, integrator_factory=OracleEnsemble)
    ens.set_state(m0)
    ens.step(1e-14, 5)
    res = ens.gather(dst=0)
    dist.barrier()
    dist.destroy_process_group()
    torch.save({"res": res, "mine": ens.mine}, out / f"rank{rank}.pt")


def test_partition_balances_cost():
    sys.path.insert(0, str(ROOT / "fenicsx-micromagnetics_b200"))
    from spinfemx_b200.ensemble import partition_samples
    costs = [9.0, 7.0, 6.0, 5.0, 4.0, 3.0, 3.0, 1.0]
    parts = partition_samples(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert partition_samples(costs, 1) == [list(range(len(costs)))]


def test_sharded_ensemble_gather_equals_single_rank(tmp_path):
    import torch.multiprocessing as mp
    sys.path.insert(0, str(ROOT / "fenicsx-micromagnetics_b200"))
    sys.path.insert(0, str(ROOT))
    from spinfemx_b200.ensemble import ShardedEnsemble
    ws, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(ws, port, tmp_path), nprocs=ws, join=True, start_method="spawn")
    r0 = torch.load(tmp_path / "rank0.pt", weights_only=False)
    r1 = torch.load(tmp_path / "rank1.pt", weights_only=False)
    assert r1["res"] is None
    assert sorted(r0["mine"] + r1["mine"]) == list(range(7)) and r0["mine"] and r1["mine"]
    meshes, m0, H0, costs = _problem()
    single = ShardedEnsemble(meshes, 8e5, rank=0, world_size=1, H0=H0, costs=costs,
                             integrator_factory=OracleEnsemble)
    single.set_state(m0)
    single.step(1e-14, 5)
    ref = single.gather()
    assert len(r0["res"]) == 7
    for a, b in zip(r0["res"], ref):
        assert np.array_equal(a, b)
