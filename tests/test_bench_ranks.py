"""The multi-rank logic of bench.py on CPU: two gloo ranks, as torchrun starts them on GPUs
(one process per GPU).  Whole-job values are the units of all ranks over the slowest rank's
time, each rank of the ensemble workload draws its own samples, and every rank takes the
same collective steps."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(ws), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    sys.path.insert(0, str(ROOT))
    import bench
    r, w, local = bench.dist_init(ws, timeout_s=60)
    assert (r, w, local) == (rank, ws, rank)
    bench.barrier(w)
    ms = 10.0 + 5.0 * rank  # this rank's device time
    ms_max = bench.allmax(ms, w)
    boxes = bench.ensemble_boxes(8, 7000 + r)
    rate = bench.job_rate(40, ms_max, w)
    bench.finish(w)
    torch.save({"ms_max": ms_max, "boxes": boxes, "rate": rate}, out / f"rank{rank}.pt")


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    ws, port = 2, _free_port()
    mp.start_processes(_rank_main, args=(ws, port, tmp_path), nprocs=ws, join=True, start_method="spawn")
    res = [torch.load(tmp_path / f"rank{r}.pt") for r in range(ws)]
    assert res[0]["ms_max"] == res[1]["ms_max"] == 15.0          # the slowest rank's time on every rank
    assert res[0]["rate"] == pytest.approx(2 * 40 / 15e-3)       # all ranks' steps over that time
    assert res[0]["boxes"] != res[1]["boxes"]                    # samples sharded by rank, no overlap
    sys.path.insert(0, str(ROOT))
    import bench
    assert res[0]["boxes"] == bench.ensemble_boxes(8, 7000)      # rank 0 draws what one GPU draws


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.allmax(3.5, 1) == 3.5
    assert bench.job_rate(40, 500.0, 1) == pytest.approx(80.0)
