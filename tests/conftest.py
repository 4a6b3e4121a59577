import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_PARENT = ROOT / "fenicsx-micromagnetics_b200"
for p in (str(ROOT), str(PKG_PARENT)):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return np.load(GOLDEN / name)
    return load


@pytest.fixture(scope="session")
def box20_mesh():
    from oracle import mesh
    return mesh.kuhn_box(20, 20, 5, 2.0)


@pytest.fixture(scope="session")
def box20_bd(box20_mesh):
    from oracle import lindholm
    return lindholm.boundary_data(*box20_mesh)


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


os.environ.setdefault("NUMBA_NUM_THREADS", str(os.cpu_count() or 1))
