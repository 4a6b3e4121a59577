"""Failure detection without a GPU fault: a grid barrier that one CTA never reaches makes the
other CTAs' bounded waits run out.  The kernel records SPX_ERR_TIMEOUT and returns, the host
reads the status, and the context keeps working (the same bounded wait guards the barriers
of the persistent CG and AMG-PCG kernels)."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from oracle import mesh as omesh

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("nblocks", [2, 16])
def test_barrier_wait_runs_out_and_reports(nblocks):
    import spinfemx_b200 as spx
    from spinfemx_b200 import _lib
    status, gave_up = C.c_int32(-1), C.c_int32(-1)
    _lib.call("spx_debug_barrier_probe", nblocks, 1 << 14, C.byref(status), C.byref(gave_up))
    assert status.value == 5  # SPX_ERR_TIMEOUT
    assert gave_up.value == nblocks - 1
    # the context is still usable: a demag evaluation runs and matches a second one
    X, T = omesh.kuhn_box(4, 4, 2, 2.0)
    d = spx.DemagFieldLindholmGPU(X, T, 8e5, boundary_backend="dense", precision="f64")
    m = torch.as_tensor(np.tile([0.0, 0.6, 0.8], X.shape[0]), device="cuda")
    H1, H2 = torch.empty_like(m), torch.empty_like(m)
    d.compute_vec(m, H1)
    d.compute_vec(m, H2)
    torch.cuda.synchronize()
    assert torch.isfinite(H1).all() and torch.allclose(H1, H2, rtol=1e-10, atol=0.0)


def test_barrier_cost_is_measured():
    """The phase boundary of the persistent solvers, timed alone: finite, a few microseconds,
    and no wait ran out (the call checks the error word)."""
    import spinfemx_b200  # noqa: F401  (loads the library)
    from spinfemx_b200 import _lib
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    for threads in (1024, 256):
        us = C.c_double()
        _lib.call("spx_debug_barrier_time", nsm, threads, 2000, C.byref(us))
        assert 0.0 < us.value < 50.0, (threads, us.value)


def test_probe_rejects_bad_arguments():
    from spinfemx_b200 import _lib
    status, gave_up = C.c_int32(), C.c_int32()
    assert _lib.lib().spx_debug_barrier_probe(1, 100, C.byref(status), C.byref(gave_up)) == 1
    assert _lib.lib().spx_debug_barrier_probe(4, 0, C.byref(status), C.byref(gave_up)) == 1
    us = C.c_double()
    assert _lib.lib().spx_debug_barrier_time(0, 1024, 10, C.byref(us)) == 1
    assert _lib.lib().spx_debug_barrier_time(4, 1000, 10, C.byref(us)) == 1


def test_hmatrix_build_recovers_from_out_of_memory():
    """An allocation failure during the H-matrix build (injected on the host, no device fault)
    makes the build retry with half the workspace; the result equals a normal build.  With
    every large allocation failing, the build raises MemoryError and the context stays usable."""
    import spinfemx_b200 as spx
    from spinfemx_b200 import _lib
    X, T = omesh.kuhn_box(30, 30, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    cfg = spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=64, batch_bytes=1 << 30)
    H0 = spx.HMatrixGPUPackedFused(geom, cfg, precision="f64")
    x = torch.as_tensor(np.random.default_rng(8).standard_normal(H0.size), device="cuda")
    y0 = H0.matvec(x).clone()
    try:
        _lib.call("spx_debug_fail_alloc", 1 << 20, 1)   # the first fill/ACA workspace fails
        H1 = spx.HMatrixGPUPackedFused(geom, cfg, precision="f64")
        assert torch.equal(H1.matvec(x), y0)
        assert H1.stats()["n_far"] == H0.stats()["n_far"]
        _lib.call("spx_debug_fail_alloc", 1 << 20, 1 << 20)   # every large allocation fails
        with pytest.raises(MemoryError):
            spx.HMatrixGPUPackedFused(geom, cfg, precision="f64")
    finally:
        _lib.call("spx_debug_fail_alloc", 0, 0)
    assert torch.equal(H0.matvec(x), y0)
