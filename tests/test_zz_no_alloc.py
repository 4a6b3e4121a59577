"""spx_hmat_apply_noalloc: the H-matrix apply for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc while they run, for example a time-stepper callback
whose device memory belongs to another allocator's pool.  For them the library offers
spx_hmat_apply_noalloc, which keeps its scratch in a fixed device array instead of
allocating it.  This file checks it through the C ABI against spx_hmat_apply on two
calls in a row (the scratch keeps the previous call's contents).  It sits last in
collection order so that a stop-at-first-failure run has already run every other test.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_hmat_apply_noalloc_matches_apply(precision):
    import spinfemx_b200 as spx
    from spinfemx_b200 import _lib
    from oracle import mesh

    X, T = mesh.kuhn_box(30, 30, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=64),
                                  precision=precision)
    stream = _lib.stream_ptr()
    rng = np.random.default_rng(4321)
    # a fresh handle: the no-allocation calls come first and must not create the apply
    # buffers that spx_hmat_apply allocates on its first call
    before = H.memory_report()["accounted_gpu_bytes"]
    xs = [torch.as_tensor(rng.standard_normal(H.size), device="cuda") for _ in range(2)]
    outs = []
    for call_no, x in enumerate(xs):
        y_na = torch.full_like(x, float("nan"))
        _lib.check(_lib.lib().spx_hmat_apply_noalloc(H._h, _lib.ptr(x), _lib.ptr(y_na), stream))
        torch.cuda.synchronize()
        outs.append(y_na.cpu().numpy())
        assert H.memory_report()["accounted_gpu_bytes"] == before, call_no
    for call_no, x in enumerate(xs):
        y_ref = torch.empty_like(x)
        _lib.check(_lib.lib().spx_hmat_apply(H._h, _lib.ptr(x), _lib.ptr(y_ref), stream))
        torch.cuda.synchronize()
        a, b = outs[call_no], y_ref.cpu().numpy()
        assert np.all(np.isfinite(a)), call_no
        assert np.linalg.norm(a - b) <= 1e-12 * np.linalg.norm(b), call_no
    assert H.memory_report()["accounted_gpu_bytes"] > before  # spx_hmat_apply did allocate
    # the Python wrapper reaches the same entry point
    out = torch.empty_like(xs[1])
    H.matvec_noalloc(xs[1], out)
    torch.cuda.synchronize()
    assert np.linalg.norm(out.cpu().numpy() - outs[1]) <= 1e-12 * np.linalg.norm(outs[1])


def test_hmat_apply_noalloc_refuses_too_large():
    """An H-matrix whose scratch does not fit the static array is refused before any launch:
    SPX_ERR_INVALID with a message that names the needed bytes, the output left untouched,
    the handle still usable.  The 32 MiB array is lowered to 4 KiB for the test
    (spx_debug_noalloc_cap) so that a small film needs more than it holds."""
    import spinfemx_b200 as spx
    from spinfemx_b200 import _lib
    from oracle import mesh

    X, T = mesh.kuhn_box(20, 20, 2, 2.5)
    H = spx.HMatrixGPUPackedFused(spx.BoundaryGeometry(X, T),
                                  spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=64), precision="f32")
    stream = _lib.stream_ptr()
    x = torch.ones(H.size, dtype=torch.float64, device="cuda")
    y = torch.full_like(x, float("nan"))
    lib = _lib.lib()
    try:
        _lib.check(lib.spx_debug_noalloc_cap(4096))
        rc = lib.spx_hmat_apply_noalloc(H._h, _lib.ptr(x), _lib.ptr(y), stream)
        msg = lib.spx_last_error().decode()
    finally:
        _lib.check(lib.spx_debug_noalloc_cap(0))
    torch.cuda.synchronize()
    assert rc == _lib.SPX_ERR_INVALID
    assert "too large" in msg and "needs" in msg
    assert torch.isnan(y).all()
    _lib.check(lib.spx_hmat_apply_noalloc(H._h, _lib.ptr(x), _lib.ptr(y), stream))
    torch.cuda.synchronize()
    assert np.abs(y.cpu().numpy() + 1.0).max() < 1e-5   # H 1 = -1
