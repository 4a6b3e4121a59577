"""SVD recompression of the ACA factors and the FP32/FP16 split packing.

Tolerances: after recompression every packing stays within the ACA tolerance 1e-5 of the
dense operator (relative L2 of B x, seeded x) and within 1e-5 of the reference's own
H-matrix product (golden hmat_film48.npz, builder.py); the reported block truncation errors
stay below epsilon; the split packing stores fewer factor bytes than FP32."""
import numpy as np
import pytest

from oracle import mesh as omesh

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda"


def rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


@pytest.mark.parametrize("nx", [48, 100])
def test_recompress_and_split_packing_vs_dense(nx):
    import spinfemx_b200 as spx
    X, T = omesh.kuhn_box(nx, nx, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5), precision="f32")
    b32 = H.memory_report()["far_bytes"]
    g = torch.Generator(device=DEV).manual_seed(11)
    x = torch.randn(H.size, dtype=torch.float64, device=DEV, generator=g)
    B = geom.dense_B()
    yd = B @ x
    del B
    y_aca = H.matvec(x).clone()
    st = H.recompress()
    assert 0 < st["entries_after"] < st["entries_before"] and st["rewritten"] > 0
    assert st["max_rel_truncation"] < 1e-5
    assert H.stats()["far_entries"] == st["entries_after"]
    for prec in ("f64", "f32", "f32_f16"):
        H.repack(prec)
        y = H.matvec(x)
        assert rel(y, yd) < 1e-5, prec
        assert rel(y, y_aca) < 1e-5, prec
        yn = torch.empty_like(x)
        H.matvec_noalloc(x, yn)
        assert torch.equal(yn, y), prec
        if prec == "f32_f16":
            assert H.memory_report()["far_bytes"] < b32
            # the transposed apply (adjoint) of a split-packed matrix: <H x, w> = <x, H^T w>
            w = torch.randn(H.size, dtype=torch.float64, device=DEV, generator=g)
            lhs = float(torch.dot(y, w))
            rhs = float(torch.dot(x, H.rmatvec(w)))
            assert abs(lhs - rhs) <= 1e-6 * float(torch.linalg.norm(y) * torch.linalg.norm(w))


def test_recompressed_vs_reference_hmatrix(golden):
    import spinfemx_b200 as spx
    gd = golden("hmat_film48.npz")
    X, T = omesh.kuhn_box(48, 48, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5, recompress=True),
                                  precision="f32_f16")
    for k in range(3):
        y = H.matvec(torch.as_tensor(gd["x"][:, k].copy(), device=DEV)).cpu().numpy()
        assert np.linalg.norm(y - gd["Hx"][:, k]) <= 1e-5 * np.linalg.norm(gd["Hx"][:, k])


def test_split_packing_in_the_demag_pipeline(golden):
    """Box of the small-box workload: the demag field with f32_f16 H factors against the oracle."""
    import math
    import spinfemx_b200 as spx
    from oracle import demag as odemag
    X, T = omesh.kuhn_box(20, 20, 5, 2.0)
    o = odemag.DemagOracle(X, T, 8e5)
    rng = np.random.default_rng(1000)
    m = np.tile(np.array([1.0, 1.0, 1.0]) / math.sqrt(3.0), (X.shape[0], 1)) + rng.normal(0.0, 0.1, (X.shape[0], 3))
    m = (m / np.linalg.norm(m, axis=1)[:, None]).ravel()
    Href = o.compute(m)
    d = spx.DemagFieldLindholmGPU(X, T, 8e5, boundary_backend="hmatrix", hmatrix_epsilon=1e-5, precision="mixed",
                                  hmatrix_precision="f32_f16", ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10, ksp_atol=0.0)
    mt = torch.as_tensor(m, device=DEV)
    out = torch.empty_like(mt)
    d.compute_vec(mt, out)
    assert np.linalg.norm(out.cpu().numpy() - Href) <= 1e-5 * np.linalg.norm(Href)
