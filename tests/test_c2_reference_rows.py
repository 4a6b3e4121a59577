"""The H-matrix of the headline film against the reference's own dense rows.

Film 400 x 400 x 2 cubes of 2.5 nm (N = 482,403, Nb = 323,202).  The fixture
``golden/c2_rows.npz`` holds 4,096 seeded rows of the reference's dense Lindholm
operator (``LindholmEntryProviderCPU.fill_block(rows, all)``,
lindholm_hmatrix_gpu/entry_provider.py:120-247, plus the diagonal jump
Omega/4pi - 1, Demag_Lindholm.py:87-96) applied to three vectors (``row_vectors``),
and the rows' sums.  It was made by ``tests/golden/make_golden.py c2_rows``.

Tolerances (relative L2 over the 4,096 rows, per vector):
  H-matrix (ACA 1e-5, leaf 64, eta 2), FP64 factors   1e-5 (the ACA tolerance)
  the same H-matrix packed with FP32 factors          1e-5
  recompressed, FP32 + FP16 split columns             1e-5
  row sums of H (H 1 = -1 on every row)               1e-5 absolute
"""
import numpy as np
import pytest

from bench import c2_row_vectors as row_vectors

CASE = (400, 400, 2, 2.5)


def rows_rel_err(y, ref):
    return [float(np.linalg.norm(y[:, k] - ref[:, k]) / np.linalg.norm(ref[:, k])) for k in range(ref.shape[1])]


def test_fixture_matches_boundary_order(golden):
    """The fixture's vectors regenerate from the library's boundary data (same node
    order and count as the oracle's, which made the fixture)."""
    import spinfemx_b200 as spx
    from spinfemx_b200.geometry import kuhn_box
    g = golden("c2_rows.npz")
    X, T = kuhn_box(*CASE[:3], CASE[3])
    bd = spx.boundary_data(X, T)
    assert bd["Xb"].shape[0] == int(g["nb"])
    x = row_vectors(bd["Xb"])
    assert np.allclose(x.sum(0), g["x_sum"], rtol=1e-12, atol=1e-9)
    assert np.allclose((x * x).sum(0), g["x_sqsum"], rtol=1e-12)
    assert np.abs(g["rowsum"] + 1.0).max() < 1e-9


def test_oracle_rows_vs_reference_rows(golden):
    """The oracle's dense rows (oracle/lindholm.py) equal the reference's on a subset."""
    from oracle import lindholm as olin
    from oracle import mesh as omesh
    g = golden("c2_rows.npz")
    X, T = omesh.kuhn_box(*CASE)
    bd = olin.boundary_data(X, T)
    x = row_vectors(bd["Xb"])
    sel = np.arange(0, g["rows"].size, 512)
    B = olin.dense_rows(bd, g["rows"][sel])
    assert np.abs(B @ x - g["y"][sel]).max() <= 1e-10 * np.abs(g["y"][sel]).max()


@pytest.mark.gpu
def test_c2_hmatrix_vs_reference_rows(golden):
    torch = pytest.importorskip("torch")
    import spinfemx_b200 as spx
    from spinfemx_b200.geometry import kuhn_box
    g = golden("c2_rows.npz")
    X, T = kuhn_box(*CASE[:3], CASE[3])
    geom = spx.BoundaryGeometry(X, T)
    bd = spx.boundary_data(X, T)
    x = row_vectors(bd["Xb"])
    rows = g["rows"]
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=64),
                                  precision="f64")
    ones = torch.ones(H.size, dtype=torch.float64, device="cuda")
    for prec in ("f64", "f32", "recompressed f32_f16"):
        if prec == "f32":
            H.repack("f32")
        elif prec.startswith("recompressed"):
            st = H.recompress()
            assert st["entries_after"] < st["entries_before"]
            H.repack("f32_f16")
        y = np.stack([H.matvec(torch.as_tensor(x[:, k].copy(), device="cuda")).cpu().numpy()[rows]
                      for k in range(3)], 1)
        errs = rows_rel_err(y, g["y"])
        assert max(errs) < 1e-5, (prec, errs)
        rs = H.matvec(ones).cpu().numpy()[rows]
        assert np.abs(rs - g["rowsum"]).max() < 1e-5, prec
