"""The multi-state apply with the far field on the tensor cores (tcgen05 kind::i8: FP32
factors as 31-bit and FP64 states as 47-bit fixed-point values cut into base-256 digits, exact
int32 digit-pair sums, FP64 epilogue) against the CUDA-core paths.

Tolerances (relative L2 per state): tensor-core batch vs single applies of the FP32 packing
1e-9 (the same FP32 factors; factor elements below 2^-7 of their tile row's maximum are rounded
at 2^-32 of that maximum, about 1/100 of the FP32 rounding that the FP32 packing already
carries); of the FP32/FP16 split packing 1e-6 (the
tensor-core plan holds every column in FP32, the split packing its trailing ones in FP16);
vs the dense operator 1e-5 (the ACA tolerance).  Smooth inputs (the thin film's cancelling
far field) are checked as well as random ones.  Batches of 8 use the tensor cores; other sizes
fall back to the CUDA-core kernels for the remainder."""
import numpy as np
import pytest

from oracle import mesh as omesh

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu
DEV = "cuda"


def rel_rows(A, B):
    return [float(torch.linalg.norm(A[r] - B[r]) / torch.linalg.norm(B[r])) for r in range(A.shape[0])]


@pytest.mark.parametrize("nx,prec", [(48, "f32"), (100, "f32"), (100, "f32_f16")])
def test_tensor_core_matmat_vs_single(nx, prec):
    import spinfemx_b200 as spx
    X, T = omesh.kuhn_box(nx, nx, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5), precision=prec)
    g = torch.Generator(device=DEV).manual_seed(5)
    Xs = torch.randn(8, H.size, dtype=torch.float64, device=DEV, generator=g)
    Ys = torch.stack([H.matvec(Xs[r].contiguous()) for r in range(8)])
    assert H.enable_tensor_cores() > 0
    Yt = H.matmat(Xs)
    torch.cuda.synchronize()
    assert H.tensor_core_status() == 0
    tol = 1e-9 if prec == "f32" else 1e-6
    assert max(rel_rows(Yt, Ys)) < tol
    # smooth states: constants and long waves over the film
    xb = torch.linspace(0.0, 1.0, H.size, dtype=torch.float64, device=DEV)
    Sm = torch.stack([torch.ones_like(xb), torch.cos(6.283 * xb), xb, 1.0 + 0.1 * xb * xb,
                      torch.sin(3.14 * xb) ** 2, torch.cos(12.566 * xb) + 2.0, 1.0 - xb, torch.exp(-xb)])
    Ysm = torch.stack([H.matvec(Sm[r].contiguous()) for r in range(8)])
    assert max(rel_rows(H.matmat(Sm), Ysm)) < tol
    if nx == 48:
        B = geom.dense_B()
        assert max(rel_rows(Yt, (B @ Xs.T).T)) < 1e-5
    # 11 states: one batch of 8 on the tensor cores, the rest on the CUDA cores
    X11 = torch.randn(11, H.size, dtype=torch.float64, device=DEV, generator=g)
    Y11 = H.matmat(X11)
    Y11s = torch.stack([H.matvec(X11[r].contiguous()) for r in range(11)])
    assert max(rel_rows(Y11, Y11s)) < tol
    # repeatable and switchable
    assert torch.equal(H.matmat(Xs), Yt)
    H.enable_tensor_cores(False)
    assert max(rel_rows(H.matmat(Xs), Ys)) < 1e-9 if prec == "f32" else True


def test_tensor_core_autotune_keeps_results():
    import spinfemx_b200 as spx
    X, T = omesh.kuhn_box(60, 60, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5), precision="f32")
    g = torch.Generator(device=DEV).manual_seed(9)
    Xs = torch.randn(8, H.size, dtype=torch.float64, device=DEV, generator=g)
    Ys = torch.stack([H.matvec(Xs[r].contiguous()) for r in range(8)])
    H.enable_tensor_cores("auto")          # keeps the fastest of three paths
    assert H.tensor_core_status() == 0
    assert max(rel_rows(H.matmat(Xs), Ys)) < 1e-9
