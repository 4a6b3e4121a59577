"""GPU parity: libspx kernels through the C ABI against the oracle and the reference fixtures.

Tolerances (relative unless stated):
  Lindholm weights / dense B           1e-12 (FP64 kernels, rounding only)
  H-matrix partition                   bit-exact (ranks within 3 of the reference's on <10% of blocks)
  H-matrix apply vs reference H (FP64) 1e-6 ; vs dense B 1e-5 (the ACA tolerance)
  demag, dense FP64, tight CG          1e-9 ; reference CG tolerance (rtol 1e-6) 1e-5
  demag, H-matrix FP64                 1e-5
  LLG field / RHS / Jv / PC (FP64)     1e-11
  RK4 trajectory (FP64, 20x20x5 box, 200 steps of 10 fs)   max|dm| 1e-8
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from oracle import demag as odemag  # noqa: E402
from oracle import fem as ofem  # noqa: E402
from oracle import hmatrix as ohmat  # noqa: E402
from oracle import lindholm as olin  # noqa: E402
from oracle import llg as ollg  # noqa: E402
from oracle import mesh as omesh  # noqa: E402

DEV = "cuda"


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def spx():
    import spinfemx_b200
    return spinfemx_b200


@pytest.fixture(scope="module")
def box20(spx):
    X, T = omesh.kuhn_box(20, 20, 5, 2.0)
    return X, T, spx.BoundaryGeometry(X, T)


def test_lindholm_pairs_vs_reference(golden, box20, box20_bd):
    g = golden("lindholm_pairs.npz")
    _, _, geom = box20
    w = geom.lindholm_pairs(torch.as_tensor(g["x0"], device=DEV),
                            torch.as_tensor(g["tri"], device=DEV)).cpu().numpy()
    assert np.abs(w - g["w"]).max() <= 1e-12 * np.abs(g["w"]).max()


def test_dense_B_vs_reference(golden, box20):
    g = golden("box20_dense.npz")
    _, _, geom = box20
    B = geom.dense_B()
    Bh = B.cpu().numpy()
    assert np.abs(Bh[g["sample_rows"]] - g["B_rows"]).max() < 1e-13
    assert np.abs(Bh.sum(1) - g["rowsum"]).max() < 1e-12
    Bx = np.stack([geom_apply(B, g["x"][:, k]) for k in range(3)], 1)
    assert np.abs(Bx - g["Bx"]).max() < 1e-11 * np.abs(g["Bx"]).max()


def geom_apply(B, x):
    import spinfemx_b200 as spx
    xt = torch.as_tensor(np.ascontiguousarray(x), device=DEV)
    return spx.dense_b_apply(B, xt).cpu().numpy()


def test_fill_block_vs_oracle(box20, box20_bd):
    _, _, geom = box20
    rng = np.random.default_rng(11)
    rows = np.sort(rng.choice(1202, 300, replace=False)).astype(np.int32)
    cols = rng.choice(1202, 777, replace=False).astype(np.int32)
    got = geom.fill_block(torch.as_tensor(rows, device=DEV), torch.as_tensor(cols, device=DEV)).cpu().numpy()
    ref = olin.fill_block(box20_bd, rows, cols)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


CASES = {"box20": (20, 20, 5, 2.0), "film30": (30, 30, 2, 2.5), "film48": (48, 48, 2, 2.5)}


@pytest.mark.parametrize("name", list(CASES))
def test_hmatrix_build_vs_reference(spx, golden, name):
    g = golden(f"hmat_{name}.npz")
    X, T = omesh.kuhn_box(*CASES[name])
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5, eta=2.0, leaf_size=64), precision="f64")
    assert np.array_equal(H.perm, g["perm"])
    blocks = H.blocks()
    far = sorted(tuple(int(v) for v in b[[0, 1, 2, 3, 5]]) for b in blocks if b[4] == 1)
    ref = sorted(tuple(int(v) for v in r) for r in g["far"])
    assert [f[:4] for f in far] == [r[:4] for r in ref]
    dr = np.array([a[4] - b[4] for a, b in zip(far, ref)])
    assert np.abs(dr).max() <= 3 and np.count_nonzero(dr) <= 0.1 * len(far)
    st = H.stats()
    assert [st["dense_blocks"], st["low_rank_blocks"], st["rejected_low_rank_blocks"],
            st["forced_subdivisions_memory"], st["compression_tolerance_subdivisions"]] == g["stats"][:5].tolist()
    # near tiles are stored dense; the reference's near CSR drops exact zeros (coplanar
    # point/triangle pairs give zero Lindholm weights), so only the tile area bounds its nnz
    near_entries = sum(int((b[1] - b[0]) * (b[3] - b[2])) for b in blocks if b[4] == 0)
    assert near_entries >= int(g["near_nnz"])
    Hx = np.stack([H.matvec(torch.as_tensor(g["x"][:, k].copy(), device=DEV)).cpu().numpy() for k in range(3)], 1)
    assert rel(Hx, g["Hx"]) < 1e-6
    # against the dense operator: within the ACA tolerance
    B = geom.dense_B().cpu().numpy()
    assert rel(Hx, B @ g["x"]) < 1e-5


def test_hmatrix_long_rows_vs_dense(spx):
    """A film whose partition has far blocks wider than one k_far_z column piece (1024
    columns): every packed precision against the dense operator, bitwise-repeatable
    applies, and the no-allocation entry point equal to the allocating one."""
    X, T = omesh.kuhn_box(100, 100, 2, 2.5)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5), precision="f64")
    b = H.blocks()
    far = b[b[:, 4] == 1]
    assert (far[:, 3] - far[:, 2]).max() > 1024
    g = torch.Generator(device=DEV).manual_seed(7)
    x = torch.randn(H.size, dtype=torch.float64, device=DEV, generator=g)
    B = geom.dense_B()
    yd = B @ x
    del B
    torch.cuda.empty_cache()
    for prec, tol in (("f64", 1e-5), ("f32", 1e-5), ("mixed", 1e-3)):
        H.repack(prec)
        y1 = H.matvec(x).clone()
        y2 = H.matvec(x).clone()
        assert torch.equal(y1, y2)
        assert float(torch.linalg.norm(y1 - yd) / torch.linalg.norm(yd)) < tol, prec
        yn = torch.empty_like(x)
        H.matvec_noalloc(x, yn)
        assert torch.equal(yn, y1)


def test_hmatrix_reduced_precisions(spx, golden):
    g = golden("hmat_film48.npz")
    X, T = omesh.kuhn_box(*CASES["film48"])
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-5), precision="f64")
    x = torch.as_tensor(g["x"][:, 0].copy(), device=DEV)
    y64 = H.matvec(x).cpu().numpy()
    H.repack("f32")
    y32 = H.matvec(x).cpu().numpy()
    H.repack("mixed")
    ymx = H.matvec(x).cpu().numpy()
    assert rel(y32, y64) < 1e-6
    assert rel(ymx, y64) < 3e-3
    ones = torch.ones(H.size, dtype=torch.float64, device=DEV)
    H.repack("f64")
    assert np.abs(H.matvec(ones).cpu().numpy() + 1.0).max() < 1e-2


@pytest.fixture(scope="module")
def box20_oracle():
    X, T = omesh.kuhn_box(20, 20, 5, 2.0)
    return odemag.DemagOracle(X, T, 8e5)


def _m0(N, seed=1000):
    rng = np.random.default_rng(seed)
    m = np.tile(np.array([1.0, 1.0, 1.0]) / math.sqrt(3.0), (N, 1)) + rng.normal(0.0, 0.1, (N, 3))
    m /= np.linalg.norm(m, axis=1)[:, None]
    return m.ravel()


def test_demag_dense_vs_oracle(spx, box20_oracle):
    o = box20_oracle
    m = _m0(o.N)
    Href, u1r, u2r, _ = o.compute(m, return_parts=True)
    mt = torch.as_tensor(m, device=DEV)
    out = torch.empty_like(mt)
    d = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, boundary_backend="dense", ksp_rtol_u1=1e-13,
                                  ksp_rtol_u2=1e-13, ksp_atol=0.0, ksp_maxit_u1=20000, ksp_maxit_u2=20000)
    d.compute_vec(mt, out)
    assert rel(out.cpu().numpy(), Href) < 1e-9
    u1, u2 = d.potentials()
    assert rel(u1.cpu().numpy(), u1r) < 1e-9
    assert rel(u2.cpu().numpy(), u2r) < 1e-9
    E = d.Energy_lumped_gpu(mt, out)
    assert abs(E / o.energy(m, Href) - 1.0) < 1e-9
    assert all(d.Energy_lumped_gpu(mt, out) == E for _ in range(3))  # fixed-order reduction
    # the reference's own CG tolerance (rtol 1e-6)
    d6 = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, boundary_backend="dense")
    d6.compute_vec(mt, out)
    assert rel(out.cpu().numpy(), Href) < 1e-5
    assert d6.last_its_u1 > 0 and d6.last_res_u1 <= 1e-6


def test_demag_hmatrix_vs_oracle(spx, box20_oracle):
    o = box20_oracle
    m = _m0(o.N)
    Href = o.compute(m)
    mt = torch.as_tensor(m, device=DEV)
    out = torch.empty_like(mt)
    d = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, boundary_backend="hmatrix", hmatrix_epsilon=1e-5,
                                  ksp_rtol_u1=1e-12, ksp_rtol_u2=1e-12, ksp_atol=0.0, ksp_maxit_u1=20000)
    d.compute_vec(mt, out)
    assert rel(out.cpu().numpy(), Href) < 1e-5
    assert d.B_hmatrix_gpu.stats()["n_far"] > 0


def test_demag_fp32_vs_oracle(spx, box20_oracle):
    o = box20_oracle
    m = _m0(o.N)
    Href = o.compute(m)
    mt = torch.as_tensor(m, device=DEV)
    out = torch.empty_like(mt)
    d = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, boundary_backend="dense", precision="f32")
    d.compute_vec(mt, out)
    assert rel(out.cpu().numpy(), Href) < 2e-5


def _small_problem(with_demag):
    X, T = omesh.kuhn_box(10, 8, 3, 2.0)
    N = X.shape[0]
    rng = np.random.default_rng(5)
    m = rng.normal(size=(N, 3))
    m /= np.linalg.norm(m, axis=1)[:, None]
    nz = np.tile([0.0, 0.0, 1.0], N)
    nani = rng.normal(size=(N, 3))
    kw = dict(Ms=1.1e6, Aex=1.6e-11, Ku=8e5, D_int=3e-3, alpha=0.3)
    H0 = np.tile([1e4, -2e4, 3e5], N)
    demag = odemag.DemagOracle(X, T, kw["Ms"]) if with_demag else None
    ohef = ollg.EffectiveFieldOracle(X, T, kw["Ms"], Aex=kw["Aex"], Ku=kw["Ku"], n_ani=nani, D_int=kw["D_int"],
                                     n_int=nz, H0=H0, demag=demag, alpha=kw["alpha"])
    return X, T, m.ravel(), nz, nani, H0, kw, ohef


@pytest.mark.parametrize("with_demag", [False, True])
def test_llg_field_rhs_jv_pc_vs_oracle(spx, with_demag):
    X, T, m, nz, nani, H0, kw, ohef = _small_problem(with_demag)
    dk = dict(boundary_backend="dense", ksp_rtol_u1=1e-13, ksp_rtol_u2=1e-13, ksp_atol=0.0, ksp_maxit_u1=20000)
    hef = spx.EffectiveField(X, T, kw["Ms"], Aex=kw["Aex"], Ku=kw["Ku"], n_ani_vec=nani, D_int=kw["D_int"],
                             n0_int_vec=nz, alpha=kw["alpha"], H0_static=H0, use_demag=with_demag, demag_kwargs=dk)
    mt = torch.as_tensor(m, device=DEV)
    out = torch.empty_like(mt)
    hef.compute_H_eff_vec(mt, out)
    assert rel(out.cpu().numpy(), ohef.h_eff(m)) < (1e-9 if with_demag else 1e-12)
    hef.llg_rhs_vec(mt, out)
    assert rel(out.cpu().numpy(), ohef.llg_rhs(m)) < (1e-9 if with_demag else 1e-12)
    # Jacobian state and Jv (demag excluded)
    hef.update_jac_state(mt)
    Hm = ohef.h_jac(m)
    v = np.random.default_rng(9).normal(size=m.size)
    vt = torch.as_tensor(v, device=DEV)
    hef.jac_vec_times_vec(vt, out)
    Hv = ohef.linear(v)
    ref = ollg.jv(m, Hm, v, Hv, hef.gamma, hef.alpha, 1.0, ohef.stab)
    assert rel(out.cpu().numpy(), ref) < 1e-11
    hef.apply_jacobian_field_vec(mt, vt, out)
    assert rel(out.cpu().numpy(), Hv) < 1e-11
    # block preconditioner
    ctx = spx.JvContext(hef)
    shift = 3e11
    ctx.update_pc_full_fast_gpu(shift)
    y = torch.empty_like(vt)
    ctx.apply(None, vt, y)
    c1 = hef.gamma / (1 + hef.alpha ** 2)
    c2 = hef.gamma * hef.alpha / (1 + hef.alpha ** 2)
    inv = ollg.pc_build(m, Hm, ohef.diagK, shift, c1, c2, ohef.stab)
    assert rel(y.cpu().numpy(), ollg.pc_apply(inv, v)) < 1e-11
    ctx.mult(None, vt, y)
    assert rel(y.cpu().numpy(), shift * v - ref) < 1e-11


def test_rk4_trajectory_box20_vs_oracle(spx, box20_oracle):
    # the small-box workload: 20x20x5 box (2 nm cubes), dense FP64 demag + exchange,
    # alpha 0.5, 200 fixed steps of 10 fs from the seeded (1,1,1)/sqrt(3) + N(0, 0.1^2) state
    o = box20_oracle
    m0 = _m0(o.N)
    ohef = ollg.EffectiveFieldOracle(o.X, o.tets, 8e5, Aex=1.3e-11, alpha=0.5, demag=o)
    nsteps = 200
    m = m0.copy()
    for _ in range(nsteps):
        m = ollg.rk4_step(ohef.llg_rhs, m, 1e-14)
    llg = spx.LLG_GPU(o.X, o.tets, 8e5, alpha=0.5)
    llg.add_exchange(1.3e-11)
    llg.add_demag(boundary_backend="dense", ksp_rtol_u1=1e-13, ksp_rtol_u2=1e-13, ksp_atol=0.0,
                  ksp_maxit_u1=20000)
    mg = llg.run_fixed(m0, 1e-14, nsteps).cpu().numpy()
    assert np.abs(mg - m).max() < 1e-8
    # end-to-end host call gives the same trajectory
    hm = llg.hef.run_host(m0.copy(), 1e-14, nsteps)
    assert np.abs(hm - mg).max() < 1e-12


def test_cg_iteration_cap_reports_not_converged(spx, box20_oracle):
    o = box20_oracle
    mt = torch.as_tensor(_m0(o.N), device=DEV)
    out = torch.empty_like(mt)
    d = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, ksp_maxit_u1=3)
    d.compute_vec(mt, out)
    assert d.last_its_u1 == 3 and d.last_res_u1 > 1e-6


def test_demag_mixed_vs_oracle(spx, box20_oracle):
    # FP64 vectors, FP32 matrices, FP32 CG inside FP64 refinement, difference-form operators
    o = box20_oracle
    m = _m0(o.N)
    Href = o.compute(m)
    mt = torch.as_tensor(m, device=DEV)
    out = torch.empty_like(mt)
    d = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, boundary_backend="dense", precision="mixed",
                                  ksp_rtol_u1=1e-10, ksp_rtol_u2=1e-10, ksp_atol=0.0, ksp_maxit_u1=20000)
    d.compute_vec(mt, out)
    assert rel(out.cpu().numpy(), Href) < 1e-7
    d6 = spx.DemagFieldLindholmGPU(o.X, o.tets, 8e5, boundary_backend="dense", precision="mixed")
    d6.compute_vec(mt, out)
    assert rel(out.cpu().numpy(), Href) < 1e-5


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_rk4_extrapolated_starts_vs_oracle(spx, box20_oracle, precision):
    # per-RK-stage extrapolated CG starts change iteration counts, not the trajectory
    o = box20_oracle
    m0 = _m0(o.N)
    ohef = ollg.EffectiveFieldOracle(o.X, o.tets, 8e5, Aex=1.3e-11, alpha=0.5, demag=o)
    nsteps = 12
    m = m0.copy()
    for _ in range(nsteps):
        m = ollg.rk4_step(ohef.llg_rhs, m, 1e-14)
    hef = spx.EffectiveField(o.X, o.tets, 8e5, Aex=1.3e-11, alpha=0.5, use_demag=True,
                             demag_kwargs=dict(boundary_backend="dense", ksp_rtol_u1=1e-11, ksp_rtol_u2=1e-11,
                                               ksp_atol=0.0, ksp_maxit_u1=20000, precision=precision,
                                               warm_start="extrapolate"))
    hef.set_state(torch.as_tensor(m0, device=DEV))
    hef.step(1e-14, nsteps)
    mg = hef.get_state().cpu().numpy()
    assert np.abs(mg - m).max() < (1e-8 if precision == "f64" else 1e-7)
