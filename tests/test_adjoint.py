"""Adjoint and tangent products: the oracle's restatement against its own finite
differences and duality identities (CPU), then the CUDA path against the oracle (GPU).

The reference has no adjoint, so there is no reference output to pin: the oracle's adjoint
(oracle/adjoint.py) is pinned by central finite differences of the oracle's FP64 forward
pipeline and by <w, J v> = <J^T w, v>, and the CUDA adjoint is compared with it.
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import adjoint as oadj
from oracle import demag as odemag
from oracle import lindholm
from oracle import llg as ollg
from oracle import mesh as omesh


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _unit(rng, N):
    m = rng.normal(size=(N, 3)) + np.array([1.0, 0.3, 0.2])
    return (m / np.linalg.norm(m, axis=1)[:, None]).ravel()


def _problem(nx=5, ny=4, nz=2, h=2.0, seed=11):
    X, T = omesh.kuhn_box(nx, ny, nz, h)
    N = X.shape[0]
    rng = np.random.default_rng(seed)
    nani = np.tile([0.1, 0.2, 1.0], (N, 1)) + 0.2 * rng.normal(size=(N, 3))
    Ku = 3e5 + 1e5 * rng.random(N)
    nz_ = np.tile([0.0, 0.0, 1.0], N)
    kw = dict(Ms=8e5, Aex=1.3e-11, D_int=2e-3, alpha=0.1)
    H0 = np.array([2e4, 4e4, -1e4])
    D = odemag.DemagOracle(X, T, kw["Ms"])
    F = ollg.EffectiveFieldOracle(X, T, kw["Ms"], Aex=kw["Aex"], Ku=Ku, n_ani=nani, D_int=kw["D_int"], n_int=nz_,
                                  H0=np.tile(H0, N), demag=D, alpha=kw["alpha"])
    return dict(X=X, T=T, N=N, nani=nani, Ku=Ku, nz=nz_, H0=H0, kw=kw, D=D, F=F, m=_unit(rng, N), rng=rng)


@pytest.fixture(scope="module")
def prob():
    return _problem()


# ------------------------------------------------------------------ oracle (CPU)
def test_oracle_demag_transpose_duality(prob):
    D, rng = prob["D"], np.random.default_rng(1)
    n3 = 3 * prob["N"]
    w, v = rng.normal(size=n3), rng.normal(size=n3)
    lhs = w @ D.compute(v)
    rhs = oadj.demag_transpose(D, w) @ v
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_oracle_rhs_vjp_duality_and_fd(prob):
    F, m, rng = prob["F"], prob["m"], np.random.default_rng(2)
    n3, N = 3 * prob["N"], prob["N"]
    w, v = rng.normal(size=n3), rng.normal(size=n3) * 1e-2
    dKu = rng.normal(size=N) * 1e4
    dH0 = np.array([3e3, -1e3, 2e3])
    a, gKu, gH0 = oadj.rhs_vjp(F, m, w)
    jv = oadj.rhs_jvp(F, m, v)
    assert abs(w @ jv - a @ v) <= 1e-11 * abs(w @ jv)
    jk = oadj.rhs_jvp(F, m, np.zeros(n3), dKu=dKu)
    assert abs(w @ jk - gKu @ dKu) <= 1e-11 * abs(w @ jk)
    jh = oadj.rhs_jvp(F, m, np.zeros(n3), dH0=dH0)
    assert abs(w @ jh - gH0 @ dH0) <= 1e-11 * abs(w @ jh)
    # tangent against central differences of the RHS
    eps = 1e-4
    fd = (F.llg_rhs(m + eps * v) - F.llg_rhs(m - eps * v)) / (2 * eps)
    assert rel(jv, fd) < 1e-7


def _loss_and_target(prob, nsteps, dt):
    F = prob["F"]
    mt = oadj.trajectory(F, _unit(np.random.default_rng(99), prob["N"]), dt, nsteps)[-1]
    return (lambda mT: float(np.sum((mT - mt) ** 2))), (lambda mT: 2.0 * (mT - mt))


def test_oracle_trajectory_gradient_vs_central_fd(prob):
    F, m0, N = prob["F"], prob["m"], prob["N"]
    nsteps, dt = 6, 2e-14
    L, dL = _loss_and_target(prob, nsteps, dt)
    Ku0, H00 = prob["Ku"].copy(), prob["H0"].copy()
    oadj.set_params(F, Ku0, H00)
    mT = oadj.trajectory(F, m0, dt, nsteps)[-1]
    gm, gKu, gH0 = oadj.trajectory_grad(F, m0, dt, nsteps, dL(mT))
    rng = np.random.default_rng(5)
    dirs = [("Ku", rng.normal(size=N) * Ku0), ("H0", rng.normal(size=3) * 1e4), ("m0", rng.normal(size=3 * N))]
    for name, d in dirs:
        h = 1e-4
        vals = []
        for sgn in (1.0, -1.0):
            Ku, H0, m = Ku0, H00, m0
            if name == "Ku":
                Ku = Ku0 + sgn * h * d
            elif name == "H0":
                H0 = H00 + sgn * h * d
            else:
                m = m0 + sgn * h * d
            oadj.set_params(F, Ku, H0)
            vals.append(L(oadj.trajectory(F, m, dt, nsteps)[-1]))
        oadj.set_params(F, Ku0, H00)
        fd = (vals[0] - vals[1]) / (2 * h)
        g = {"Ku": gKu, "H0": gH0, "m0": gm}[name] @ d
        assert abs(g - fd) <= 1e-6 * abs(fd), name


# ------------------------------------------------------------------ CUDA path (GPU)
torch = pytest.importorskip("torch")
DEV = "cuda"
TIGHT = dict(ksp_rtol_u1=1e-13, ksp_rtol_u2=1e-13, ksp_atol=0.0, ksp_maxit_u1=20000, ksp_maxit_u2=20000)


@pytest.fixture(scope="module")
def spx():
    import spinfemx_b200 as spx
    return spx


def _gpu_field(spx, prob, backend="dense", **extra):
    kw = prob["kw"]
    dk = dict(boundary_backend=backend, **TIGHT)
    dk.update(extra)
    return spx.EffectiveField(prob["X"], prob["T"], kw["Ms"], Aex=kw["Aex"], Ku=0.0, Ku_nodes=prob["Ku"],
                              n_ani_vec=prob["nani"], D_int=kw["D_int"], n0_int_vec=prob["nz"], alpha=kw["alpha"],
                              H0_static=prob["H0"], use_demag=True, demag_kwargs=dk)


def _t(x):
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=DEV)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_hmat_transpose_apply(spx, precision):
    X, T = omesh.kuhn_box(16, 12, 3, 2.0)
    geom = spx.BoundaryGeometry(X, T)
    H = spx.HMatrixGPUPackedFused(geom, spx.HMatrixBuildConfig(epsilon=1e-6, eta=2.0, leaf_size=16),
                                  precision=precision)
    rng = np.random.default_rng(3)
    x, y = rng.normal(size=geom.Nb), rng.normal(size=geom.Nb)
    Hx = H.matvec(_t(x)).cpu().numpy()
    HTy = H.rmatvec(_t(y)).cpu().numpy()
    # the transposed operator is the exact transpose of the stored one
    assert abs(y @ Hx - HTy @ x) <= 1e-12 * np.linalg.norm(y) * np.linalg.norm(Hx)
    B = lindholm.dense_B(lindholm.boundary_data(X, T))
    assert rel(HTy, B.T @ y) < (1e-5 if precision == "f64" else 1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("backend,warm_start", [("dense", False), ("hmatrix", False),
                                                ("dense", "extrapolate_corrected")])
def test_demag_transpose_vs_oracle(spx, prob, backend, warm_start):
    D = prob["D"]
    kw = dict(boundary_backend=backend, precision="f64", warm_start=warm_start, **TIGHT)
    if backend == "hmatrix":
        kw.update(hmatrix_epsilon=1e-8, hmatrix_leaf_size=8)
    d = spx.DemagFieldLindholmGPU(prob["X"], prob["T"], prob["kw"]["Ms"], **kw)
    rng = np.random.default_rng(4)
    n3 = 3 * prob["N"]
    w, v = rng.normal(size=n3), rng.normal(size=n3)
    out = torch.empty(n3, dtype=torch.float64, device=DEV)
    d.compute_vec_transpose(_t(w), out)
    g = out.cpu().numpy()
    assert rel(g, oadj.demag_transpose(D, w)) < (1e-9 if backend == "dense" else 1e-6)
    Hv = torch.empty_like(out)
    d.compute_vec(_t(v), Hv)
    d.compute_vec_transpose(_t(w), out)  # after a forward solve of another scale
    assert rel(out.cpu().numpy(), g) < 1e-9
    lhs = w @ Hv.cpu().numpy()
    assert abs(lhs - g @ v) <= 1e-9 * abs(lhs)


@pytest.mark.gpu
def test_rhs_vjp_vs_oracle(spx, prob):
    F, m = prob["F"], prob["m"]
    N = prob["N"]
    hef = _gpu_field(spx, prob)
    w = np.random.default_rng(6).normal(size=3 * N)
    out = torch.empty(3 * N, dtype=torch.float64, device=DEV)
    gKu = torch.zeros(N, dtype=torch.float64, device=DEV)
    gH0 = torch.zeros(3, dtype=torch.float64, device=DEV)
    hef.rhs_vjp(_t(m), _t(w), out, gKu, gH0)
    a, rKu, rH0 = oadj.rhs_vjp(F, m, w)
    assert rel(out.cpu().numpy(), a) < 1e-9
    assert rel(gKu.cpu().numpy(), rKu) < 1e-9
    assert rel(gH0.cpu().numpy(), rH0) < 1e-9


@pytest.mark.gpu
def test_step_vjp_and_jvp_vs_oracle(spx, prob):
    F, m = prob["F"], prob["m"]
    N, dt = prob["N"], 2e-14
    hef = _gpu_field(spx, prob)
    rng = np.random.default_rng(7)
    lam = rng.normal(size=3 * N)
    lo = torch.empty(3 * N, dtype=torch.float64, device=DEV)
    gKu = torch.zeros(N, dtype=torch.float64, device=DEV)
    gH0 = torch.zeros(3, dtype=torch.float64, device=DEV)
    hef.step_vjp(_t(m), dt, _t(lam), lo, gKu, gH0)
    rl, rKu, rH0 = oadj.step_vjp(F, m, dt, lam)
    assert rel(lo.cpu().numpy(), rl) < 1e-9
    assert rel(gKu.cpu().numpy(), rKu) < 1e-9
    assert rel(gH0.cpu().numpy(), rH0) < 1e-9
    dm = rng.normal(size=3 * N) * 1e-2
    dKu = rng.normal(size=N) * 1e4
    dH0 = np.array([1e3, 2e3, -3e3])
    mo, dmo = torch.empty_like(lo), torch.empty_like(lo)
    hef.step_jvp(_t(m), _t(dm), dt, mo, dmo, _t(dKu), dH0)
    rm, rdm = oadj.step_jvp(F, m, dm, dt, dKu, dH0)
    assert rel(mo.cpu().numpy(), rm) < 1e-12
    assert rel(dmo.cpu().numpy(), rdm) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("warm_start,precision", [(False, "f64"), ("extrapolate_corrected", "f64"),
                                                  ("extrapolate_corrected", "mixed")])
def test_trajectory_gradient_vs_oracle_fd_and_tangent(spx, prob, warm_start, precision):
    """Gradients of ||m(T) - m_target||^2 through the autograd Function (checkpoints every 3 of
    8 steps) against central finite differences of the FP64 oracle (h = 1e-4 relative),
    and against the CUDA tangent.  Warm-started solves keep separate states for the forward,
    adjoint and tangent solves (their right-hand sides differ in scale by many orders)."""
    F, m0, N = prob["F"], prob["m"], prob["N"]
    nsteps, dt = 8, 2e-14
    L, _ = _loss_and_target(prob, nsteps, dt)
    mt = oadj.trajectory(F, _unit(np.random.default_rng(99), N), dt, nsteps)[-1]
    Ku0, H00 = prob["Ku"].copy(), prob["H0"].copy()
    tight = precision == "f64"
    hef = _gpu_field(spx, prob, warm_start=warm_start, precision=precision,
                     **({} if tight else dict(ksp_rtol_u1=1e-11, ksp_rtol_u2=1e-11)))
    m0t = _t(m0).requires_grad_(True)
    Kut = _t(Ku0).requires_grad_(True)
    H0t = _t(H00).requires_grad_(True)
    mT = spx.llg_trajectory(hef, m0t, dt, nsteps, Ku=Kut, H0=H0t, checkpoint_every=3)
    loss = torch.sum((mT - _t(mt)) ** 2)
    loss.backward()
    oadj.set_params(F, Ku0, H00)
    assert abs(loss.item() - L(oadj.trajectory(F, m0, dt, nsteps)[-1])) <= (1e-9 if tight else 1e-6) * loss.item()
    rng = np.random.default_rng(8)
    dirs = {"Ku": rng.normal(size=N) * Ku0, "H0": rng.normal(size=3) * 1e4, "m0": rng.normal(size=3 * N)}
    grads = {"Ku": Kut.grad.cpu().numpy(), "H0": H0t.grad.cpu().numpy(), "m0": m0t.grad.cpu().numpy()}
    h = 1e-4
    for name, d in dirs.items():
        vals = []
        for sgn in (1.0, -1.0):
            Ku, H0, m = Ku0, H00, m0
            if name == "Ku":
                Ku = Ku0 + sgn * h * d
            elif name == "H0":
                H0 = H00 + sgn * h * d
            else:
                m = m0 + sgn * h * d
            oadj.set_params(F, Ku, H0)
            vals.append(L(oadj.trajectory(F, m, dt, nsteps)[-1]))
        oadj.set_params(F, Ku0, H00)
        fd = (vals[0] - vals[1]) / (2 * h)
        g = grads[name] @ d
        assert abs(g - fd) <= 1e-4 * abs(fd), (name, g, fd)
        # forward-mode tangent of the same trajectory
        kw = {"Ku": dict(dKu=d), "H0": dict(dH0=d), "m0": dict(dm0=d)}[name]
        mT2, dmT = spx.trajectory_tangent(hef, m0, dt, nsteps, Ku=Ku0, H0=H00, **kw)
        tan = float(torch.sum(2.0 * (mT2 - _t(mt)) * dmT).item())
        assert abs(tan - g) <= (1e-8 if tight else 1e-6) * abs(g), (name, tan, g)
