"""Generate the golden fixtures in this folder from the reference itself.

Run in a container that has the reference checkout and numba:

    python tests/golden/make_golden.py

Each fixture holds seeded inputs and the outputs of the REFERENCE's own code:

* ``lindholm_pairs.npz``  gpu/fields/Lindholm_kernel.py (numba) weights and
  solid angles for random (target, triangle) pairs of the 20x20x5 box (2 nm cubes).
* ``box20_dense.npz``  lindholm_hmatrix_gpu/entry_provider.py
  ``LindholmEntryProviderCPU.fill_block(all, all)`` + diag jump: row sums,
  B @ x for seeded x, sample rows.
* ``trees.npz``  lindholm_hmatrix_gpu/tree.py permutations.
* ``hmat_<case>.npz``  lindholm_hmatrix_gpu/builder.py ``HMatrixBuilder``
  (CPU, full-pivot ACA): block partition, ranks, near nnz, H @ x.
* ``hcache_film14.npz``  the reference's own npz cache (``HMatrixCPUData.save``,
  storage.py:72-149) of a 14x14x2 film H-matrix (eps 1e-4, leaf 16), for the cache reader.
* ``c2_rows.npz``  4,096 seeded boundary rows of the dense operator of the 400x400x2 film
  (2.5 nm cubes, Nb = 323,202): ``LindholmEntryProviderCPU.fill_block(rows, all)`` plus the
  diagonal jump, applied to three vectors defined by ``c2_row_vectors`` (random, smooth
  in-plane, linear through the thickness); stores the row sums and B[rows] @ x.  About two
  minutes on 8 cores (``python tests/golden/make_golden.py c2_rows``).
* ``example_chain_mesh.npz``  the reference's octahedral-nanoparticle chain example mesh
  (examples/cpu/hysteresis_octahedral_nanoparticles/chain.xdmf + .h5) read by spinfemx_b200.io.
* ``torque_kernels.npz``  the reference's STT / SOT per-node kernel bodies
  (llg_stt_module_GPU.py, llg_SOT_module_GPU.py) compiled the same way.
* ``llg_kernels.npz``  the reference's per-node CUDA-C kernel bodies compiled
  with gcc by ``oracle/ref_build.py`` plus the CPU numba Jv kernel.

Boundary geometry comes from the oracle restatement (the reference's own
``build_boundary_data_serial`` needs DOLFINx); it is deterministic and shared
by the oracle and the product.
"""
from __future__ import annotations

import math
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import lindholm, mesh, ref_build  # noqa: E402

OUT = Path(__file__).resolve().parent
REF_EXAMPLES = ref_build.REF_ROOT.parents[1] / "examples"

CASES = {
    # name: (nx, ny, nz, h)
    "box20": (20, 20, 5, 2.0),
    "film30": (30, 30, 2, 2.5),
    "film48": (48, 48, 2, 2.5),
}


def provider_for(mods, bd):
    ep = mods["entry_provider"]
    return ep.LindholmEntryProviderCPU(
        Xb=bd["Xb"], tri_lid=bd["tri_lid"], tri_pts=bd["tri_pts"], ntri=bd["ntri"],
        area=bd["area"], s_edge=bd["s_edge"], eta=bd["eta"], gamma=bd["gamma"],
        incident_policy=0)


def make_lindholm_pairs(mods, bd):
    rng = np.random.default_rng(1001)
    lk = mods["Lindholm_kernel"]
    P = 3000
    Nb, Nt = bd["Xb"].shape[0], bd["tri_lid"].shape[0]
    rows = rng.integers(0, Nb, P)
    tri = rng.integers(0, Nt, P)
    x0 = bd["Xb"][rows].copy()
    # a third of the targets are perturbed off the surface (general position)
    x0[: P // 3] += rng.normal(0, 0.7, (P // 3, 3))
    w = np.empty((P, 3))
    om = np.empty(P)
    for k in range(P):
        t = tri[k]
        w[k] = lk.lindholm_weights_precomp(x0[k], bd["tri_pts"][t, 0], bd["tri_pts"][t, 1],
                                           bd["tri_pts"][t, 2], bd["ntri"][t], bd["area"][t],
                                           bd["s_edge"][t], bd["eta"][t], bd["gamma"][t])
        om[k] = lk.solid_angle_with_atan2(x0[k], bd["tri_pts"][t, 0], bd["tri_pts"][t, 1],
                                          bd["tri_pts"][t, 2])
    np.savez_compressed(OUT / "lindholm_pairs.npz", x0=x0, tri=tri.astype(np.int32), w=w, omega=om)


def make_dense(mods, bd):
    prov = provider_for(mods, bd)
    Nb = bd["Xb"].shape[0]
    idx = np.arange(Nb, dtype=np.int32)
    B = prov.fill_block(idx, idx)
    B[idx, idx] += bd["omega_sum"] / (4.0 * math.pi) - 1.0
    rng = np.random.default_rng(1002)
    X = rng.standard_normal((Nb, 3))
    sample = np.sort(rng.choice(Nb, 24, replace=False))
    np.savez_compressed(OUT / "box20_dense.npz", rowsum=B.sum(axis=1), x=X, Bx=B @ X,
                        sample_rows=sample.astype(np.int32), B_rows=B[sample],
                        omega_sum=bd["omega_sum"])


def make_trees(mods, cases_bd):
    tr = mods["tree"]
    out = {}
    for name, bd in cases_bd.items():
        for leaf in (16, 32, 64):
            t = tr.build_cluster_tree(bd["Xb"], leaf_size=leaf)
            out[f"{name}_leaf{leaf}"] = t.perm
    np.savez_compressed(OUT / "trees.npz", **out)


def make_hmatrix(mods, name, bd, eps=1e-5, eta=2.0, leaf=64):
    bl = mods["builder"]
    prov = provider_for(mods, bd)
    dj = bd["omega_sum"] / (4.0 * math.pi) - 1.0
    cfg = bl.HMatrixBuildConfig(epsilon=eps, eta=eta, leaf_size=leaf, compressor="fullaca",
                                build_backend="cpu")
    data = bl.HMatrixBuilder(bd["Xb"], dj, prov, cfg).build()
    far = np.array([(b.row_start, b.row_stop, b.col_start, b.col_stop, b.rank)
                    for b in data.far_blocks], dtype=np.int64).reshape(-1, 5)
    # the near-field block structure: recover dense blocks as the partition minus far
    rng = np.random.default_rng(1003)
    Nb = bd["Xb"].shape[0]
    X = rng.standard_normal((Nb, 3))
    HX = np.stack([data.matvec_cpu(X[:, k]) for k in range(3)], axis=1)
    meta = data.metadata
    np.savez_compressed(
        OUT / f"hmat_{name}.npz", perm=data.perm, far=far,
        far_relres=np.array([b.relative_residual for b in data.far_blocks]),
        near_nnz=np.int64(data.near_csr.nnz), near_rowptr=data.near_csr.indptr.astype(np.int64),
        x=X, Hx=HX, eps=eps, eta=eta, leaf=leaf,
        stats=np.array([meta["dense_blocks"], meta["low_rank_blocks"],
                        meta["rejected_low_rank_blocks"], meta["forced_subdivisions_memory"],
                        meta["compression_tolerance_subdivisions"], meta["max_observed_rank"],
                        meta["sum_observed_rank"]], dtype=np.int64),
        far_U0=(data.far_blocks[0].U if data.far_blocks else np.zeros((0, 0))),
        far_V0=(data.far_blocks[0].V if data.far_blocks else np.zeros((0, 0))))
    return data


CACHE_CASE = (14, 14, 2, 2.5)  # with eps 1e-4, eta 2, leaf 16


def make_cache(mods):
    """The reference's npz cache of an H-matrix, written by its own HMatrixCPUData.save."""
    X, T = mesh.kuhn_box(*CACHE_CASE)
    bd = lindholm.boundary_data(X, T)
    bl = mods["builder"]
    dj = bd["omega_sum"] / (4.0 * math.pi) - 1.0
    cfg = bl.HMatrixBuildConfig(epsilon=1e-4, eta=2.0, leaf_size=16, compressor="fullaca", build_backend="cpu")
    data = bl.HMatrixBuilder(bd["Xb"], dj, provider_for(mods, bd), cfg).build()
    data.save(OUT / "hcache_film14.npz", compressed=True)
    return data


def make_aca(mods):
    cp = mods["compressors"]
    rng = np.random.default_rng(1004)
    out = {}
    for k, (m, n, r) in enumerate([(40, 30, 5), (64, 64, 12), (33, 70, 70)]):
        A = rng.standard_normal((m, r)) @ rng.standard_normal((r, n))
        A += 1e-7 * rng.standard_normal((m, n))
        res = cp.fullaca_dense(A, rtol=1e-5)
        out[f"A{k}"] = A
        out[f"U{k}"] = res.U
        out[f"V{k}"] = res.V
        out[f"rel{k}"] = res.relative_residual
    np.savez_compressed(OUT / "aca.npz", **out)


def make_llg_kernels():
    ref = ref_build.RefElementwise(ref_build.build(force=True))
    rng = np.random.default_rng(1005)
    n = 257
    m = rng.normal(size=(n, 3))
    m[: n // 2] /= np.linalg.norm(m[: n // 2], axis=1)[:, None]
    H = rng.normal(size=(n, 3)) * 1e5
    v = rng.normal(size=(n, 3))
    Hv = rng.normal(size=(n, 3)) * 1e5
    D = rng.normal(size=(n, 3)) * 1e4
    Dc = rng.normal(size=(n, 3)) * 1e3
    nax = rng.normal(size=(n, 3))
    nax /= np.linalg.norm(nax, axis=1)[:, None]
    gamma, alpha, Ms = 2.211e5, 0.3, 8e5
    pref = -gamma / (1 + alpha ** 2)
    stab = Ms * gamma / (1 + alpha ** 2) * 0.5
    rhs = ref.call("_LLG_RHS_KERNEL", n, dict(mx=m[:, 0], my=m[:, 1], mz=m[:, 2], hx=H[:, 0],
                                               hy=H[:, 1], hz=H[:, 2], prefactor=pref,
                                               alpha=alpha, do_precess=1.0, Stab=stab))
    jv = ref.call("_JAC_VEC_KERNEL", n, dict(mx=m[:, 0], my=m[:, 1], mz=m[:, 2], hx=H[:, 0],
                                              hy=H[:, 1], hz=H[:, 2], vx=v[:, 0], vy=v[:, 1],
                                              vz=v[:, 2], hvx=Hv[:, 0], hvy=Hv[:, 1],
                                              hvz=Hv[:, 2], gamma=gamma, alpha=alpha,
                                              do_precess=1.0, Stab=stab))
    out = dict(m=m, H=H, v=v, Hv=Hv, D=D, Dc=Dc, nax=nax, gamma=gamma, alpha=alpha, Ms=Ms,
               rhs=np.stack([rhs["rx"], rhs["ry"], rhs["rz"]], 1),
               jv=np.stack([jv["ox"], jv["oy"], jv["oz"]], 1))
    c1 = gamma * 1.0 / (1 + alpha ** 2)
    c2 = gamma * alpha / (1 + alpha ** 2)
    for tag, (shift, inc, absk, cub) in {"a": (1e12, 1, 1, 0), "b": (3e11, 0, 0, 0),
                                         "c": (5e11, 1, 1, 1)}.items():
        pc = ref.call("_PC_BUILD_INV3_KERNEL", n, dict(
            mx=m[:, 0], my=m[:, 1], mz=m[:, 2], hx=H[:, 0], hy=H[:, 1], hz=H[:, 2],
            dx=D[:, 0], dy=D[:, 1], dz=D[:, 2], dcx=Dc[:, 0], dcy=Dc[:, 1], dcz=Dc[:, 2],
            use_cubic=cub, include_stab=inc, use_abs_kappa=absk, shift=shift, eps_reg=1e-14,
            det_eps=1e-30, c1=c1, c2=c2, Stab=stab))
        inv = np.stack([pc[k] for k in ("i00", "i01", "i02", "i10", "i11", "i12", "i20", "i21", "i22")],
                       1).reshape(n, 3, 3)
        out[f"pc_{tag}"] = inv
        out[f"pc_{tag}_params"] = np.array([shift, inc, absk, cub], dtype=np.float64)
        ap = ref.call("_PC_APPLY_KERNEL", n, dict(
            i00=inv[:, 0, 0], i01=inv[:, 0, 1], i02=inv[:, 0, 2], i10=inv[:, 1, 0],
            i11=inv[:, 1, 1], i12=inv[:, 1, 2], i20=inv[:, 2, 0], i21=inv[:, 2, 1],
            i22=inv[:, 2, 2], x0=v[:, 0], x1=v[:, 1], x2=v[:, 2]))
        out[f"pcapply_{tag}"] = np.stack([ap["y0"], ap["y1"], ap["y2"]], 1)
    Ku = 4e5
    aprf = 2 * Ku / (4e-7 * math.pi * Ms)
    an = ref.call("_ANISOTROPY_NODAL_KERNEL", n, dict(mx=m[:, 0], my=m[:, 1], mz=m[:, 2],
                                                       nx=nax[:, 0], ny=nax[:, 1], nz=nax[:, 2],
                                                       pref=aprf))
    ad = ref.call("_ANISOTROPY_DIAG_KERNEL", n, dict(nx=nax[:, 0], ny=nax[:, 1], nz=nax[:, 2],
                                                      pref=aprf))
    out["ani"] = np.stack([an["hx"], an["hy"], an["hz"]], 1)
    out["ani_diag"] = np.stack([ad["dx"], ad["dy"], ad["dz"]], 1)
    out["Ku"] = Ku
    jcpu = ref_build.load_cpu_jv()
    o = np.empty(3 * n)
    jcpu(m, H, v, Hv, o, gamma, alpha, 1.0, stab)
    out["jv_cpu"] = o.reshape(n, 3)
    np.savez_compressed(OUT / "llg_kernels.npz", **out)


def make_torque_kernels():
    """The reference's STT / SOT per-node kernels on seeded inputs (torque_kernels.npz)."""
    from oracle import torques
    ref = ref_build.RefElementwise(ref_build.build(force=True))
    rng = np.random.default_rng(1006)
    n = 211
    m = rng.normal(size=(n, 3))
    m[: n // 2] /= np.linalg.norm(m[: n // 2], axis=1)[:, None]
    H = rng.normal(size=(n, 3)) * 1e5
    z = rng.normal(size=(n, 3)) * 0.3
    v = rng.normal(size=(n, 3))
    Hv = rng.normal(size=(n, 3)) * 1e5
    zv = rng.normal(size=(n, 3)) * 0.3
    p = rng.normal(size=(n, 3))
    p /= np.linalg.norm(p, axis=1)[:, None]
    D = rng.normal(size=(n, 3)) * 1e4
    gamma, alpha, Ms, beta = 2.211e5, 0.3, 8e5, 0.05
    pref = -gamma / (1 + alpha ** 2)
    stab = Ms * gamma / (1 + alpha ** 2) * 0.5
    prefZ = torques.pref_zhang(1e12, 0.6, beta, Ms, alpha)
    c_fl, c_dl = torques.sot_coefficients(gamma, alpha, 3e4, -1e4)
    d3 = lambda a, pfx: {f"{pfx}x": a[:, 0], f"{pfx}y": a[:, 1], f"{pfx}z": a[:, 2]}  # noqa: E731
    out = dict(m=m, H=H, z=z, v=v, Hv=Hv, zv=zv, p=p, D=D, gamma=gamma, alpha=alpha, Ms=Ms, beta=beta,
               prefZ=prefZ, c_fl=c_fl, c_dl=c_dl)
    r = ref.call("_LLG_RHS_STT_KERNEL", n, dict(**d3(m, "m"), **d3(H, "h"), **d3(z, "z"), prefactor=pref,
                                                 alpha=alpha, do_precess=1.0, Stab=stab, prefZhang=prefZ,
                                                 stt_a=beta - alpha, stt_b=1.0 + alpha * beta))
    out["rhs_stt"] = np.stack([r["rx"], r["ry"], r["rz"]], 1)
    j = ref.call("_JAC_VEC_STT_KERNEL", n, dict(**d3(m, "m"), **d3(H, "h"), **d3(z, "jm"), **d3(v, "v"),
                                                 **d3(Hv, "hv"), **d3(zv, "jv"), prefactor=pref, alpha=alpha,
                                                 do_precess=1.0, Stab=stab, prefZhang=prefZ, beta=beta))
    out["jv_stt"] = np.stack([j["ox"], j["oy"], j["oz"]], 1)
    c1 = gamma / (1 + alpha ** 2)
    c2 = gamma * alpha / (1 + alpha ** 2)
    c3 = (beta - alpha) * prefZ
    c4 = -(1.0 + alpha * beta) * prefZ
    keys = ("i00", "i01", "i02", "i10", "i11", "i12", "i20", "i21", "i22")
    for tag, (shift, inc, absk) in {"a": (1e12, 1, 1), "b": (3e11, 0, 0)}.items():
        pc = ref.call("_PC_BUILD_INV3_STT_KERNEL", n, dict(**d3(m, "m"), **d3(H, "h"), **d3(z, "g"),
                                                            d0=D[:, 0], d1=D[:, 1], d2=D[:, 2], shift=shift,
                                                            eps_reg=1e-14, det_eps=1e-30, c1=c1, c2=c2, c3=c3,
                                                            c4=c4, Stab=stab, include_stab=inc, use_abs_kappa=absk))
        out[f"pc_stt_{tag}"] = np.stack([pc[k] for k in keys], 1).reshape(n, 3, 3)
        out[f"pc_stt_{tag}_params"] = np.array([shift, inc, absk], dtype=np.float64)
    r = ref.call("_LLG_RHS_SOT_KERNEL", n, dict(**d3(m, "m"), **d3(H, "h"), **d3(p, "p"), prefactor=pref,
                                                 alpha=alpha, do_precess=1.0, Stab=stab, c_fl=c_fl, c_dl=c_dl))
    out["rhs_sot"] = np.stack([r["rx"], r["ry"], r["rz"]], 1)
    j = ref.call("_JAC_VEC_SOT_KERNEL", n, dict(**d3(m, "m"), **d3(H, "h"), **d3(p, "p"), **d3(v, "v"),
                                                 **d3(Hv, "hv"), prefactor=pref, alpha=alpha, do_precess=1.0,
                                                 Stab=stab, c_fl=c_fl, c_dl=c_dl))
    out["jv_sot"] = np.stack([j["ox"], j["oy"], j["oz"]], 1)
    for tag, (shift, absd) in {"a": (1e12, 0), "b": (3e11, 1)}.items():
        pc = ref.call("_PC_BUILD_INV3_SOT_KERNEL", n, dict(**d3(m, "m"), **d3(H, "h"), **d3(p, "p"),
                                                            d0=D[:, 0], d1=D[:, 1], d2=D[:, 2], shift=shift,
                                                            eps_reg=1e-14, det_eps=1e-30, prefactor=pref,
                                                            alpha=alpha, do_precess=1.0, Stab=stab, c_fl=c_fl,
                                                            c_dl=c_dl, use_abs_diag=absd))
        out[f"pc_sot_{tag}"] = np.stack([pc[k] for k in keys], 1).reshape(n, 3, 3)
        out[f"pc_sot_{tag}_params"] = np.array([shift, absd], dtype=np.float64)
    np.savez_compressed(OUT / "torque_kernels.npz", **out)


C2_CASE = (400, 400, 2, 2.5)
C2_ROWS_SEED = 3100


def c2_row_vectors(Xb):
    """The three vectors the c2_rows fixture applies B to (boundary order, Nb x 3):
    seeded standard normal; cos(2 pi x / 1000) cos(2 pi y / 1000) (smooth at the film's
    scale); z - mean(z) plus 0.1 x seeded noise (linear through the thickness)."""
    Nb = Xb.shape[0]
    rng = np.random.default_rng(C2_ROWS_SEED + 1)
    x = np.empty((Nb, 3))
    x[:, 0] = rng.standard_normal(Nb)
    x[:, 1] = np.cos(2 * math.pi * Xb[:, 0] / 1000.0) * np.cos(2 * math.pi * Xb[:, 1] / 1000.0)
    x[:, 2] = (Xb[:, 2] - Xb[:, 2].mean()) + 0.1 * rng.standard_normal(Nb)
    return x


def make_c2_rows(mods, nrows=4096, chunk=256):
    """Rows of the reference's dense Lindholm operator on the 400x400x2 film (the
    H-matrix headline mesh), with the diagonal jump Omega/4pi - 1 added, applied to
    c2_row_vectors: the reference answer for the H-matrix apply at full size."""
    X, T = mesh.kuhn_box(*C2_CASE)
    bd = lindholm.boundary_data(X, T)
    Nb = bd["Xb"].shape[0]
    prov = provider_for(mods, bd)
    rng = np.random.default_rng(C2_ROWS_SEED)
    rows = np.sort(rng.choice(Nb, nrows, replace=False)).astype(np.int32)
    x = c2_row_vectors(bd["Xb"])
    cols = np.arange(Nb, dtype=np.int32)
    y = np.empty((nrows, 3))
    rowsum = np.empty(nrows)
    jump = bd["omega_sum"] / (4.0 * math.pi) - 1.0
    for s in range(0, nrows, chunk):
        r = rows[s:s + chunk]
        B = prov.fill_block(r, cols)
        B[np.arange(r.size), r] += jump[r]
        y[s:s + chunk] = B @ x
        rowsum[s:s + chunk] = B.sum(axis=1)
        print(f"c2_rows {s + r.size}/{nrows}", flush=True)
    np.savez_compressed(OUT / "c2_rows.npz", rows=rows, y=y, rowsum=rowsum, nb=np.int64(Nb),
                        x_sum=x.sum(axis=0), x_sqsum=(x * x).sum(axis=0), seed=np.int64(C2_ROWS_SEED),
                        case=np.array(C2_CASE, dtype=np.float64))


def make_example_mesh():
    """The reference's hysteresis_octahedral_nanoparticles/chain mesh (XDMF + gzip HDF5) read by
    spinfemx_b200.io, stored as example_chain_mesh.npz: a small unstructured mesh for the GPU
    tests (nothing on the GPU side reads the reference)."""
    sys.path.insert(0, str(ROOT / "fenicsx-micromagnetics_b200"))
    from spinfemx_b200 import io as sio
    X, T, _ = sio.read_xdmf_mesh(REF_EXAMPLES / "cpu/hysteresis_octahedral_nanoparticles/chain.xdmf")
    np.savez_compressed(OUT / "example_chain_mesh.npz", X=X, tets=T)


def main():
    mods = ref_build.import_reference_hmatrix()
    if sys.argv[1:] == ["c2_rows"]:
        make_c2_rows(mods)
        return
    bds = {}
    for name, (nx, ny, nz, h) in CASES.items():
        X, T = mesh.kuhn_box(nx, ny, nz, h)
        bds[name] = lindholm.boundary_data(X, T)
        print(name, "N", X.shape[0], "E", T.shape[0], "Nb", bds[name]["Xb"].shape[0], flush=True)
    make_llg_kernels()
    make_torque_kernels()
    make_example_mesh()
    make_lindholm_pairs(mods, bds["box20"])
    make_dense(mods, bds["box20"])
    make_trees(mods, bds)
    make_aca(mods)
    for name in CASES:
        d = make_hmatrix(mods, name, bds[name])
        print(name, "far", len(d.far_blocks), "near nnz", d.near_csr.nnz, flush=True)
    make_cache(mods)
    make_c2_rows(mods)


if __name__ == "__main__":
    main()
