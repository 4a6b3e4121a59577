"""Known answers for the interfacial DMI operator (DMI_Interfacial_GPU.py:140-172).

The reference assembles  int (div(m) n - grad(n.m)) . v  plus a boundary term
0.5 int_ds ((n x nu) x m) . v, row-scaled by -2D/(mu0 Ms)/1e-9/V_i (mesh in nm).
At a node whose support does not touch the boundary the boundary term vanishes,
and for a linear m and a constant n the volume integrand is constant, so the
lumped row gives the continuum field exactly:

    H_i = (2 D / (mu0 Ms)) (grad(n.m) - div(m) n) / 1e-9.

For the helix m = (cos kx, 0, sin kx), n = z the continuum field is
(2 D k / (mu0 Ms)) m; P1 with lumping reproduces it at interior nodes to O((kh)^2).

Tolerances: linear fields 1e-10 relative (rounding only); helix 2e-2 at kh = 0.31
and second-order convergence under refinement (error ratio >= 3 for h -> h/2).
"""
import math

import numpy as np
import pytest

from oracle import fem as ofem
from oracle import lindholm as olin
from oracle import mesh as omesh

MU0 = 4e-7 * math.pi
D, MS = 3e-3, 8e5


def interior_nodes(X, T):
    tris, _ = olin.boundary_facets(X, T)
    inner = np.ones(X.shape[0], bool)
    inner[np.unique(tris.ravel())] = False
    return np.nonzero(inner)[0]


def oracle_dmi_field(X, T, m, n):
    bd = olin.boundary_data(X, T)
    K = ofem.dmi_interfacial_matrix(X, T, D, MS, np.tile(n, X.shape[0]).reshape(-1, 3), bd["tris"], bd["ntri"])
    return (K @ m.ravel()).reshape(-1, 3)


def linear_case(seed):
    rng = np.random.default_rng(seed)
    G = rng.normal(size=(3, 3)) * 0.02      # 1/nm
    m0 = rng.normal(size=3)
    n = rng.normal(size=3)
    n /= np.linalg.norm(n)
    return G, m0, n


def linear_expected(G, n):
    div = np.trace(G)                        # d_c m_c
    grad_nm = G.T @ n                        # d_c (n_d m_d) = n_d G_dc
    return (2.0 * D / (MU0 * MS)) * (grad_nm - div * n) / 1e-9


@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_dmi_linear_field_exact(seed):
    X, T = omesh.kuhn_box(6, 5, 4, 2.0)
    G, m0, n = linear_case(seed)
    m = m0[None, :] + X @ G.T
    H = oracle_dmi_field(X, T, m, n)
    I = interior_nodes(X, T)
    assert I.size > 20
    ref = linear_expected(G, n)
    err = np.abs(H[I] - ref[None, :]).max() / np.linalg.norm(ref)
    assert err < 1e-10


def helix_error(h, period=20.0):
    L = 2 * period
    X, T = omesh.kuhn_box(int(round(L / h)), 4, 4, h)
    k = 2 * math.pi / period                  # 1/nm
    m = np.stack([np.cos(k * X[:, 0]), np.zeros(X.shape[0]), np.sin(k * X[:, 0])], 1)
    H = oracle_dmi_field(X, T, m, np.array([0.0, 0.0, 1.0]))
    I = interior_nodes(X, T)
    ref = (2.0 * D * (k / 1e-9) / (MU0 * MS)) * m[I]
    return float(np.linalg.norm(H[I] - ref) / np.linalg.norm(ref))


def test_oracle_dmi_helix_converges():
    e1 = helix_error(1.0)
    e2 = helix_error(0.5)
    assert e1 < 2e-2
    assert e1 / e2 >= 3.0


@pytest.mark.gpu
def test_product_dmi_linear_field_exact():
    torch = pytest.importorskip("torch")
    import spinfemx_b200 as spx
    X, T = omesh.kuhn_box(6, 5, 4, 2.0)
    G, m0, n = linear_case(3)
    m = m0[None, :] + X @ G.T
    hef = spx.EffectiveField(X, T, MS, D_int=D, n0_int_vec=n, alpha=0.3)
    mt = torch.as_tensor(m.ravel().copy(), device="cuda")
    out = torch.empty_like(mt)
    hef.compute_H_eff_vec(mt, out)
    H = out.cpu().numpy().reshape(-1, 3)
    I = interior_nodes(X, T)
    ref = linear_expected(G, n)
    assert np.abs(H[I] - ref[None, :]).max() / np.linalg.norm(ref) < 1e-10
    # every node (boundary rows included) equals the oracle operator
    Ho = oracle_dmi_field(X, T, m, n)
    assert np.abs(H - Ho).max() <= 1e-11 * np.abs(Ho).max()


# ---------------------------------------------------------------- bulk DMI (DMI_Bulk_GPU.py:52-66)
# H = -(2 D / (mu0 Ms)) curl(m) / 1e-9 at interior nodes for linear m (exact); for the helix
# m = (0, cos kx, sin kx), curl m = -k m, so H = (2 D k / (mu0 Ms)) m.

def oracle_bulk_field(X, T, m):
    bd = olin.boundary_data(X, T)
    K = ofem.dmi_bulk_matrix(X, T, D, MS, bd["tris"], bd["ntri"])
    return (K @ m.ravel()).reshape(-1, 3)


def curl_of_linear(G):
    # m_c = G_cd x_d: curl_x = d_y m_z - d_z m_y, ...
    return np.array([G[2, 1] - G[1, 2], G[0, 2] - G[2, 0], G[1, 0] - G[0, 1]])


@pytest.mark.parametrize("seed", [4, 5])
def test_oracle_bulk_dmi_linear_field_exact(seed):
    X, T = omesh.kuhn_box(6, 5, 4, 2.0)
    G, m0, _ = linear_case(seed)
    m = m0[None, :] + X @ G.T
    H = oracle_bulk_field(X, T, m)
    I = interior_nodes(X, T)
    ref = -(2.0 * D / (MU0 * MS)) * curl_of_linear(G) / 1e-9
    assert np.abs(H[I] - ref[None, :]).max() / np.linalg.norm(ref) < 1e-10


def bulk_helix_error(h, period=20.0):
    X, T = omesh.kuhn_box(int(round(2 * period / h)), 4, 4, h)
    k = 2 * math.pi / period
    m = np.stack([np.zeros(X.shape[0]), np.cos(k * X[:, 0]), np.sin(k * X[:, 0])], 1)
    H = oracle_bulk_field(X, T, m)
    I = interior_nodes(X, T)
    ref = (2.0 * D * (k / 1e-9) / (MU0 * MS)) * m[I]
    return float(np.linalg.norm(H[I] - ref) / np.linalg.norm(ref))


def test_oracle_bulk_dmi_helix_converges():
    e1, e2 = bulk_helix_error(1.0), bulk_helix_error(0.5)
    assert e1 < 2e-2 and e1 / e2 >= 3.0


def test_oracle_bulk_dmi_energy_symmetry():
    """The bulk form with its boundary term is symmetric (a conservative field): m.K m' = m'.K m
    with K unscaled by the (node-dependent) lumped volumes."""
    X, T = omesh.kuhn_box(4, 4, 3, 2.0)
    bd = olin.boundary_data(X, T)
    vol = ofem.lumped_volume(X, T)
    K = ofem.dmi_bulk_matrix(X, T, D, MS, bd["tris"], bd["ntri"], vol)
    Ku = ofem.sp.diags(np.repeat(vol, 3)) @ K
    assert abs(Ku - Ku.T).max() <= 1e-12 * abs(Ku).max()


@pytest.mark.gpu
def test_product_bulk_dmi_vs_oracle():
    torch = pytest.importorskip("torch")
    import spinfemx_b200 as spx
    X, T = omesh.kuhn_box(6, 5, 4, 2.0)
    G, m0, n = linear_case(6)
    m = m0[None, :] + X @ G.T
    for kw in (dict(D_bulk=D), dict(D_bulk=D, D_int=0.7 * D, n0_int_vec=n)):
        hef = spx.EffectiveField(X, T, MS, alpha=0.3, **kw)
        mt = torch.as_tensor(m.ravel().copy(), device="cuda")
        out = torch.empty_like(mt)
        hef.compute_H_eff_vec(mt, out)
        Ho = oracle_bulk_field(X, T, m)
        if "D_int" in kw:
            Ho = Ho + 0.7 * oracle_dmi_field(X, T, m, n)
        assert np.abs(out.cpu().numpy().reshape(-1, 3) - Ho).max() <= 1e-11 * np.abs(Ho).max()
