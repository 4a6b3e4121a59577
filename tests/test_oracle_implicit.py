"""The implicit driver's oracle (oracle/implicit.py) against known answers.

* the variable-step BDF coefficients reduce to BDF2 at constant steps (3/2, -2, 1/2) / h and the
  quadratic predictor to (3, -3, 1);
* GMRES(restart) with a left preconditioner solves small nonsymmetric systems to its tolerance,
  across restarts, and ends on a happy breakdown after as many iterations as the matrix has
  distinct eigenvalues;
* Newton with the quadratic backtracking line search converges on a problem whose full Newton
  step overshoots;
* relax_implicit converges to a fine RK4 trajectory as the tolerance falls, at the rate of a
  second-order method with a third-order error control (global error ~ tol^(2/3)).
"""
import numpy as np
import pytest

from oracle import implicit as oimp
from oracle import llg as ollg
from oracle import mesh as omesh


def test_bdf2_coefficients_at_constant_step():
    h, t = 1e-13, 5e-12
    a = oimp.lagrange_derivs(t + h, [t + h, t, t - h])
    assert np.allclose(np.array(a) * h, [1.5, -2.0, 0.5], rtol=1e-10, atol=0)
    lv = oimp.lagrange_values(t + h, [t, t - h, t - 2 * h])
    assert np.allclose(lv, [3.0, -3.0, 1.0], rtol=1e-10, atol=0)
    # backward Euler on two nodes
    a1 = oimp.lagrange_derivs(t + h, [t + h, t])
    assert np.allclose(np.array(a1) * h, [1.0, -1.0], rtol=1e-12)


@pytest.mark.parametrize("restart", [30, 4])
def test_gmres_solves_nonsymmetric_system(restart):
    rng = np.random.default_rng(1)
    n = 40
    A = np.eye(n) * 4.0 + rng.normal(size=(n, n)) * 0.3
    d = np.diag(A).copy()
    b = rng.normal(size=n)
    x, its, reason = oimp.gmres_left(lambda v: A @ v, lambda v: v / d, b, 1e-10, 1e-50, 1e5, 500, restart)
    assert reason > 0 and its > 0
    xs = np.linalg.solve(A, b)
    assert np.linalg.norm(x - xs) <= 1e-8 * np.linalg.norm(xs)
    # the reported convergence is on the preconditioned residual
    assert np.linalg.norm((b - A @ x) / d) <= 1e-10 * np.linalg.norm(b / d) * 1.0001


def test_gmres_happy_breakdown():
    n = 12
    A = np.diag(np.repeat([1.0, 2.0, 5.0], n // 3))
    b = np.arange(1.0, n + 1)
    x, its, reason = oimp.gmres_left(lambda v: A @ v, lambda v: v.copy(), b, 1e-14, 1e-50, 1e5, 100, 30)
    assert its == 3 and reason > 0
    assert np.allclose(A @ x, b, rtol=0, atol=1e-11 * np.abs(b).max())


def test_gmres_iteration_limit():
    rng = np.random.default_rng(3)
    n = 60
    A = np.eye(n) + rng.normal(size=(n, n))
    b = rng.normal(size=n)
    x, its, reason = oimp.gmres_left(lambda v: A @ v, lambda v: v.copy(), b, 1e-12, 1e-50, 1e5, 7, 5)
    assert its == 7 and reason == oimp.KSP_DIVERGED_ITS


class _Arctan:
    """F(y) = shift y + base - f(y) with f = -atan(y) per entry: Newton from far away overshoots."""

    def __init__(self):
        self.fevals = 0
        self.y = None

    def F(self, y):
        self.fevals += 1
        return np.arctan(y)

    def setup(self, y):
        self.y = y.copy()

    def A(self, v):
        return v / (1.0 + self.y * self.y)

    def P(self, v):
        return v.copy()


def test_newton_line_search_backtracks():
    o = dict(oimp.DEFAULTS, snes_rtol=1e-12, snes_atol=1e-14, snes_max_it=30)
    pb = _Arctan()
    y, reason, nits, lits = oimp.newton_solve(pb, np.array([10.0, -3.0]), o)
    assert reason > 0 and np.abs(y).max() < 1e-10
    # the full step from 10 lands at |y| > 100: the line search must have cut it
    assert pb.fevals > nits + 1


def test_relax_implicit_converges_to_fine_rk4():
    X, T = omesh.kuhn_box(4, 4, 3, 2.0)
    N = X.shape[0]
    hef = ollg.EffectiveFieldOracle(X, T, 8e5, Aex=1.3e-11, alpha=0.5, H0=np.tile([0.0, 0.0, 3e4], N))
    rng = np.random.default_rng(2)
    m0 = rng.normal(size=(N, 3))
    m0 = (m0 / np.linalg.norm(m0, axis=1)[:, None]).ravel()
    errs = []
    for tol in (1e-6, 1e-8):
        m, st = oimp.relax_implicit(hef, m0, 0.0, 1e-12, 1e-13, tol, tol)
        assert st["reason"] == 1 and st["snes_failures"] == 0 and st["rejected"] >= 1
        n = 2000
        h = st["t_end"] / n
        mr = m0.copy()
        for _ in range(n):
            mr = ollg.rk4_step(hef.llg_rhs, mr, h)
        errs.append(np.abs(m - mr).max())
    assert errs[0] < 2e-3
    assert errs[0] / errs[1] > 10.0 ** (2.0 / 3.0 * 2.0) / 2.0
