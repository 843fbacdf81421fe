"""LBFGS geometry optimisation (lbfgs.f restated): the optimiser on
analytic functions (CPU), and the full driver on the GPU engine against the
same driver on the CPU restatement."""
import numpy as np
import pytest

from amdkiit_b200.geo_opt import GeometryOptimizer, lbfgs, line_search


def rosen(x):
    f = np.sum(100.0 * (x[1:] - x[:-1] ** 2) ** 2 + (1.0 - x[:-1]) ** 2)
    g = np.zeros_like(x)
    g[:-1] += -400.0 * x[:-1] * (x[1:] - x[:-1] ** 2) - 2.0 * (1.0 - x[:-1])
    g[1:] += 200.0 * (x[1:] - x[:-1] ** 2)
    return float(f), g


@pytest.mark.parametrize("n", [2, 5, 10])
def test_lbfgs_rosenbrock(n):
    x0 = np.full(n, -1.2)
    x0[1::2] = 1.0
    r = lbfgs(rosen, x0, eps=1e-8, max_iter=500)
    assert r.converged
    assert np.allclose(r.x, 1.0, atol=1e-6)


def test_lbfgs_quadratic_is_exact_in_few_steps():
    rng = np.random.default_rng(0)
    Q = rng.standard_normal((6, 6))
    A = Q @ Q.T + 6 * np.eye(6)
    b = rng.standard_normal(6)
    fun = lambda x: (0.5 * x @ A @ x - b @ x, A @ x - b)
    r = lbfgs(fun, np.zeros(6), eps=1e-7, max_iter=100)
    assert r.converged and r.iterations <= 30
    assert np.allclose(r.x, np.linalg.solve(A, b), atol=1e-7)


def test_line_search_meets_strong_wolfe():
    x = np.array([-1.2, 1.0])
    f, g = rosen(x)
    s = -g
    r = line_search(rosen, x, f, g, s, 1.0 / np.linalg.norm(g))
    assert r.info == 1
    dg0, dg = g @ s, r.g @ s
    assert r.f <= f + 1e-4 * r.stp * dg0
    assert abs(dg) <= 0.9 * abs(dg0)


def test_line_search_rejects_ascent():
    x = np.array([0.0, 0.0])
    f, g = rosen(x)
    assert line_search(rosen, x, f, g, g, 1.0).info == -1


@pytest.mark.gpu
def test_geometry_optimisation_follows_oracle():
    from amdkiit_b200 import configs
    from amdkiit_b200.engine import FP64, Engine
    from tests.helpers import OracleEngine, start_coefficients
    s = configs.small_water()
    e = Engine(s, FP64)
    g = e.gvectors()
    e.set_wfn(start_coefficients(g["hg"][: e.ngpw], 2 * np.pi / s.alat, e.nstate, 1234))
    og = GeometryOptimizer(e, gcut_wfn=1e-7, gcut_geo=2e-3, max_step=30)
    oo = GeometryOptimizer(OracleEngine(s), gcut_wfn=1e-7, gcut_geo=2e-3, max_step=30)
    rg, xg = og.run()
    ro, xo = oo.run()
    assert rg.converged and ro.converged
    assert rg.iterations == ro.iterations and rg.evaluations == ro.evaluations
    assert np.max(np.abs(xg - xo)) < 1e-6
    assert abs(rg.f - ro.f) < 1e-8
    # energy went down along the way
    assert rg.history[-1][0] < rg.history[0][0]
