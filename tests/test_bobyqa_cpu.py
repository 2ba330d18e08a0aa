"""The library's bound-constrained derivative-free maximiser (host code, no GPU)."""
import numpy as np


def test_maximises_concave_quadratic_in_the_interior(xg):
    c = np.array([0.7, -0.3, 1.9])
    f = lambda x: -np.sum((x - c) ** 2 * np.array([1.0, 10.0, 0.1]))
    x, fm, ev = xg.bobyqa_maximize(f, [0.0, 0.0, 0.0], [-5, -5, -5], [5, 5, 5], ftol_abs=0, rhoend=1e-8)
    assert np.allclose(x, c, atol=1e-5) and fm > -1e-9 and ev < 300


def test_active_bounds(xg):
    f = lambda x: -((x[0] - 3) ** 2 + (x[1] + 2) ** 2)
    x, fm, _ = xg.bobyqa_maximize(f, [0.5, 0.5], [0.01, 0.01], [1.0, 5.0], ftol_abs=0, rhoend=1e-9)
    assert np.allclose(x, [1.0, 0.01], atol=1e-7)


def test_rosenbrock_from_a_bound_start(xg):
    f = lambda x: -(100 * (x[1] - x[0] ** 2) ** 2 + (1 - x[0]) ** 2)
    x, fm, ev = xg.bobyqa_maximize(f, [-1.5, -1.0], [-2, -2], [2, 2], ftol_abs=0, rhoend=1e-8, maxeval=3000)
    assert np.allclose(x, [1, 1], atol=1e-4), (x, ev)


def test_maxeval_and_ftol(xg):
    calls = []
    f = lambda x: calls.append(1) or -np.sum(x ** 2)
    xg.bobyqa_maximize(f, [1.0, 1.0, 1.0], [-2] * 3, [2] * 3, maxeval=12, ftol_abs=0)
    assert len(calls) <= 12


def test_matern_mle_on_oracle_objective(xg, ora):
    """Maximise the oracle log-likelihood of a small synthetic field from the
    reference's start (the lower bounds); the maximiser must beat the truth's
    likelihood and lie near it."""
    N = 400
    theta0 = [1.0, 0.1, 0.5]
    x, y, z, _ = ora.synthetic_field(N, 0, theta0)
    f = lambda t: ora.dmle(x, y, z, t)[0]
    lb, ub = [0.01] * 3, [5.0] * 3
    th, fm, ev = xg.bobyqa_maximize(f, lb, lb, ub, ftol_abs=1e-9)
    assert fm >= f(theta0) - 1e-6
    assert ev < 600
    # a gradient-based maximiser from an interior start finds the same point
    from scipy.optimize import minimize

    r = minimize(lambda t: -f(t), [0.5, 0.5, 0.5], bounds=list(zip(lb, ub)), method="L-BFGS-B")
    assert abs(fm + r.fun) < 1e-6 * abs(fm)
    assert np.allclose(th, r.x, rtol=1e-3)
