"""The FP64 Newton polish of the two-stage MLE on smooth test functions
shaped like the Matern likelihood's flat sigma^2-beta ridge (no GPU)."""
import numpy as np

from exageostat_b200.mle import newton_polish


def _ridge(th):
    """f = -(log s - 2 log b - c)^2 * 400 - (log b - 0.3)^2 * 0.05 - (n - 0.5)^2 * 40:
    steep across the ridge s / b^2 = e^c, flat along it."""
    s, b, n = th
    u = np.log(s) - 2 * np.log(b) - 1.0
    v = np.log(b) + 2.0
    f = -400 * u * u - 0.05 * v * v - 40 * (n - 0.5) ** 2
    g = np.array([-800 * u / s, (1600 * u - 0.1 * v) / b, -80 * (n - 0.5)])
    return f, g


def test_newton_polish_reaches_the_ridge_optimum_from_a_nearby_start():
    lb, ub = [0.01] * 3, [5.0] * 3
    # optimum: v = 0 -> b = e^-2, u = 0 -> s = e b^2
    b0 = np.exp(-2.0)
    opt = np.array([np.e * b0 * b0, b0, 0.5])
    start = opt * np.array([1.02, 1.01, 1.003])
    th, f, evals = newton_polish(_ridge, start, lb, ub)
    assert np.max(np.abs(th - opt) / opt) < 1e-5
    assert evals <= 6 * (2 * 3 + 6) + 1


def test_newton_polish_never_decreases_and_respects_bounds():
    lb, ub = np.array([0.01] * 3), np.array([5.0] * 3)
    start = np.array([4.9, 0.02, 0.02])
    f0, _ = _ridge(start)
    th, f, _ = newton_polish(_ridge, start, lb, ub, max_steps=3)
    assert f >= f0
    assert np.all(th >= lb) and np.all(th <= ub)


def test_newton_polish_treats_failing_evaluations_as_minus_infinity():
    """A parameter region where the objective raises (as a covariance that is
    not positive definite does) rejects steps instead of aborting."""
    lb, ub = [0.01] * 3, [5.0] * 3
    b0 = np.exp(-2.0)
    opt = np.array([np.e * b0 * b0, b0, 0.5])

    def guarded(th):
        if th[2] > 0.5005:
            raise RuntimeError("not positive definite")
        return _ridge(th)

    th, f, _ = newton_polish(guarded, opt * np.array([1.02, 1.01, 1.0]), lb, ub)
    assert np.isfinite(f) and th[2] <= 0.5005
    assert f >= guarded(opt * np.array([1.02, 1.01, 1.0]))[0]
    th2, f2, ev2 = newton_polish(guarded, opt * np.array([1.0, 1.0, 1.01]), lb, ub)
    assert f2 == -np.inf and ev2 == 1
