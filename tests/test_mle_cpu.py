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


def _ridge2(th):
    """A ridge with the curvatures of a Matern likelihood near its optimum
    (across the ridge 2000, along it 20, in nu 200, in log theta): a gradient
    stop at |g| = 0.1 leaves theta ~3e-3 along the ridge."""
    s, b, n = th
    u = np.log(s) - 2 * np.log(b) - 1.0
    v = np.log(b) + 2.0
    w = np.log(n / 0.5)
    f = -2000 * u * u - 20 * v * v - 200 * w * w
    g = np.array([-4000 * u / s, (8000 * u - 40 * v) / b, -400 * w / n])
    return f, g


class _FakeSession:
    """The calls fit_mixed makes of a Session, on _ridge2 (no GPU)."""

    def __init__(self):
        self.values = 0

    def set_sliced(self):
        pass

    def set_fp64(self):
        pass

    def z(self):
        return np.array([1.0, -1.0])

    def loglik(self, th, grad=False):
        f, g = _ridge2(np.asarray(th, dtype=float))
        if grad:
            return f, g
        self.values += 1
        return f


def test_fit_mixed_polishes_along_a_flat_ridge_after_a_loose_gradient_stop():
    """A gradient stop at the loose tolerance of the sliced gradient can leave
    theta ~3e-3 along the flat ridge: the trust region's Newton step says so,
    the value-based polish runs and lands on the optimum."""
    from exageostat_b200.mle import fit_mixed

    lb, ub = [0.01] * 3, [5.0] * 3
    b0 = np.exp(-2.0)
    opt = np.array([np.e * b0 * b0, b0, 0.5])
    th, f, ev, nvals, th1 = fit_mixed(_FakeSession(), lb, ub, theta0=opt * np.array([1.8, 0.7, 1.4]), gtol=0.1)
    assert np.max(np.abs(th1 - opt) / opt) > 1e-3
    assert nvals > 0 and np.max(np.abs(th - opt) / opt) < 1e-6


def test_fit_mixed_skips_the_polish_when_the_newton_step_is_tiny():
    """A gradient stop whose learned model puts the optimum within 5e-4 in log
    theta spends no polish values; a stop before the model has seen 2 n
    updates always polishes."""
    from exageostat_b200.mle import fit_mixed

    lb, ub = [0.01] * 3, [5.0] * 3
    b0 = np.exp(-2.0)
    opt = np.array([np.e * b0 * b0, b0, 0.5])
    th, f, ev, nvals, th1 = fit_mixed(_FakeSession(), lb, ub, theta0=opt * np.array([1.3, 1.14, 1.0]), gtol=0.1)
    assert nvals == 0 and np.array_equal(th, th1) and np.max(np.abs(th - opt) / opt) < 1e-4
    th, f, ev, nvals, th1 = fit_mixed(_FakeSession(), lb, ub, theta0=opt * (1 + 1e-6), gtol=0.1)
    assert ev == 1 and nvals > 0
