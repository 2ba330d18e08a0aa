"""Adjoint gradient of the log-likelihood against finite differences of the
oracle (FP64).  Tolerance 1e-6 relative to max(|grad|, 1): the 4th-order
central difference with h = 1e-4 theta is accurate to ~1e-9 here."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fd_grad(f, th, rel=1e-4):
    th = np.asarray(th, dtype=float)
    g = np.zeros_like(th)
    for i in range(th.size):
        h = rel * th[i]
        e = np.zeros_like(th)
        e[i] = h
        g[i] = (8 * (f(th + e) - f(th - e)) - (f(th + 2 * e) - f(th - 2 * e))) / (12 * h)
    return g


@pytest.mark.parametrize("n,ts,theta,kernel", [
    (700, 128, [1.0, 0.1, 0.5], 0),
    (900, 256, [1.3, 0.07, 0.73], 0),
    (650, 128, [0.8, 0.2, 1.5], 0),
    (800, 128, [1.0, 0.1, 1.0, 0.01], 1),
])
def test_gradient_matches_finite_differences(gpu, ora, n, ts, theta, kernel):
    x, y, z, _ = ora.synthetic_field(n, 3, theta, kernel)
    with gpu.Session(x, y, kernel=kernel, dts=ts) as s:
        s.set_data(z=z)
        ll, g = s.loglik(theta, grad=True)
        # the value is the plain evaluation's
        assert ll == pytest.approx(ora.dmle(x, y, z, theta, kernel)[0], rel=1e-10)
        # and a plain evaluation after a gradient one is unaffected
        assert s.loglik(theta) == pytest.approx(ll, rel=1e-12)
    ref = _fd_grad(lambda t: ora.dmle(x, y, z, t, kernel)[0], theta)
    scale = max(np.abs(ref).max(), 1.0)
    assert np.abs(g - ref).max() / scale < 1e-6, (g, ref)


def test_autograd_function_and_gradcheck(gpu, ora):
    import torch

    from exageostat_b200.autograd import loglik

    x, y, z, _ = ora.synthetic_field(500, 1, [1.0, 0.1, 0.5])
    with gpu.Session(x, y, dts=128) as s:
        s.set_data(z=z)
        th = torch.tensor([0.9, 0.12, 0.6], dtype=torch.float64, requires_grad=True)
        ll = loglik(th, s)
        ll.backward()
        _, g = s.loglik(th.detach().numpy(), grad=True)
        assert np.allclose(th.grad.numpy(), g)
        assert torch.autograd.gradcheck(lambda t: loglik(t, s), (th,), eps=1e-6, atol=1e-5, rtol=1e-4)


def test_lbfgsb_and_bobyqa_reach_the_same_maximiser(gpu, ora):
    """C1-sized MLE (N = 1600, theta0 = (1, 0.1, 0.5), bounds [0.01, 5]^3):
    the gradient driver and the derivative-free driver agree on theta-hat and
    the maximum."""
    from exageostat_b200.autograd import fit_lbfgsb

    x, y, z, _ = ora.synthetic_field(1600, 0, [1.0, 0.1, 0.5])
    lb, ub = [0.01] * 3, [5.0] * 3
    with gpu.Session(x, y, dts=320) as s:
        s.set_data(z=z)
        th_b, ll_b, ev_b = s.fit_bobyqa(lb, ub, ftol_abs=1e-9)
        th_l, ll_l, ev_l = fit_lbfgsb(s, lb, ub, x0=[0.5, 0.5, 0.5])
    assert abs(ll_b - ll_l) < 1e-6 * abs(ll_b)
    assert np.allclose(th_b, th_l, rtol=1e-3)
    assert ev_l < ev_b
