"""FP64 tiles with INT8-sliced trailing updates (precision = 3, left-looking)
against LAPACK and the oracle.  Each update is an exact integer product of
operands carried to ~32 bits relative to their row maximum (2^-32 ~ 2.3e-10
per chunk product, amplified by the triangular solves), so the factor stays
within 5e-8 of LAPACK's (relative to max |L|) and the log-likelihood within
1e-7 relative; the accuracy target for reduced precision is 1e-6."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,ts", [(700, 128), (1300, 256), (1900, 384), (2100, 512), (3500, 512)])
def test_sliced_factor_matches_lapack(gpu, ora, n, ts):
    x, y = ora.generate_xy_loc(n, 4)
    theta = [1.0, 0.1, 0.5]
    L = gpu.sliced_factor_dense(x, y, theta, ts=ts)
    C = ora.covariance_lower(x, y, theta)
    C = C + np.tril(C, -1).T
    Lref = np.linalg.cholesky(C)
    err = np.abs(L - Lref).max() / np.abs(Lref).max()
    assert err < 5e-8, err
    assert np.all(np.triu(L, 1) == 0)


@pytest.mark.parametrize("ts", [128, 256])
def test_sliced_loglik_close_to_oracle(gpu, ora, ts):
    n = 3000
    theta = [1.0, 0.05, 0.5]
    x, y, z, _ = ora.synthetic_field(n, 0, theta)
    ref = ora.dmle(x, y, z, theta)[0]
    got = gpu.dmle_host_sliced(x, y, z, theta, ts=ts)[0]
    assert abs(got - ref) / abs(ref) < 1e-7, (got, ref)


def test_sliced_smooth_field_through_mle_alg(gpu, ora):
    """nu = 1.5, cond(Sigma) ~ 3e6: the FP32 off-band scheme needs a band of
    4 tiles for 1e-6 here; the sliced updates stay within 1e-7."""
    n = 2100
    theta = [1.0, 0.1, 1.5]
    x, y, z, _ = ora.synthetic_field(n, 2, theta)
    with gpu.Session(x, y, dts=256) as s:
        s.set_data(z=z)
        fp64 = s.mle_alg(theta)
        s.set_sliced()
        assert s.data.precision == 3
        sl = s.mle_alg(theta)
        assert abs(sl - fp64) / abs(fp64) < 1e-7, (sl, fp64)
        s.set_fp64()
        assert s.mle_alg(theta) == pytest.approx(fp64, rel=1e-14)


def test_sliced_nugget_and_general_nu(gpu, ora):
    theta = [1.0, 0.1, 0.73, 0.01]
    x, y, z, _ = ora.synthetic_field(1800, 5, theta, kernel=1)
    ref = ora.dmle(x, y, z, theta, 1)[0]
    got = gpu.dmle_host_sliced(x, y, z, theta, kernel=1, ts=128)[0]
    assert abs(got - ref) / abs(ref) < 1e-7, (got, ref)


def test_sliced_rejects_non_spd(gpu, ora):
    x, y = ora.generate_xy_loc(600, 1)
    x = x.copy()
    x[5] = np.nan
    z = np.ones(600)
    with pytest.raises(gpu.XgError):
        gpu.dmle_host_sliced(x, y, z, [1.0, 0.1, 0.5], ts=128)


@pytest.mark.parametrize("n,ts,theta,kernel", [
    (1500, 128, [1.0, 0.1, 0.5], 0),
    (2100, 256, [1.3, 0.07, 0.73], 0),
    (1400, 128, [1.0, 0.1, 1.0, 0.01], 1),
])
def test_sliced_gradient_matches_fp64_adjoint(gpu, ora, n, ts, theta, kernel):
    """Gradient with the sliced factor, inverse factor and X X^T (precision 3)
    against the FP64 adjoint on the same field and against 4th-order finite
    differences of the oracle: within 1e-5 of max(|grad|, 1) (the inverse
    factor carries the ~2^-32 slicing error times the conditioning of L; the
    FP64 gradient meets 1e-6)."""
    x, y, z, _ = ora.synthetic_field(n, 3, theta, kernel)
    with gpu.Session(x, y, kernel=kernel, dts=ts) as s:
        s.set_data(z=z)
        ll64, g64 = s.loglik(theta, grad=True)
        s.set_sliced()
        ll, g = s.loglik(theta, grad=True)
        assert abs(ll - ll64) / abs(ll64) < 1e-7
        # the sliced value after a gradient evaluation is unaffected
        assert s.loglik(theta) == pytest.approx(ll, rel=1e-12)
    scale = max(np.abs(g64).max(), 1.0)
    assert np.abs(g - g64).max() / scale < 1e-5, (g, g64)
    h = 1e-4
    th = np.asarray(theta, dtype=float)
    fd = np.zeros_like(th)
    for i in range(th.size):
        e = np.zeros_like(th)
        e[i] = h * th[i]
        f = lambda t: ora.dmle(x, y, z, t, kernel)[0]
        fd[i] = (8 * (f(th + e) - f(th - e)) - (f(th + 2 * e) - f(th - 2 * e))) / (12 * e[i])
    assert np.abs(g - fd).max() / max(np.abs(fd).max(), 1.0) < 1e-5, (g, fd)
