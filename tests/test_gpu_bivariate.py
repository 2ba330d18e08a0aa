"""Bivariate parsimonious Matern (kernel_fun = "bivariate_matern_parsimonious",
theta = (sigma_1^2, sigma_2^2, beta, nu_1, nu_2, rho)) on the GPU against the
oracle: the generated covariance to 1e-13, the log-likelihood to 1e-10 (FP64)
and 1e-7 (INT8-sliced), synthetic z = L e to 1e-10, and the identity
loglik(rho = 0) = the sum of the two univariate log-likelihoods."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nloc,ts,theta", [
    (600, 128, [1.0, 2.0, 0.1, 0.5, 1.2, 0.4]),
    (1000, 256, [0.7, 1.3, 0.05, 1.0, 0.6, -0.3]),
])
def test_bivariate_covariance_and_loglik(gpu, ora, nloc, ts, theta):
    N = 2 * nloc
    x, y, z, _ = ora.synthetic_field(N, 4, theta, kernel=2)
    C = gpu.covariance_dense(x[:200], y[:200], theta, kernel=2, ts=128)  # the lower triangle
    Co = np.tril(ora.covariance_full(x[:200], y[:200], theta, kernel=2))
    assert np.abs(C - Co).max() < 1e-13 * np.abs(Co).max()
    ref = ora.dmle(x, y, z, theta, kernel=2)[0]
    assert gpu.dmle_host(x, y, z, theta, kernel=2, ts=ts)[0] == pytest.approx(ref, rel=1e-10)
    got = gpu.dmle_host_sliced(x, y, z, theta, kernel=2, ts=ts)[0]
    assert abs(got - ref) / abs(ref) < 1e-7


def test_bivariate_reference_workflow(gpu, ora):
    """EXAGEOSTAT_dmle_Call with N = 2 x locations, MLE_zvg, MLE_alg."""
    theta = [1.0, 2.0, 0.1, 0.5, 1.2, 0.4]
    N = 1400
    x, y, z_ref, e = ora.synthetic_field(N, 6, theta, kernel=2)
    with gpu.Session(x, y, kernel=2, dts=128) as s:
        assert s.N == N and s.nparams == 6
        s.zvg(theta, e)
        z = s.z()
        assert np.abs(z - z_ref).max() < 1e-10 * np.abs(z_ref).max()
        ref = ora.dmle(x, y, z_ref, theta, kernel=2)[0]
        assert s.mle_alg(theta) == pytest.approx(ref, rel=1e-10)
        s.set_sliced()
        assert abs(s.mle_alg(theta) - ref) / abs(ref) < 1e-7
        s.set_fp64()
        with pytest.raises(gpu.XgError) as ei:
            s.loglik(theta, grad=True)
        assert ei.value.code == gpu.XG_ERR_UNSUPPORTED
        with pytest.raises(gpu.XgError):
            s.fisher([1.0, 0.1, 0.5])


def test_bivariate_uncorrelated_is_two_univariate_fields(gpu, ora):
    theta = [1.3, 0.8, 0.1, 0.7, 1.1, 0.0]
    N = 1200
    x, y, z, _ = ora.synthetic_field(N, 5, theta, kernel=2)
    ll = gpu.dmle_host(x, y, z, theta, kernel=2, ts=128)[0]
    l0 = gpu.dmle_host(x, y, z[0::2], [theta[0], theta[2], theta[3]], ts=128)[0]
    l1 = gpu.dmle_host(x, y, z[1::2], [theta[1], theta[2], theta[4]], ts=128)[0]
    assert ll == pytest.approx(l0 + l1, rel=1e-11)


def test_bivariate_short_mle(gpu, ora):
    """The derivative-free maximiser runs on the 6-parameter objective."""
    theta = [1.0, 1.5, 0.1, 0.5, 0.8, 0.5]
    N = 800
    x, y, z, _ = ora.synthetic_field(N, 7, theta, kernel=2)
    lb, ub = [0.1, 0.1, 0.01, 0.1, 0.1, -0.9], [5, 5, 1, 3, 3, 0.9]
    with gpu.Session(x, y, kernel=2, dts=128) as s:
        s.set_data(z=z)
        th, f, ev = s.fit_bobyqa(lb, ub, x0=[1.0, 1.0, 0.2, 0.6, 0.6, 0.0], ftol_abs=1e-5, maxeval=300)
        assert np.isfinite(f) and ev > 10
        assert f >= s.mle_alg([1.0, 1.0, 0.2, 0.6, 0.6, 0.0])
        assert f == pytest.approx(ora.dmle(x, y, z, th, kernel=2)[0], rel=1e-10)


def test_bivariate_holdout_and_kriging(gpu, ora):
    """pick_random_points2 (bit-exact against the oracle with the same libc
    draws) and kriging of both variables through EXAGEOSTAT_dmle_Predict_Tile
    with the row counts 2 nZmiss, 2 nZobs (1e-9), with the per-variable
    errors in data.mserror1 / mserror2 and results.mse_pred1 / _pred2."""
    import ctypes

    libc = ctypes.CDLL(None)
    theta = [1.0, 2.0, 0.1, 0.5, 1.2, 0.4]
    nloc, nmiss = 600, 50
    x, y, z_ref, e = ora.synthetic_field(2 * nloc, 8, theta, kernel=2)
    P = ctypes.POINTER(ctypes.c_double)
    with gpu.Session(x, y, kernel=2, dts=128) as s:
        s.zvg(theta, e)
        z = s.z()
        zobs, zact = np.empty(2 * (nloc - nmiss)), np.empty(2 * nmiss)
        libc.srand(11)
        s.L.pick_random_points2(ctypes.byref(s.data), zobs.ctypes.data_as(P), zact.ctypes.data_as(P), nmiss,
                                nloc - nmiss, 2 * nloc)
        xm = np.ctypeslib.as_array(s.data.lmiss.x, (nmiss,)).copy()
        ym = np.ctypeslib.as_array(s.data.lmiss.y, (nmiss,)).copy()
        xo = np.ctypeslib.as_array(s.data.lobs.x, (nloc - nmiss,)).copy()
        yo = np.ctypeslib.as_array(s.data.lobs.y, (nloc - nmiss,)).copy()
        libc.srand(11)
        ref = ora.pick_random_points2(x, y, z, nmiss)
        for a, b in ((xm, "x_miss"), (ym, "y_miss"), (xo, "x_obs"), (yo, "y_obs"), (zobs, "z_obs"),
                     (zact, "z_actual")):
            assert np.array_equal(a, ref[b]), b
        mse, zmiss = s.predict(theta, xm, ym, xo, yo, zobs, zact)
        res = gpu.Output.in_dll(gpu.lib(), "results")
        m1, m2 = s.data.mserror1, s.data.mserror2
        assert (res.mse_pred1, res.mse_pred2) == (m1, m2)
    mse_ref, zm_ref = ora.dpredict(xm, ym, xo, yo, zobs, zact, theta, kernel=2)
    assert zmiss.size == 2 * nmiss
    assert np.allclose(zmiss, zm_ref, rtol=1e-9, atol=1e-12)
    assert mse == pytest.approx(mse_ref, rel=1e-9)
    assert m1 == pytest.approx(np.mean((zact[0::2] - zm_ref[0::2]) ** 2), rel=1e-9)
    assert m2 == pytest.approx(np.mean((zact[1::2] - zm_ref[1::2]) ** 2), rel=1e-9)


# kernel_fun = "bivariate_matern_flexible" (core_zcmg.c:1514-1580), 11
# parameters; theta[8], theta[9] chosen so that the Matern terms tend to
# theta[0], theta[1] at zero distance (the reference stores those there), which
# keeps these covariances positive definite
FLEX = [
    [0.1, 0.15, 0.5, 0.5, 0.8, 1.2, 0.3, 0.5, 3.68961, 6.95741, 0.3],
    [0.08, 0.12, 1.0, 0.2, 0.5, 1.0, 0.2, 0.8, 1.24479, 4.41137, -0.4],
]


@pytest.mark.parametrize("theta", FLEX)
def test_flexible_bivariate_covariance_loglik_and_workflow(gpu, ora, theta):
    nloc = 700
    N = 2 * nloc
    x, y, z_ref, e = ora.synthetic_field(N, 8, theta, kernel=3)
    C = gpu.covariance_dense(x[:200], y[:200], theta, kernel=3, ts=128)
    Co = np.tril(ora.covariance_full(x[:200], y[:200], theta, kernel=3))
    assert np.abs(C - Co).max() < 1e-13 * np.abs(Co).max()
    ref = ora.dmle(x, y, z_ref, theta, kernel=3)[0]
    assert gpu.dmle_host(x, y, z_ref, theta, kernel=3, ts=256)[0] == pytest.approx(ref, rel=1e-10)
    with gpu.Session(x, y, kernel=3, dts=128) as s:
        assert s.N == N and s.nparams == 11
        s.zvg(theta, e)
        z = s.z()
        assert np.abs(z - z_ref).max() < 1e-10 * np.abs(z_ref).max()
        assert s.mle_alg(theta) == pytest.approx(ref, rel=1e-10)
        s.set_sliced()
        assert abs(s.mle_alg(theta) - ref) / abs(ref) < 1e-7
