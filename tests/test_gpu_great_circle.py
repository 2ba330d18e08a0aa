"""Great-circle distance (dm = "gc" / "gcd") through every GPU path against the
oracle: locations are (latitude, longitude) in degrees over a 10 x 10 degree
box, distances in km (distanceEarth, core_zcmg.c:51-60), beta in km.  Bars as
for the Euclidean tests: log-likelihood 1e-10, kriging 1e-9, gradient 1e-6 of
finite differences, Fisher 1e-8, MLOE / MMOM 1e-8, INT8-sliced 1e-7."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-10


def _latlon(n, seed):
    rng = np.random.default_rng(seed)
    return 20 + 10 * rng.random(n), 40 + 10 * rng.random(n)


@pytest.mark.parametrize("n,ts,theta,kernel", [
    (900, 128, [1.0, 100.0, 0.5], 0),
    (1300, 256, [1.3, 60.0, 0.73], 0),
    (700, 128, [1.0, 80.0, 1.0, 0.01], 1),
])
def test_loglik_great_circle(gpu, ora, n, ts, theta, kernel):
    lat, lon = _latlon(n, 1)
    _, _, z, _ = ora.synthetic_field(n, 2, theta, kernel, metric=1, locations=(lat, lon))
    ref = ora.dmle(lat, lon, z, theta, kernel, metric=1)[0]
    got = gpu.dmle_host(lat, lon, z, theta, kernel=kernel, metric=1, ts=ts)[0]
    assert got == pytest.approx(ref, rel=LL_RTOL)
    with gpu.Session(lat, lon, kernel=kernel, dm="gcd", dts=ts) as s:
        s.set_data(z=z)
        assert s.mle_alg(theta) == pytest.approx(ref, rel=LL_RTOL)


def test_prediction_and_gradient_great_circle(gpu, ora):
    theta = [1.0, 100.0, 0.5]
    lat, lon = _latlon(1000, 3)
    _, _, z, _ = ora.synthetic_field(1000, 3, theta, metric=1, locations=(lat, lon))
    m = np.zeros(1000, dtype=bool)
    m[np.random.default_rng(3).choice(1000, 80, replace=False)] = True
    mse_ref, zm_ref = ora.dpredict(lat[m], lon[m], lat[~m], lon[~m], z[~m], z[m], theta, metric=1)
    with gpu.Session(lat, lon, dm="gc", dts=128) as s:
        mse, zm = s.predict(theta, lat[m], lon[m], lat[~m], lon[~m], z[~m], z[m])
        assert np.allclose(zm, zm_ref, rtol=1e-9, atol=1e-12) and mse == pytest.approx(mse_ref, rel=1e-9)
        s.set_data(z=z)
        _, g = s.loglik(theta, grad=True)

    def f(t):
        return ora.dmle(lat, lon, z, t, metric=1)[0]

    th = np.asarray(theta)
    fd = np.zeros(3)
    for i in range(3):
        h = 1e-4 * th[i]
        e = np.zeros(3)
        e[i] = h
        fd[i] = (8 * (f(th + e) - f(th - e)) - (f(th + 2 * e) - f(th - 2 * e))) / (12 * h)
    assert np.abs(g - fd).max() / max(np.abs(fd).max(), 1.0) < 1e-6, (g, fd)


def test_fisher_and_mloe_great_circle(gpu, ora):
    theta = [1.0, 100.0, 0.5]
    lat, lon = _latlon(700, 4)
    F = gpu.fisher_host(lat, lon, theta, metric=1, ts=128)
    Fo, _ = ora.fisher(lat, lon, theta, metric=1)
    assert (np.abs(F - Fo) / np.sqrt(np.outer(np.diag(Fo), np.diag(Fo)))).max() < 1e-8
    lat, lon = _latlon(900, 5)
    est = [0.9, 120.0, 0.6]
    mloe, mmom, _, _ = gpu.mloe_mmom_host(lat[:100], lon[:100], lat[100:], lon[100:], theta, est, metric=1, ts=128)
    mo, mmo, _ = ora.mloe_mmom(lat[:100], lon[:100], lat[100:], lon[100:], theta, est, metric=1)
    assert mloe == pytest.approx(mo, abs=1e-8) and mmom == pytest.approx(mmo, abs=1e-8)


def test_sliced_great_circle(gpu, ora):
    theta = [1.0, 100.0, 0.5]
    lat, lon = _latlon(1500, 6)
    _, _, z, _ = ora.synthetic_field(1500, 6, theta, metric=1, locations=(lat, lon))
    ref = ora.dmle(lat, lon, z, theta, metric=1)[0]
    got = gpu.dmle_host_sliced(lat, lon, z, theta, metric=1, ts=128)[0]
    assert abs(got - ref) / abs(ref) < 1e-7


def test_batch_and_mixed_great_circle(gpu, ora):
    """Batched regional fields and the banded TF32 path with great-circle
    distance (per-field bar relative to the scale of the loglik terms, as in
    the Euclidean batch tests; mixed 1e-6)."""
    import math

    rng = np.random.default_rng(9)
    xs, ys, zs, th = [], [], [], []
    for f in range(8):
        n = int(rng.integers(300, 1200))
        lat0, lon0 = rng.uniform(-40, 40), rng.uniform(-120, 120)
        x, y = lat0 + 5 * rng.random(n), lon0 + 5 * rng.random(n)
        theta = [rng.uniform(0.5, 2.0), rng.uniform(30.0, 80.0), rng.uniform(0.3, 1.0)]
        zs.append(ora.dzvg(x, y, theta, rng.standard_normal(n), metric=1))
        xs.append(x), ys.append(y), th.append(theta)
    th = np.array(th)
    with gpu.Batch(xs, ys, zs, metric=1, ts=256) as b:
        got = b.loglik(th)
    for i in range(8):
        l, ld, dp, _ = ora.dmle(xs[i], ys[i], zs[i], th[i], metric=1)
        scale = 0.5 * abs(dp) + 0.5 * abs(ld) + 0.5 * len(xs[i]) * math.log(2 * math.pi)
        assert abs(got[i] - l) / scale < 1e-10
    theta = [1.0, 100.0, 0.5]
    lat, lon = _latlon(1300, 10)
    _, _, z, _ = ora.synthetic_field(1300, 10, theta, metric=1, locations=(lat, lon))
    ref = ora.dmle(lat, lon, z, theta, metric=1)[0]
    got = gpu.dmle_host_mixed(lat, lon, z, theta, metric=1, ts=256, band=1, passes=3)[0]
    assert abs(got - ref) / abs(ref) < 1e-6
