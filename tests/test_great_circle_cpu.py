"""Great-circle distance (dm = "gc", distanceEarth, core_zcmg.c:51-60) in the
oracle, pinned against an independent numpy haversine (no GPU)."""
import numpy as np


def _haversine_km(lat1, lon1, lat2, lon2):
    p1, p2 = np.radians(lat1), np.radians(lat2)
    a = np.sin((p2 - p1) / 2) ** 2 + np.cos(p1) * np.cos(p2) * np.sin(np.radians(lon2 - lon1) / 2) ** 2
    return 2 * 6371.0 * np.arcsin(np.sqrt(a))


def test_oracle_great_circle_covariance(ora):
    rng = np.random.default_rng(0)
    n = 200
    lat, lon = 20 + 10 * rng.random(n), 40 + 10 * rng.random(n)
    theta = [1.0, 100.0, 0.5]  # beta in km; nu = 1/2: exp(-d / beta)
    C = ora.covariance_full(lat, lon, theta, metric=1)
    d = _haversine_km(lat[:, None], lon[:, None], lat[None, :], lon[None, :])
    assert np.allclose(C, np.exp(-d / theta[1]), rtol=1e-13, atol=1e-300)
    # the metric is per call: the next Euclidean call is unaffected
    C0 = ora.covariance_full(lat, lon, theta)
    assert np.allclose(C0, np.exp(-np.hypot(lat[:, None] - lat, lon[:, None] - lon) / theta[1]), rtol=1e-13)
