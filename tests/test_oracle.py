"""The CPU oracle pinned against golden vectors (no GPU)."""
import json
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _kv_rows():
    with open(os.path.join(GOLD, "kv_mpmath.json")) as f:
        return json.load(f)["rows"]


def _ll_cases():
    with open(os.path.join(GOLD, "loglik_mpmath.json")) as f:
        return json.load(f)["cases"]


def test_oracle_knu_matches_mpmath(ora):
    worst = 0.0
    for r in _kv_rows():
        ref = float(r["k"])
        got = ora.bessel_knu(r["nu"], r["x"])
        worst = max(worst, abs(got - ref) / ref)
    # GSL documents ~1e-15 relative for gsl_sf_bessel_Knu; the restatement stays within 1e-14
    assert worst < 1e-14, worst


def test_oracle_knu_matches_scipy_second_opinion(ora):
    from scipy.special import kv

    for nu in (0.2, 0.5, 1.37, 3.9):
        for x in (1e-3, 0.4, 1.99, 2.01, 7.0, 90.0):
            assert ora.bessel_knu(nu, x) == pytest.approx(kv(nu, x), rel=1e-13)


@pytest.mark.parametrize("case", _ll_cases(), ids=lambda c: c["name"])
def test_oracle_locations_and_loglik_match_mpmath(ora, case):
    x, y = ora.generate_xy_loc(case["n"], case["seed"])
    # GenerateXYLoc restated twice (C oracle, Python golden script): bit-exact
    assert np.array_equal(x, np.array(case["x"])) and np.array_equal(y, np.array(case["y"]))
    ll, ld, dot, _ = ora.dmle(x, y, np.array(case["z"]), case["theta"], case["kernel"])
    assert ll == pytest.approx(float(case["loglik"]), rel=1e-11, abs=1e-9)
    assert ld == pytest.approx(float(case["logdet"]), rel=1e-10, abs=1e-9)
    assert dot == pytest.approx(float(case["dotp"]), rel=1e-10)


def test_generate_xy_loc_structure(ora):
    n = 1600
    x, y = ora.generate_xy_loc(n, 0)
    # quantised to 1/65535 and Morton ordered (MLE_misc.c:297-319)
    qx, qy = np.rint(x * 65535).astype(np.int64), np.rint(y * 65535).astype(np.int64)
    assert np.array_equal(qx / 65535.0, x) and np.array_equal(qy / 65535.0, y)

    def spread(v):
        out = np.zeros_like(v)
        for b in range(16):
            out |= ((v >> b) & 1) << (2 * b)
        return out

    code = (spread(qy) << 1) + spread(qx)
    assert np.all(np.diff(code) > 0)
    # jitter rule: every point within 0.4/40 (+ quantisation) of a grid centre
    g = np.sort((x * 40 - 0.5).round())
    assert len(set(zip(qx.tolist(), qy.tolist()))) == n


def test_truncated_grid(ora):
    # N = 100000 uses a 317 x 317 grid truncated at N (ceil(sqrt(N)) = 317)
    x, y = ora.generate_xy_loc(1000, 3)
    assert x.size == 1000 and np.all((x > 0) & (x < 1)) and np.all((y > 0) & (y < 1))


def test_dlarnv_reproducible(ora):
    from exageostat_b200.synthetic import dlarnv

    e1 = ora.dlarnv(0, 1000)
    e2 = dlarnv(0, 1000)
    assert np.array_equal(e1, e2)
    assert abs(e1.mean()) < 0.1 and abs(e1.std() - 1) < 0.1


def test_pick_random_points_partition(ora):
    N, nmiss = 400, 40
    x, y = ora.generate_xy_loc(N, 5)
    z = np.arange(N, dtype=float)
    split = ora.pick_random_points(x, y, z, nmiss, seed=5)
    allz = np.concatenate([split["z_actual"], split["z_obs"]])
    assert sorted(allz.tolist()) == z.tolist()
    # the values travel with their locations
    for zz, xx, yy in zip(split["z_obs"], split["x_obs"], split["y_obs"]):
        assert x[int(zz)] == xx and y[int(zz)] == yy


def test_oracle_zvg_is_l_times_e(ora):
    N = 200
    x, y = ora.generate_xy_loc(N, 1)
    e = ora.dlarnv(1, N)
    th = [1.0, 0.1, 0.5]
    z = ora.dzvg(x, y, th, e)
    C = ora.covariance_lower(x, y, th)
    C = C + np.tril(C, -1).T
    L = np.linalg.cholesky(C)
    assert np.allclose(z, L @ e, rtol=1e-12, atol=1e-12)


def test_oracle_predict_matches_numpy(ora):
    N, nmiss = 300, 30
    x, y = ora.generate_xy_loc(N, 2)
    th = [1.0, 0.1, 0.5]
    z = ora.dzvg(x, y, th, ora.dlarnv(2, N))
    s = ora.pick_random_points(x, y, z, nmiss, seed=2)
    mse, zm = ora.dpredict(s["x_miss"], s["y_miss"], s["x_obs"], s["y_obs"], s["z_obs"], s["z_actual"], th)
    C22 = ora.covariance_lower(s["x_obs"], s["y_obs"], th)
    C22 = C22 + np.tril(C22, -1).T
    C12 = ora.core_dcmg(nmiss, N - nmiss, 0, 0, s["x_miss"], s["y_miss"], s["x_obs"], s["y_obs"], th)
    ref = C12 @ np.linalg.solve(C22, s["z_obs"])
    assert np.allclose(zm, ref, rtol=1e-9, atol=1e-12)
    assert mse == pytest.approx(np.mean((s["z_actual"] - ref) ** 2), rel=1e-9)
