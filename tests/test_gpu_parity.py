"""GPU parity: every kernel on the exact path against the CPU oracle and the
mpmath golden vectors.  Tolerances: K_nu 1e-14 relative (mpmath); Matern
elements 1e-13; log-likelihood 1e-10 relative (the bar the path is built to);
Cholesky factor / z / kriging 1e-9 relative in the norm (conditioning of the
covariance enters)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
LL_RTOL = 1e-10


def _rows():
    with open(os.path.join(GOLD, "kv_mpmath.json")) as f:
        return json.load(f)["rows"]


def _ll_cases():
    with open(os.path.join(GOLD, "loglik_mpmath.json")) as f:
        return json.load(f)["cases"]


def test_device_knu_matches_mpmath(gpu):
    rows = _rows()
    nu = np.array([r["nu"] for r in rows])
    x = np.array([r["x"] for r in rows])
    ref = np.array([float(r["k"]) for r in rows])
    got = gpu.bessel_knu(nu, x)
    rel = np.abs(got - ref) / ref
    assert rel.max() < 1e-14, (rel.max(), rows[int(rel.argmax())])


@pytest.mark.parametrize("theta,kernel", [([1.0, 0.1, 0.5], 0), ([1.3, 0.07, 0.73], 0), ([0.8, 0.3, 1.5], 0),
                                          ([1.0, 0.05, 2.5], 0), ([2.0, 0.2, 3.3], 0), ([1.0, 0.1, 1.0, 0.01], 1),
                                          ([0.7, 4.9, 0.011], 0), ([1.0, 0.011, 4.99], 0)])
def test_matern_elements_match_oracle(gpu, ora, theta, kernel):
    rng = np.random.default_rng(1)
    n = 4000
    x1, y1, x2, y2 = (rng.random(n) for _ in range(4))
    x2[:10], y2[:10] = x1[:10], y1[:10]  # zero-distance branch
    got = gpu.matern_pairs(x1, y1, x2, y2, theta, kernel)
    ref = np.array([ora.core_dcmg(1, 1, 0, 0, x1[i:i + 1], y1[i:i + 1], x2[i:i + 1], y2[i:i + 1], theta, kernel)[0, 0]
                    for i in range(n)])
    scale = np.maximum(np.abs(ref), 1e-300)
    rel = np.abs(got - ref) / scale
    big = np.abs(ref) > 1e-250
    assert rel[big].max() < 1e-13, rel[big].max()


@pytest.mark.parametrize("n,ts", [(300, 128), (640, 256), (700, 512)])
def test_covariance_tiles_match_oracle(gpu, ora, n, ts):
    x, y = ora.generate_xy_loc(n, 3)
    theta = [1.0, 0.1, 0.73]
    got = gpu.covariance_dense(x, y, theta, ts=ts)
    ref = ora.covariance_lower(x, y, theta)
    assert np.allclose(got, ref, rtol=1e-13, atol=1e-300)


@pytest.mark.parametrize("n,ts", [(300, 128), (1000, 256), (1300, 512)])
def test_cholesky_factor_matches_lapack(gpu, ora, n, ts):
    x, y = ora.generate_xy_loc(n, 4)
    theta = [1.0, 0.1, 0.5]
    L = gpu.covariance_dense(x, y, theta, ts=ts, factor=True)
    C = ora.covariance_lower(x, y, theta)
    C = C + np.tril(C, -1).T
    Lref = np.linalg.cholesky(C)
    assert np.linalg.norm(L - Lref) / np.linalg.norm(Lref) < 1e-11
    # factorisation residual (the reference's check_factorization idea, LAPACKE_MLE.c:589-648)
    res = np.abs(L @ L.T - C).max() / (np.abs(C).max() * n * np.finfo(float).eps)
    assert res < 60


def test_zvg_matches_oracle_across_tile_sizes(gpu, ora):
    """z = L e (TRMV over full stored tiles): exercises the zeroed upper
    triangle of the diagonal tiles."""
    from exageostat_b200.synthetic import dlarnv

    N = 1000
    x, y = ora.generate_xy_loc(N, 6)
    e = dlarnv(6, N)
    th = [1.0, 0.1, 0.5]
    zref = ora.dzvg(x, y, th, e)
    for ts in (128, 256, 512):
        with gpu.Session(x, y, dts=ts) as s:
            s.zvg(th, e)
            z = s.z()
        assert np.linalg.norm(z - zref) / np.linalg.norm(zref) < 1e-11, ts


@pytest.mark.parametrize("case", _ll_cases(), ids=lambda c: c["name"])
@pytest.mark.parametrize("ts", [128, 256])
def test_loglik_matches_mpmath_golden(gpu, case, ts):
    ll, ld, dot = gpu.dmle_host(case["x"], case["y"], case["z"], case["theta"], case["kernel"], ts=ts)
    assert ll == pytest.approx(float(case["loglik"]), rel=1e-11, abs=1e-9)
    assert ld == pytest.approx(float(case["logdet"]), rel=1e-10, abs=1e-9)
    assert dot == pytest.approx(float(case["dotp"]), rel=1e-10)


def _synthetic(ora, n, seed, theta, kernel=0):
    from exageostat_b200.synthetic import dlarnv

    x, y = ora.generate_xy_loc(n, seed)
    e = dlarnv(seed, n)
    z = ora.dzvg(x, y, theta, e, kernel)
    return x, y, z, e


@pytest.mark.parametrize("dts", [0, 128, 320, 512])
def test_config_c1_loglik_matches_oracle(gpu, ora, dts):
    """N = 1600 (40 x 40 jittered grid), theta = (1, 0.1, 0.5), the reference's
    tile size 320 among others (rounded up to a multiple of 128)."""
    x, y, z, _ = _synthetic(ora, 1600, 0, [1.0, 0.1, 0.5])
    for theta in ([1.0, 0.1, 0.5], [0.5, 0.3, 0.9], [2.0, 0.05, 0.73], [1.2, 0.02, 2.5]):
        ref = ora.dmle(x, y, z, theta)[0]
        got = gpu.dmle_host(x, y, z, theta, ts=dts)[0]
        assert got == pytest.approx(ref, rel=LL_RTOL), (theta, got, ref)


def test_ragged_and_tiny_sizes(gpu, ora):
    for n in (1, 2, 17, 129, 255, 513):
        x, y = ora.generate_xy_loc(n, 9)
        z = np.random.default_rng(n).standard_normal(n)
        theta = [1.0, 0.2, 0.5]
        ref = ora.dmle(x, y, z, theta)[0]
        for ts in (128, 256):
            got = gpu.dmle_host(x, y, z, theta, ts=ts)[0]
            assert got == pytest.approx(ref, rel=LL_RTOL), (n, ts)


def test_nugget_kernel_matches_oracle(gpu, ora):
    theta = [1.0, 0.1, 1.0, 0.01]
    x, y, z, _ = _synthetic(ora, 2000, 1, theta, kernel=1)
    for th in (theta, [0.8, 0.2, 0.6, 0.05]):
        ref = ora.dmle(x, y, z, th, 1)[0]
        got = gpu.dmle_host(x, y, z, th, kernel=1, ts=256)[0]
        assert got == pytest.approx(ref, rel=LL_RTOL)


def test_reference_workflow_session(gpu, ora):
    """exageostat_init -> EXAGEOSTAT_dmle_Call -> MLE_zvg -> MLE_alg ->
    pick_random_points -> EXAGEOSTAT_dmle_Predict_Tile, against the oracle
    running the same workflow (synthetic_dmle_test.c:136-494)."""
    from exageostat_b200.synthetic import dlarnv

    N, nmiss, seed = 1600, 100, 0
    theta0 = [1.0, 0.1, 0.5]
    x, y = gpu.generate_xy_loc(N, seed)
    e = dlarnv(seed, N)
    with gpu.Session(x, y, dts=320) as s:
        s.zvg(theta0, e)
        z = s.z()
        zref = ora.dzvg(x, y, theta0, e)
        assert np.linalg.norm(z - zref) / np.linalg.norm(zref) < 1e-11
        for th in ([1.0, 0.1, 0.5], [0.9, 0.12, 0.45]):
            got = s.mle_alg(th)
            ref = ora.dmle(x, y, z, th)[0]
            assert got == pytest.approx(ref, rel=LL_RTOL)
        assert s.data.iter_count == 2
        assert s.data.final_loglik == pytest.approx(got)
        split = ora.pick_random_points(x, y, z, nmiss, seed=seed)
        mse, zm = s.predict(theta0, split["x_miss"], split["y_miss"], split["x_obs"], split["y_obs"],
                            split["z_obs"], split["z_actual"])
        mref, zmref = ora.dpredict(split["x_miss"], split["y_miss"], split["x_obs"], split["y_obs"], split["z_obs"],
                                   split["z_actual"], theta0)
        assert np.linalg.norm(zm - zmref) / np.linalg.norm(zmref) < 1e-9
        assert mse == pytest.approx(mref, rel=1e-9)
        mse2, _ = s.predict(theta0, split["x_miss"], split["y_miss"], split["x_obs"], split["y_obs"],
                            split["z_obs"], None)
        assert mse2 == -1


def test_library_pick_random_points_matches_oracle(gpu, ora):
    """pick_random_points through the library (z from the device) equals the
    oracle split when both continue the same libc rand() stream."""
    import ctypes

    from exageostat_b200.synthetic import dlarnv

    N, nmiss, seed = 900, 90, 4
    theta0 = [1.0, 0.1, 0.5]
    x, y = gpu.generate_xy_loc(N, seed)  # leaves libc rand() after 2N draws
    e = dlarnv(seed, N)
    with gpu.Session(x, y) as s:
        s.zvg(theta0, e)
        z = s.z()
        zobs, zact = np.empty(N - nmiss), np.empty(nmiss)
        P = ctypes.POINTER(ctypes.c_double)
        gpu.lib().pick_random_points(ctypes.byref(s.data), zobs.ctypes.data_as(P), zact.ctypes.data_as(P), nmiss,
                                     N - nmiss, N)
        split = ora.pick_random_points(x, y, z, nmiss, seed=seed)
        assert np.array_equal(zobs, split["z_obs"]) and np.array_equal(zact, split["z_actual"])
        xo = np.ctypeslib.as_array(s.data.lobs.x, shape=(N - nmiss,))
        assert np.array_equal(xo, split["x_obs"])


def test_not_spd_reports_error_and_context_survives(gpu, ora):
    """A NaN location makes a pivot NaN: the library reports a non-positive-
    definite covariance (the reference exits, MLE_misc.h:343-348) and the next
    evaluation on the same context still works."""
    x, y = ora.generate_xy_loc(400, 2)
    x[150] = np.nan
    z = np.ones(400)
    with pytest.raises(gpu.XgError) as ei:
        gpu.dmle_host(x, y, z, [1.0, 0.1, 0.5], ts=128)
    assert ei.value.code == gpu.XG_ERR_NOT_SPD
    with gpu.Session(x, y, dts=128) as s:
        s.set_data(z=z)
        assert s.mle_alg([1.0, 0.1, 0.5]) == -np.inf
        assert s.data.final_loglik == -np.inf
    x2, y2 = ora.generate_xy_loc(400, 2)
    ref = ora.dmle(x2, y2, z, [1.0, 0.1, 0.5])[0]
    assert gpu.dmle_host(x2, y2, z, [1.0, 0.1, 0.5], ts=128)[0] == pytest.approx(ref, rel=LL_RTOL)


def test_duplicate_locations_do_not_crash(gpu, ora):
    """Exactly repeated locations make Sigma singular in exact arithmetic; the
    rounded pivot may come out on either side of zero (as in LAPACK), so the
    call either reports NOT_SPD or returns a finite value."""
    x, y = ora.generate_xy_loc(400, 2)
    x[5], y[5] = x[6], y[6]
    try:
        ll = gpu.dmle_host(x, y, np.ones(400), [1.0, 0.1, 0.5], ts=128)[0]
        assert np.isfinite(ll)
    except gpu.XgError as e:
        assert e.code == gpu.XG_ERR_NOT_SPD


def test_bad_theta_is_rejected(gpu, ora):
    x, y = ora.generate_xy_loc(100, 2)
    for th in ([np.nan, 0.1, 0.5], [1.0, -0.1, 0.5], [1.0, 0.1, 0.0]):
        with pytest.raises(gpu.XgError) as ei:
            gpu.dmle_host(x, y, np.ones(100), th)
        assert ei.value.code == gpu.XG_ERR_BAD_ARGUMENT


def test_profile_counts_launches(gpu, ora):
    x, y, z, _ = _synthetic(ora, 1100, 5, [1.0, 0.1, 0.5])
    with gpu.Session(x, y, dts=256) as s:
        s.set_data(z=z)
        s.set_profiling(True)
        s.loglik([1.0, 0.1, 0.5])
        p = s.profile()
        nt = 5
        potrf = 3 * (256 // 128) - 2  # the sub-block POTRF sequence of a 256 tile
        assert p["nt"] == nt and p["launches"] == nt * potrf + 3 * nt - 2 and p["evals"] == 1
        assert p["t_gemm"] > 0 and p["gemm_flops"] > 0


@pytest.mark.slow
def test_config_ctest_size_6400(gpu, ora):
    """N = 6400 (the reference CTest size), nu = 0.73 general Bessel path."""
    x, y, z, _ = _synthetic(ora, 6400, 0, [1.0, 0.1, 0.5])
    for th in ([1.0, 0.1, 0.73], [1.0, 0.1, 0.5]):
        ref = ora.dmle(x, y, z, th)[0]
        for ts in (256, 512):
            got = gpu.dmle_host(x, y, z, th, ts=ts)[0]
            assert got == pytest.approx(ref, rel=LL_RTOL)
