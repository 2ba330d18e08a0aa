"""Banded mixed precision (precision = 2) against the FP64 path and the
oracle.  Bars: band tiles of the factor 1e-11; off-band (FP32-stored) tiles
1e-5 of max |L|; log-likelihood |dl|/|l| <= 1e-6 with three TF32 passes
(the accuracy target for reduced precision), reported and bounded by 1e-4 with
one pass."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,ts,band,passes", [(1000, 256, 1, 3), (1300, 256, 2, 3), (1100, 256, 1, 1),
                                              (1500, 512, 1, 3)])
def test_mixed_factor_matches_lapack(gpu, ora, n, ts, band, passes):
    x, y = ora.generate_xy_loc(n, 4)
    theta = [1.0, 0.1, 0.5]
    L = gpu.mixed_factor_dense(x, y, theta, ts=ts, band=band, passes=passes)
    C = ora.covariance_lower(x, y, theta)
    C = C + np.tril(C, -1).T
    Lref = np.linalg.cholesky(C)
    scale = np.abs(Lref).max()
    nt = (n + ts - 1) // ts
    rows = np.arange(n) // ts
    inband = (rows[:, None] - rows[None, :]) < band
    err_band = np.abs(L - Lref)[inband & (np.arange(n)[:, None] >= np.arange(n)[None, :])].max() / scale
    err_off = np.abs(L - Lref)[~inband].max() / scale if nt > band else 0.0
    assert err_off < (1e-5 if passes == 3 else 2e-3), err_off
    # band tiles inherit the FP32 rounding of their off-band operands from
    # earlier steps, so they are only FP32-accurate too, except the first band
    assert err_band < (1e-5 if passes == 3 else 2e-3), err_band


@pytest.mark.parametrize("band", [1, 2])
def test_mixed_loglik_within_1e6_of_fp64(gpu, ora, band):
    n = 3000
    theta = [1.0, 0.05, 0.5]
    x, y, z, _ = ora.synthetic_field(n, 0, theta)
    ref = ora.dmle(x, y, z, theta)[0]
    got = gpu.dmle_host_mixed(x, y, z, theta, ts=256, band=band, passes=3)[0]
    assert abs(got - ref) / abs(ref) < 1e-6, (got, ref)
    one = gpu.dmle_host_mixed(x, y, z, theta, ts=256, band=band, passes=1)[0]
    assert abs(one - ref) / abs(ref) < 1e-4, (one, ref)


def test_mixed_through_mle_alg(gpu, ora):
    """A smooth field (nu = 1.5, cond(Sigma) ~ 3e6) needs a wider FP64 band for
    1e-6: FP32 off-band storage alone costs ~4e-6 at band 2 here (the same as
    the reference's FP32 off-band scheme)."""
    n = 2100
    theta = [1.0, 0.1, 1.5]
    x, y, z, _ = ora.synthetic_field(n, 2, theta)
    with gpu.Session(x, y, dts=256) as s:
        s.set_data(z=z)
        fp64 = s.mle_alg(theta)
        s.set_mixed(band=4, passes=3)
        assert s.data.precision == 2 and s.data.diag_thick == 4
        mixed = s.mle_alg(theta)
        assert abs(mixed - fp64) / abs(fp64) < 1e-6
        assert gpu.lib().EXAGEOSTAT_sdmle_Tile(3, np.asarray(theta).ctypes.data_as(
            __import__("ctypes").POINTER(__import__("ctypes").c_double)), None,
            __import__("ctypes").cast(__import__("ctypes").byref(s.data), __import__("ctypes").c_void_p)) == \
            pytest.approx(mixed, rel=1e-13)
        s.set_fp64()
        assert s.mle_alg(theta) == pytest.approx(fp64, rel=1e-14)


def test_mixed_nugget_and_general_nu(gpu, ora):
    theta = [1.0, 0.1, 0.73, 0.01]
    x, y, z, _ = ora.synthetic_field(1800, 5, theta, kernel=1)
    ref = ora.dmle(x, y, z, theta, 1)[0]
    got = gpu.dmle_host_mixed(x, y, z, theta, kernel=1, ts=256, band=1, passes=3)[0]
    assert abs(got - ref) / abs(ref) < 1e-6
