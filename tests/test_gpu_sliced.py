"""FP64 tiles with INT8-sliced off-band updates (precision = 3) against
LAPACK and the oracle.  The off-band update is an exact integer product of
operands carried to ~32 bits relative to their row maximum, so the factor
stays within 1e-8 of LAPACK's (relative to max |L|) and the log-likelihood
within 1e-7 relative; the north-star bar for reduced precision is 1e-6."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,ts,band", [(700, 128, 1), (1300, 256, 1), (1300, 256, 2), (2100, 512, 1)])
def test_sliced_factor_matches_lapack(gpu, ora, n, ts, band):
    x, y = ora.generate_xy_loc(n, 4)
    theta = [1.0, 0.1, 0.5]
    L = gpu.sliced_factor_dense(x, y, theta, ts=ts, band=band)
    C = ora.covariance_lower(x, y, theta)
    C = C + np.tril(C, -1).T
    Lref = np.linalg.cholesky(C)
    err = np.abs(L - Lref).max() / np.abs(Lref).max()
    assert err < 1e-8, err
    assert np.all(np.triu(L, 1) == 0)


@pytest.mark.parametrize("band", [1, 2])
def test_sliced_loglik_close_to_oracle(gpu, ora, band):
    n = 3000
    theta = [1.0, 0.05, 0.5]
    x, y, z, _ = ora.synthetic_field(n, 0, theta)
    ref = ora.dmle(x, y, z, theta)[0]
    got = gpu.dmle_host_sliced(x, y, z, theta, ts=256, band=band)[0]
    assert abs(got - ref) / abs(ref) < 1e-7, (got, ref)


def test_sliced_smooth_field_through_mle_alg(gpu, ora):
    """nu = 1.5, cond(Sigma) ~ 3e6: the FP32 off-band scheme needs a band of
    4 tiles for 1e-6 here; the sliced updates meet it at band 1."""
    n = 2100
    theta = [1.0, 0.1, 1.5]
    x, y, z, _ = ora.synthetic_field(n, 2, theta)
    with gpu.Session(x, y, dts=256) as s:
        s.set_data(z=z)
        fp64 = s.mle_alg(theta)
        s.set_sliced(band=1)
        assert s.data.precision == 3 and s.data.diag_thick == 1
        sl = s.mle_alg(theta)
        assert abs(sl - fp64) / abs(fp64) < 1e-7, (sl, fp64)
        s.set_fp64()
        assert s.mle_alg(theta) == pytest.approx(fp64, rel=1e-14)


def test_sliced_nugget_and_general_nu(gpu, ora):
    theta = [1.0, 0.1, 0.73, 0.01]
    x, y, z, _ = ora.synthetic_field(1800, 5, theta, kernel=1)
    ref = ora.dmle(x, y, z, theta, 1)[0]
    got = gpu.dmle_host_sliced(x, y, z, theta, kernel=1, ts=128, band=1)[0]
    assert abs(got - ref) / abs(ref) < 1e-7, (got, ref)


def test_sliced_rejects_non_spd(gpu, ora):
    x, y = ora.generate_xy_loc(600, 1)
    x = x.copy()
    x[5] = np.nan
    z = np.ones(600)
    with pytest.raises(gpu.XgError):
        gpu.dmle_host_sliced(x, y, z, [1.0, 0.1, 0.5], ts=128)
