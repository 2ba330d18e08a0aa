"""Fisher information and MLOE / MMOM on the GPU against the oracle.

Bars: Fisher entries within 1e-8 of sqrt(F_jj F_kk) (1e-6 for the smooth
nu = 1.5 field, whose Sigma has cond ~1e8); F_{sigma^2 sigma^2} = N / (2 sigma^4)
to 1e-9; per-point MLOE / MMOM terms within 1e-9 sigma^2 and the means within
1e-8; the identities MLOE = MMOM = 0 (estimate = truth) and MLOE = 0,
MMOM = c - 1 (variance scaled by c) to 1e-9."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,ts,theta,kernel,tol", [
    (600, 128, [1.0, 0.1, 0.5], 0, 1e-8),
    (900, 256, [1.3, 0.07, 0.73], 0, 1e-8),
    (700, 128, [0.8, 0.1, 1.5], 0, 1e-6),
    (800, 128, [1.0, 0.1, 1.0, 0.01], 1, 1e-8),
    (1100, 512, [1.0, 0.05, 0.5], 0, 1e-8),
])
def test_fisher_matches_oracle(gpu, ora, n, ts, theta, kernel, tol):
    x, y = ora.generate_xy_loc(n, 5)
    F = gpu.fisher_host(x, y, theta, kernel=kernel, ts=ts)
    Fo, _ = ora.fisher(x, y, theta, kernel)
    scale = np.sqrt(np.outer(np.diag(Fo), np.diag(Fo)))
    assert (np.abs(F - Fo) / scale).max() < tol, (F, Fo)
    assert np.array_equal(F, F.T)
    if kernel == 0:
        assert F[0, 0] == pytest.approx(n / (2 * theta[0] ** 2), rel=1e-9)


def test_fisher_reference_entry_points(gpu, ora):
    """EXAGEOSTAT_Fisher_Tile returns the inverse (10 doubles, column-major)
    and fills results.fisher_*; a log-likelihood and a gradient afterwards are
    unaffected."""
    theta = [1.0, 0.1, 0.5]
    x, y, z, _ = ora.synthetic_field(640, 0, theta)
    with gpu.Session(x, y, dts=128) as s:
        s.set_data(z=z)
        ll0 = s.loglik(theta)
        F, Finv = s.fisher(theta)
        inv = s.fisher_tile(theta)
        res = gpu.Output.in_dll(gpu.lib(), "results")
        assert (res.fisher_00, res.fisher_11, res.fisher_22) == (inv[0, 0], inv[1, 1], inv[2, 2])
        assert res.fisher_time > 0
        assert s.loglik(theta) == pytest.approx(ll0, rel=1e-13)
        _, g_after = s.loglik(theta, grad=True)  # the gradient after a Fisher call
    with gpu.Session(x, y, dts=128) as s2:
        s2.set_data(z=z)
        _, g_fresh = s2.loglik(theta, grad=True)
    assert np.allclose(g_after, g_fresh, rtol=1e-12, atol=0)
    Fo, Fio = ora.fisher(x, y, theta)
    assert np.allclose(F, Fo, rtol=1e-8)
    assert np.allclose(inv, Fio, rtol=1e-6)
    assert np.allclose(Finv, inv, rtol=1e-12)


def _split(ora, n, nmiss, seed):
    x, y = ora.generate_xy_loc(n, seed)
    perm = np.random.default_rng(seed).permutation(n)
    m, o = perm[:nmiss], perm[nmiss:]
    return x[m], y[m], x[o], y[o]


@pytest.mark.parametrize("nobs,nmiss,ts,truth,est,kernel", [
    (900, 100, 128, [1.0, 0.1, 0.5], [0.9, 0.08, 0.6], 0),
    (1500, 300, 256, [1.3, 0.07, 0.73], [1.1, 0.1, 0.9], 0),
    (700, 64, 128, [1.0, 0.1, 1.0, 0.01], [1.2, 0.12, 0.8, 0.02], 1),
    (1300, 1, 512, [1.0, 0.1, 0.5], [2.0, 0.3, 0.5], 0),
])
def test_mloe_mmom_matches_oracle(gpu, ora, nobs, nmiss, ts, truth, est, kernel):
    xm, ym, xo, yo = _split(ora, nobs + nmiss, nmiss, 6)
    mloe, mmom, terms, times = gpu.mloe_mmom_host(xm, ym, xo, yo, truth, est, kernel=kernel, ts=ts)
    mo, mmo, to = ora.mloe_mmom(xm, ym, xo, yo, truth, est, kernel)
    assert np.abs(terms[:, :4] - to[:, :4]).max() < 1e-9 * truth[0]
    assert np.abs(terms[:, 4:] - to[:, 4:]).max() < 1e-8
    assert mloe == pytest.approx(mo, abs=1e-8) and mmom == pytest.approx(mmo, abs=1e-8)
    assert np.all(times > 0)


def test_mloe_mmom_identities_on_gpu(gpu, ora):
    xm, ym, xo, yo = _split(ora, 1200, 150, 7)
    theta = [1.3, 0.1, 0.7]
    mloe, mmom, _, _ = gpu.mloe_mmom_host(xm, ym, xo, yo, theta, theta, ts=256)
    assert abs(mloe) < 1e-9 and abs(mmom) < 1e-9
    c = 2.5
    mloe, mmom, _, _ = gpu.mloe_mmom_host(xm, ym, xo, yo, theta, [c * theta[0], theta[1], theta[2]], ts=256)
    assert abs(mloe) < 1e-9 and mmom == pytest.approx(c - 1, abs=1e-9)


def test_mloe_mmom_reference_entry_points(gpu, ora):
    """mloe_mmom_init + EXAGEOSTAT_dmle_mloe_mmom_Tile(_Async) + mloe_mmom_finalize
    on data.lobs / data.lmiss: data.mloe / mmom and results.mloe / mmom."""
    x, y = ora.generate_xy_loc(1000, 3)
    xm, ym, xo, yo = _split(ora, 1000, 120, 3)
    truth, est = [1.0, 0.1, 0.5], [0.8, 0.13, 0.55]
    with gpu.Session(x, y, dts=128) as s:
        m_sync = s.mloe_mmom(truth, est, xm, ym, xo, yo)
        res = gpu.Output.in_dll(gpu.lib(), "results")
        assert (res.mloe, res.mmom) == m_sync and res.mloe_exec == b"sync"
        m_async = s.mloe_mmom(truth, est, xm, ym, xo, yo, asynchronous=True)
        assert res.mloe_exec == b"async"
        assert res.total_mloe_mmom_time > 0 and res.cho_fact_mloe_mmom_time > 0
    assert m_async == pytest.approx(m_sync, rel=1e-13)
    mo, mmo, _ = ora.mloe_mmom(xm, ym, xo, yo, truth, est)
    assert m_sync == pytest.approx((mo, mmo), abs=1e-8)


def test_mloe_mmom_non_spd_is_an_error(gpu, ora):
    """A NaN observed location makes a pivot NaN: an error status (the
    reference exits, MLE_dexact.c:1253), and the context stays usable."""
    xm, ym, xo, yo = _split(ora, 600, 50, 8)
    xo = xo.copy()
    keep = xo[10]
    xo[10] = np.nan
    with pytest.raises(gpu.XgError) as ei:
        gpu.mloe_mmom_host(xm, ym, xo, yo, [1.0, 0.1, 0.5], [1.0, 0.1, 0.5], ts=128)
    assert ei.value.code == gpu.XG_ERR_NOT_SPD
    xo[10] = keep
    x, y = ora.generate_xy_loc(300, 8)
    with pytest.raises(gpu.XgError):
        bad = x.copy()
        bad[7] = np.nan
        gpu.fisher_host(bad, y, [1.0, 0.1, 0.5], ts=128)
    mloe, mmom, _, _ = gpu.mloe_mmom_host(xm, ym, xo, yo, [1.0, 0.1, 0.5], [1.0, 0.1, 0.5], ts=128)
    assert abs(mloe) < 1e-9
