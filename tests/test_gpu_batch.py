"""Batches of independent fields (one graph launch per evaluation) against the
oracle, field by field (1e-10 relative)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
LL_RTOL = 1e-10


def _fields(ora, nfields, seed, nmin=300, nmax=2200):
    """Regional fields in the shape of the batched workload: sizes uniform in
    [nmin, nmax], locations uniform in each region's unit square, sigma2 in
    U(0.5, 2), beta in U(0.02, 0.3), nu in U(0.3, 2.5), z = L e."""
    rng = np.random.default_rng(seed)
    xs, ys, zs, th = [], [], [], []
    for f in range(nfields):
        n = int(rng.integers(nmin, nmax + 1))
        x, y = rng.random(n), rng.random(n)
        theta = [rng.uniform(0.5, 2.0), rng.uniform(0.02, 0.3), rng.uniform(0.3, 2.5)]
        z = ora.dzvg(x, y, theta, rng.standard_normal(n))
        xs.append(x), ys.append(y), zs.append(z), th.append(theta)
    return xs, ys, zs, np.array(th)


def test_batch_matches_oracle_per_field(gpu, ora):
    xs, ys, zs, th = _fields(ora, 24, 7)
    with gpu.Batch(xs, ys, zs, ts=256) as b:
        for trial in range(2):  # graph replay with new parameters
            th_t = th * (1.0 + 0.05 * trial)
            got = b.loglik(th_t)
            ref = np.array([ora.dmle(x, y, z, t)[0] for x, y, z, t in zip(xs, ys, zs, th_t)])
            assert np.allclose(got, ref, rtol=LL_RTOL, atol=0), np.abs(got - ref) / np.abs(ref)


def test_batch_isolates_a_failing_field(gpu, ora):
    xs, ys, zs, th = _fields(ora, 6, 3, 300, 900)
    xs[2] = xs[2].copy()
    xs[2][10] = np.nan
    with gpu.Batch(xs, ys, zs, ts=256) as b:
        got = b.loglik(th)
    assert got[2] == -np.inf
    ok = [i for i in range(6) if i != 2]
    ref = np.array([ora.dmle(xs[i], ys[i], zs[i], th[i])[0] for i in ok])
    assert np.allclose(got[ok], ref, rtol=LL_RTOL)


def test_batch_single_tile_fields_and_nugget(gpu, ora):
    rng = np.random.default_rng(11)
    xs, ys, zs, th = [], [], [], []
    for n in (1, 7, 128, 255, 256, 257, 600):
        x, y = rng.random(n), rng.random(n)
        t = [1.0, 0.1, 0.8, 0.02]
        xs.append(x), ys.append(y), zs.append(rng.standard_normal(n)), th.append(t)
    with gpu.Batch(xs, ys, zs, kernel=1, ts=256) as b:
        got = b.loglik(np.array(th))
    ref = np.array([ora.dmle(x, y, z, t, 1)[0] for x, y, z, t in zip(xs, ys, zs, th)])
    assert np.allclose(got, ref, rtol=LL_RTOL)
