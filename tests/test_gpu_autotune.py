"""Autotuner: tile size (and band width for the banded scheme) chosen by
timing; the rebuilt descriptors must give the same log-likelihood."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_fp64_field_keeps_the_value(gpu, ora):
    theta = [1.0, 0.1, 0.5]
    x, y, z, _ = ora.synthetic_field(3000, 1, theta)
    ref = ora.dmle(x, y, z, theta)[0]
    with gpu.Session(x, y, dts=128) as s:
        s.set_data(z=z)
        ts, band, rep = s.autotune(theta)
        assert ts in (128, 256, 384, 512) and band == 0
        assert len(rep) >= 2 and all(sec > 0 for _, sec in rep)
        assert ts == min(rep, key=lambda r: r[1])[0]
        assert s.mle_alg(theta) == pytest.approx(ref, rel=1e-10)


def test_autotune_banded_scheme_picks_a_band_within_tolerance(gpu, ora):
    theta = [1.0, 0.1, 0.5]
    x, y, z, _ = ora.synthetic_field(4000, 2, theta)
    ref = ora.dmle(x, y, z, theta)[0]
    with gpu.Session(x, y, dts=256) as s:
        s.set_data(z=z)
        s.set_mixed(band=1, passes=3)
        ts, band, rep = s.autotune(theta, tol=1e-6)
        assert ts in (256, 512) and band in (1, 2, 4, 8)
        assert s.data.diag_thick == band
        got = s.mle_alg(theta)
        assert abs(got - ref) / abs(ref) < 1e-6


def test_batch_autotune_matches_the_oracle(gpu, ora):
    rng = np.random.default_rng(4)
    xs, ys, zs, th = [], [], [], []
    for f in range(20):
        n = int(rng.integers(300, 1800))
        x, y = rng.random(n), rng.random(n)
        t = [rng.uniform(0.5, 2.0), rng.uniform(0.02, 0.1), rng.uniform(0.3, 1.0)]
        xs.append(x), ys.append(y), zs.append(ora.dzvg(x, y, t, rng.standard_normal(n))), th.append(t)
    th = np.array(th)
    with gpu.Batch(xs, ys, zs, autotune_theta=th) as b:
        assert b.ts in (128, 256, 384, 512) and len(b.autotune_report) >= 2
        got = b.loglik(th)
    for g, x, y, z, t in zip(got, xs, ys, zs, th):
        l, ld, dp, _ = ora.dmle(x, y, z, t)
        scale = 0.5 * abs(dp) + 0.5 * abs(ld) + 0.5 * len(x) * math.log(2 * math.pi)
        assert abs(g - l) / scale < 1e-10
