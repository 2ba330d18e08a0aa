"""Failure detection without a GPU fault.

Every pipeline wait inside the kernels is bounded; when it runs out the kernel
records XG_ST_TIMEOUT in its status word and returns.  The diagnostic entry
point makes one such wait run out on purpose (a barrier that nothing arrives
on, 1 ms limit); the host must see XG_ERR_TIMEOUT and the next evaluation on
the same context must still match the oracle (the context survived)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-10


def test_bounded_wait_times_out_and_the_context_survives(gpu, ora):
    from exageostat_b200.synthetic import dlarnv

    rc, waited = gpu.diag_wait_timeout(1000.0)
    assert rc == gpu.XG_ERR_TIMEOUT, (rc, gpu.last_error())
    assert "timed out" in gpu.last_error()
    assert 1000.0 <= waited < 1e6, waited
    N, seed, theta = 1600, 0, [1.0, 0.1, 0.5]
    x, y = gpu.generate_xy_loc(N, seed)
    e = dlarnv(seed, N)
    with gpu.Session(x, y, dts=320) as s:
        s.zvg(theta, e)
        z = s.z()
        ll = s.mle_alg(theta)
    ref = ora.dmle(x, y, z, theta)[0]
    assert ll == pytest.approx(ref, rel=LL_RTOL)
    # a second timeout right after, then a one-shot evaluation again
    rc, _ = gpu.diag_wait_timeout(50.0)
    assert rc == gpu.XG_ERR_TIMEOUT
    got = gpu.dmle_host(x, y, z, theta, ts=128)[0]
    assert got == pytest.approx(ref, rel=LL_RTOL)


def test_bounded_wait_rejects_limits_out_of_range(gpu):
    rc, _ = gpu.diag_wait_timeout(0.0)
    assert rc == gpu.XG_ERR_BAD_ARGUMENT
    rc, _ = gpu.diag_wait_timeout(5e6)
    assert rc == gpu.XG_ERR_BAD_ARGUMENT
