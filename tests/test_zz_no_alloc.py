"""The no-allocation entry point (exageostat_b200_dmle_device_noalloc).

It serves callers that cannot call cudaMalloc (code inside another
framework's allocator or memory pool, code that must run with the device heap
exhausted): they pass device buffers for the inputs and the result, and the
library works in its own static device scratch.  This file is collected last
so a failing run that stops at the first failure has already run every other
test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LL_RTOL = 1e-10
MAX_N = 2048


def _noalloc(xg, n, dx, dy, dz, theta, kernel, dout, stream, metric=0):
    """Device pointers (ints) for x, y, z and the 3-double result; stream is a
    cudaStream_t handle (0 = the default stream)."""
    th = np.ascontiguousarray(theta, dtype=np.float64)
    P = ctypes.POINTER(ctypes.c_double)
    return xg.lib().exageostat_b200_dmle_device_noalloc(n, ctypes.cast(dx, P), ctypes.cast(dy, P),
                                                        ctypes.cast(dz, P), th.ctypes.data_as(P), kernel, metric,
                                                        ctypes.cast(dout, P), ctypes.c_void_p(stream))


def _gc_locations(n, seed):
    rng = np.random.default_rng(seed)
    lat = rng.uniform(20.0, 24.0, n)
    lon = rng.uniform(40.0, 44.0, n)
    return lat, lon


def _run_cases(gpu, ora, stream_handle, cases):
    import torch

    for n, seed, theta, kernel, metric in cases:
        if metric:
            x, y = _gc_locations(n, seed)
        else:
            x, y = ora.generate_xy_loc(n, seed)
        z = np.random.default_rng(seed).standard_normal(n)
        dx, dy, dz = (torch.tensor(a, dtype=torch.float64, device="cuda") for a in (x, y, z))
        dout = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
        rc = _noalloc(gpu, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), theta, kernel, dout.data_ptr(),
                      stream_handle, metric)
        assert rc == 0, gpu.last_error()
        got = dout.cpu().numpy()
        ref = np.array(gpu.dmle_host(x, y, z, theta, kernel, metric, ts=128))
        assert np.allclose(got, ref, rtol=LL_RTOL, atol=0), (got, ref)
        ora_ll = ora.dmle(x, y, z, theta, kernel, metric)[0]
        assert abs(got[0] - ora_ll) <= LL_RTOL * abs(ora_ll), (got[0], ora_ll)


def test_noalloc_matches_allocating_entry_point_twice(gpu, ora):
    """Two calls in a row on the default stream, each checked against the
    allocating entry point and the oracle."""
    import torch

    torch.cuda.init()
    _run_cases(gpu, ora, 0, [(1600, 0, [1.0, 0.1, 0.5], 0, 0), (2000, 3, [1.2, 0.07, 0.73, 0.02], 1, 0)])


def test_noalloc_on_a_side_stream_large_then_small(gpu, ora):
    """A caller's own (non-default) stream; the largest size first and a
    smaller one after it, so contents the first call left in the scratch must
    not leak into the second; a great-circle field last."""
    import torch

    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        _run_cases(gpu, ora, s.cuda_stream, [(MAX_N, 5, [1.0, 0.1, 1.5], 0, 0), (700, 6, [0.8, 0.05, 0.5], 0, 0),
                                             (900, 7, [1.0, 150.0, 0.8], 0, 1)])


def test_noalloc_rejects_bad_arguments_and_keeps_the_result_buffer(gpu):
    import torch

    n = MAX_N + 1
    buf = torch.zeros(n, dtype=torch.float64, device="cuda")
    dout = torch.full((3,), 7.0, dtype=torch.float64, device="cuda")
    rc = _noalloc(gpu, n, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), [1.0, 0.1, 0.5], 0, dout.data_ptr(), 0)
    assert rc == gpu.XG_ERR_BAD_ARGUMENT
    assert str(MAX_N) in gpu.last_error()
    rc = _noalloc(gpu, 100, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), [1.0, 0.1, 0.5], 0, dout.data_ptr(), 0,
                  metric=2)
    assert rc == gpu.XG_ERR_BAD_ARGUMENT
    assert "metric" in gpu.last_error()
    # all locations equal: a singular covariance, reported without touching d_out
    rc = _noalloc(gpu, 100, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), [1.0, 0.1, 0.5], 0, dout.data_ptr(), 0)
    assert rc == gpu.XG_ERR_NOT_SPD, gpu.last_error()
    assert torch.all(dout == 7.0)
