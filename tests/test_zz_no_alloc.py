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


def _noalloc(xg, n, dx, dy, dz, theta, kernel, dout, stream):
    """Device pointers (ints) for x, y, z and the 3-double result; stream is a
    cudaStream_t handle (0 = the default stream)."""
    th = np.ascontiguousarray(theta, dtype=np.float64)
    P = ctypes.POINTER(ctypes.c_double)
    return xg.lib().exageostat_b200_dmle_device_noalloc(n, ctypes.cast(dx, P), ctypes.cast(dy, P),
                                                        ctypes.cast(dz, P), th.ctypes.data_as(P), kernel, 0,
                                                        ctypes.cast(dout, P), ctypes.c_void_p(stream))


def test_noalloc_matches_allocating_entry_point_twice(gpu, ora):
    import torch

    torch.cuda.init()
    s = torch.cuda.current_stream()
    cases = [(1600, 0, [1.0, 0.1, 0.5], 0), (2000, 3, [1.2, 0.07, 0.73, 0.02], 1)]
    for n, seed, theta, kernel in cases:
        x, y = ora.generate_xy_loc(n, seed)
        z = np.random.default_rng(seed).standard_normal(n)
        dx, dy, dz = (torch.tensor(a, dtype=torch.float64, device="cuda") for a in (x, y, z))
        dout = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
        rc = _noalloc(gpu, n, dx.data_ptr(), dy.data_ptr(), dz.data_ptr(), theta, kernel, dout.data_ptr(),
                      s.cuda_stream)
        assert rc == 0, gpu.last_error()
        got = dout.cpu().numpy()
        ref = np.array(gpu.dmle_host(x, y, z, theta, kernel, ts=128))
        assert np.allclose(got, ref, rtol=LL_RTOL, atol=0), (got, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    import torch

    n = MAX_N + 1
    buf = torch.zeros(n, dtype=torch.float64, device="cuda")
    dout = torch.zeros(3, dtype=torch.float64, device="cuda")
    rc = _noalloc(gpu, n, buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), [1.0, 0.1, 0.5], 0, dout.data_ptr(), 0)
    assert rc == gpu.XG_ERR_BAD_ARGUMENT
    assert str(MAX_N) in gpu.last_error()
