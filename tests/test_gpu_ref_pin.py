"""The GPU path against fixtures written by the reference's own C code
(tests/golden/gen_ref_fixtures.py, from sources compiled unchanged into
oracle/_ref): covariance tiles of the Matern, nugget, bivariate
parsimonious and flexible, and great-circle generators within 1e-13 relative (the device
has its own K_nu, pinned to mpmath to 1e-14), and the library's hold-out
split (pick_random_points on the device's z) bit for bit."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KERNELS = {"matern": 0, "nuggets": 1, "bivariate_parsimonious": 2, "bivariate_flexible": 3}


def _sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def test_device_covariance_tiles_match_the_reference(gpu):
    with open(os.path.join(GOLD, "ref_fixtures.json")) as f:
        meta = json.load(f)
    tiles = dict(np.load(os.path.join(GOLD, "ref_fixtures.npz")))
    x, y = gpu.generate_xy_loc(1600, 0)
    t = meta["tile"]
    for name, kern, theta, metric in meta["cov_cases"]:
        if kern not in KERNELS:
            continue
        a, b = (20.0 + 10.0 * x, 40.0 + 10.0 * y) if metric else (x, y)
        C = gpu.covariance_dense(a, b, theta, kernel=KERNELS[kern], metric=metric, ts=128)
        for m0, n0 in meta["offsets"]:
            ref = tiles["%s_%d_%d" % (name, m0, n0)]
            got = C[m0:m0 + t, n0:n0 + t]
            low = np.tril(np.ones((t, t), dtype=bool), n0 - m0) if m0 - n0 < t else np.ones((t, t), dtype=bool)
            scale = np.maximum(np.abs(ref), 1e-300)
            rel = (np.abs(got - ref) / scale)[low & (np.abs(ref) > 1e-250)]
            assert rel.max() < 1e-13, (name, m0, n0, rel.max())


def test_library_hold_out_split_is_the_reference_bits(gpu, ora):
    import ctypes

    with open(os.path.join(GOLD, "ref_fixtures.json")) as f:
        meta = json.load(f)
    for key, h in meta["pick_random_points"].items():
        N, seed, nmiss = map(int, key.split("_"))
        x, y = gpu.generate_xy_loc(N, seed)  # leaves libc rand() after 2 N draws
        z = ora.dlarnv(seed, N)
        with gpu.Session(x, y) as s:
            s.set_data(z=z)
            zobs, zact = np.empty(N - nmiss), np.empty(nmiss)
            P = ctypes.POINTER(ctypes.c_double)
            gpu.lib().pick_random_points(ctypes.byref(s.data), zobs.ctypes.data_as(P), zact.ctypes.data_as(P),
                                         nmiss, N - nmiss, N)
            got = dict(z_obs=zobs, z_actual=zact,
                       x_obs=np.ctypeslib.as_array(s.data.lobs.x, shape=(N - nmiss,)),
                       y_obs=np.ctypeslib.as_array(s.data.lobs.y, shape=(N - nmiss,)),
                       x_miss=np.ctypeslib.as_array(s.data.lmiss.x, shape=(nmiss,)),
                       y_miss=np.ctypeslib.as_array(s.data.lmiss.y, shape=(nmiss,)))
            assert {k: _sha(v) for k, v in got.items()} == h, key
