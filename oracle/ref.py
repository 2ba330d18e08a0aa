"""ctypes binding to oracle/_ref/libexageostat_ref.so: a subset of the
reference's OWN C sources compiled unchanged from the reference tree by
``make -C oracle ref`` (see oracle/Makefile).  Test infrastructure only: it
pins the oracle restatement (oracle/oracle.c) to the reference code, and it
writes the fixtures in tests/golden/ (tests/golden/gen_ref_fixtures.py).  It
only exists where the reference tree is present; available() says whether.

Functions (reference file:line):
  GenerateXYLoc, uniform_distribution, zsort_locations  misc/compute/MLE_misc.c:297-319, 753-792
  pick_random_points, shuffle, locations_obs_zsort_inplace  misc/compute/MLE_misc.c:405-534, 1238-1259, 1700-1741
  core_dcmg, calculateDistance, distanceEarth  exageostat_exact/cpu_core/compute/core_zcmg.c:30-92, 963-994
  core_dcmg_nuggets  exageostat_exact/cpu_core/compute/core_zcmg_nuggets.c:107-156
  core_dcmg_bivariate_parsimonious  exageostat_exact/cpu_core/compute/core_zcmg.c:1628-1726
  core_dcmg_bivariate_flexible  exageostat_exact/cpu_core/compute/core_zcmg.c:1514-1580
  core_dcmg_matern_dsigma_square, _dbeta, _dnu  exageostat_exact/cpu_core/compute/core_zcmg.c:315-488
  core_dmdet  exageostat_exact/cpu_core/compute/core_zmdet.c:50-59
K_nu inside the Matern kernels is the oracle's (GSL is absent; see
oracle/ref_shim/ref_shim.c).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_TREE = os.environ.get("EXAGEOSTAT_REFERENCE_TREE", "/root/reference")
LIB_PATH = os.path.join(_HERE, "_ref", "libexageostat_ref.so")
_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)


class Location(ctypes.Structure):
    _fields_ = [("x", _PD), ("y", _PD), ("z", _PD)]


def available() -> bool:
    return os.path.exists(LIB_PATH) or os.path.isdir(os.path.join(REF_TREE, "misc", "compute"))


def build() -> str | None:
    """Compiles the reference subset when the reference tree is present;
    returns the library path, or None where the tree is absent."""
    if not os.path.isdir(os.path.join(REF_TREE, "misc", "compute")):
        return LIB_PATH if os.path.exists(LIB_PATH) else None
    subprocess.run(["make", "-s", "-C", _HERE, "ref", "REF=" + REF_TREE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if build() is None:
            raise RuntimeError("the reference tree is absent and oracle/_ref is not built")
        L = ctypes.CDLL(LIB_PATH)
        PL = ctypes.POINTER(Location)
        L.GenerateXYLoc.restype = PL
        L.GenerateXYLoc.argtypes = [_I, _I]
        L.uniform_distribution.restype = _D
        L.uniform_distribution.argtypes = [_D, _D]
        L.ref_pick_random_points.restype = None
        L.ref_pick_random_points.argtypes = [_I, _PD, _PD, _PD, _I] + [_PD] * 6
        for name in ("core_dcmg", "core_dcmg_nuggets", "core_dcmg_bivariate_parsimonious", "core_dcmg_bivariate_flexible",
                     "core_dcmg_matern_dsigma_square", "core_dcmg_matern_dbeta", "core_dcmg_matern_dnu"):
            f = getattr(L, name)
            f.restype = None
            f.argtypes = [_PD, _I, _I, _I, _I, PL, PL, _PD, _I]
        L.core_dmdet.restype = _D
        L.core_dmdet.argtypes = [_PD, _I, _I, _I, _I]
        _lib = L
    return _lib


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _p(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def generate_xy_loc(n: int, seed: int):
    """The reference's GenerateXYLoc(n, seed) (srand(seed), jittered grid,
    Morton sort with uint16 quantisation).  Returns copies of (x, y)."""
    loc = lib().GenerateXYLoc(int(n), int(seed)).contents
    x = np.ctypeslib.as_array(loc.x, shape=(n,)).copy()
    y = np.ctypeslib.as_array(loc.y, shape=(n,)).copy()
    return x, y


def pick_random_points(x, y, z, n_miss: int):
    """The reference's pick_random_points on the current libc rand() stream
    (replay it first, as the oracle's rand_replay does)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    N = x.size
    n_obs = N - n_miss
    out = [np.empty(n_miss), np.empty(n_miss), np.empty(n_miss), np.empty(n_obs), np.empty(n_obs), np.empty(n_obs)]
    lib().ref_pick_random_points(N, _p(x), _p(y), _p(z), int(n_miss), *[_p(a) for a in out])
    xm, ym, za, xo, yo, zo = out
    return dict(x_miss=xm, y_miss=ym, z_actual=za, x_obs=xo, y_obs=yo, z_obs=zo)


def _loc(x, y):
    x, y = _f64(x), _f64(y)
    return Location(_p(x), _p(y), None), (x, y)


def cmg(kernel: str, m, n, m0, n0, x1, y1, x2, y2, theta, metric=0) -> np.ndarray:
    """One tile of a reference generator, column-major m x n (A[i + j m]),
    returned as an (m, n) array.  kernel: "matern", "nuggets",
    "bivariate_parsimonious", "bivariate_flexible", "dsigma_square", "dbeta",
    "dnu"."""
    name = {"matern": "core_dcmg", "nuggets": "core_dcmg_nuggets",
            "bivariate_parsimonious": "core_dcmg_bivariate_parsimonious",
            "bivariate_flexible": "core_dcmg_bivariate_flexible",
            "dsigma_square": "core_dcmg_matern_dsigma_square", "dbeta": "core_dcmg_matern_dbeta",
            "dnu": "core_dcmg_matern_dnu"}[kernel]
    l1, keep1 = _loc(x1, y1)
    l2, keep2 = _loc(x2, y2)
    th = _f64(theta)
    A = np.zeros(m * n)
    getattr(lib(), name)(_p(A), int(m), int(n), int(m0), int(n0), ctypes.byref(l1), ctypes.byref(l2), _p(th),
                         int(metric))
    return A.reshape(n, m).T.copy()


def dmdet(A: np.ndarray) -> float:
    """core_dmdet on a square tile (column-major): sum of log of the positive
    diagonal entries."""
    A = np.asfortranarray(A, dtype=np.float64)
    m, n = A.shape
    return lib().core_dmdet(A.ctypes.data_as(_PD), m, n, 0, 0)
