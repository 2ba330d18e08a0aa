"""Synthetic-data helpers of the reference driver (examples/synthetic_dmle_test.c).

``dlarnv`` draws the N(0,1) vector e exactly as the driver does,
``LAPACKE_dlarnv(3, {seed, seed, seed, 1}, N, e)`` (synthetic_dmle_test.c:111,147),
by calling LAPACK's dlarnv from the OpenBLAS that numpy bundles (a library
call, as the reference calls MKL's).
"""
from __future__ import annotations

import ctypes
import glob
import os

import numpy as np

_blas = None


def _openblas():
    global _blas
    if _blas is None:
        d = os.path.realpath(os.path.join(os.path.dirname(np.__file__), "..", "numpy.libs"))
        cands = glob.glob(os.path.join(d, "libscipy_openblas64_*.so"))
        if not cands:
            raise RuntimeError("numpy's bundled ILP64 OpenBLAS was not found in %s" % d)
        L = ctypes.CDLL(cands[0])
        f = L.scipy_LAPACKE_dlarnv64_
        f.restype = ctypes.c_int64
        f.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_int64), ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]
        _blas = L
    return _blas


def dlarnv(seed: int, n: int) -> np.ndarray:
    iseed = (ctypes.c_int64 * 4)(seed, seed, seed, 1)
    out = np.empty(n)
    info = _openblas().scipy_LAPACKE_dlarnv64_(3, iseed, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if info != 0:
        raise RuntimeError("dlarnv info=%d" % info)
    return out
