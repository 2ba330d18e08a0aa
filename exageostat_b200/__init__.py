"""exageostat_b200 -- Python bindings over the C ABI (include/exageostat_b200.h).

The library ``exageostat_b200/lib/libexageostat_b200.so`` is built in-tree by
``python -m exageostat_b200.build``.  There is no CPU fallback: loading
raises if the library is missing, and every compute call runs on the GPU.

``MLEData`` / ``Location`` / ``Output`` mirror the reference structures
(misc/include/MLE_misc.h:111-328) field for field; ``check_abi()`` compares
their layout with the compiled library.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libexageostat_b200.so")

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p
_CP = ctypes.c_char_p


class Location(ctypes.Structure):
    _fields_ = [("x", _PD), ("y", _PD), ("z", _PD)]


_OUTPUT_FIELDS = [
    ("problem_size", _I), ("computation", _CP), ("kernel", _CP), ("ds_type", _CP), ("precision", _CP),
    ("z_sample", _I), ("dense_ts", _I), ("lr_ts", _I), ("lr_acc", _I), ("lr_maxrank", _I), ("ncores", _I),
    ("ngpus", _I), ("p", _I), ("q", _I), ("num_params", _I), ("initial_theta", _PD), ("starting_theta", _PD),
    ("estimated_theta", _PD), ("final_loglik", _D), ("time_per_iteration", _D), ("cholesky_per_iter", _D),
    ("flops_per_iteration", _D), ("generation_per_iter", _D), ("solve_per_iter", _D), ("total_mle_time", _D),
    ("avg_exec_time_gen_stage", _D), ("avg_flops_gen_stage", _D), ("mse_pred1", _D), ("mse_pred2", _D),
    ("mse_pred3", _D), ("mse_pred", _D), ("trace_pred_sum", _D), ("trace_pred_mean", _D), ("total_pred_time", _D),
    ("total_pred_flops", _D), ("mloe", _D), ("mmom", _D), ("mloe_exec", _CP), ("total_mloe_mmom_time", _D),
    ("matrix_gen_mloe_mmom_time", _D), ("cho_fact_mloe_mmom_time", _D), ("loop_mloe_mmom_time", _D),
    ("total_mloe_mmom_flops", _D), ("fisher_00", _D), ("fisher_11", _D), ("fisher_22", _D), ("fisher_time", _D),
]


class Output(ctypes.Structure):
    _fields_ = _OUTPUT_FIELDS


_MLE_FIELDS = (
    [("variance", _D), ("variance1", _D), ("variance2", _D), ("variance3", _D), ("computation", _CP),
     ("c_fun", _CP), ("test", _I), ("async", _I), ("iter_count", _I), ("l1", Location), ("lmiss", Location),
     ("lobs", Location), ("lm", Location)]
    + [(n, _VP) for n in ("descC", "descsubC11", "descsubC12", "descsubC21", "descsubC22", "descZ", "descZ1",
                          "descZ2", "descZ3")]
    + [("Adense", _PD), ("Adense2", _PD)]
    + [(n, _VP) for n in ("descZcpy", "descdet", "descsum", "descproduct", "descproduct1", "descproduct2",
                          "descproduct3", "descZmiss", "descC11", "descC21", "descC12", "descC22", "descZactual",
                          "descZobs", "descmse", "descmse1", "descmse2", "descmse3", "descZtrace", "sequence",
                          "request")]
    + [("verbose", _I), ("check", _I), ("log", _I)]
    + [(n, _D) for n in ("avg_exec_time_per_iter", "total_exec_time", "avg_flops_per_iter",
                         "avg_generation_per_iter", "avg_solve_per_iter", "avg_cholesky_per_iter",
                         "avg_exec_time_gen_stage", "avg_flops_gen_stage", "final_loglik")]
    + [(n, _CP) for n in ("locsFPath", "timeFPath", "obsFPath", "obsFPath2", "obsFPath3", "actualZFPath",
                          "actualZFPath2", "actualZFPath3", "actualZLocFPath", "actualTimeFPath")]
    + [(n, _D) for n in ("det", "sum", "dotp", "dotp1", "dotp2", "dotp3")]
    + [("sdotp", ctypes.c_float)]
    + [(n, _D) for n in ("mserror", "mserror1", "mserror2", "mserror3")]
    + [("dm", _CP), ("diag_thick", _I), ("nFileLog", _CP), ("pFileLog", _VP), ("hicma_maxrank", _I),
       ("hicma_data_type", _I)]
    + [(n, _VP) for n in ("hicma_descC", "hicma_descZ", "hicma_descCD", "hicma_descCUV", "hicma_descCrk",
                          "hicma_descZcpy", "hicma_descdet", "hicma_descproduct", "hicma_descC12D",
                          "hicma_descC12UV", "hicma_descC12rk", "hicma_descC22D", "hicma_descC22UV",
                          "hicma_descC22rk")]
    + [("hicma_acc", _D), ("hsequence", _VP), ("hrequest", _VP), ("opt_tol", _I), ("opt_max_iters", _I),
       ("ooc", _I), ("kernel_fun", _CP), ("precision", _I)]
    + [(n, _VP) for n in ("desctemp", "desctemp22", "desck_t", "desck_a", "desck_ttmp", "desck_atmp", "descK_t",
                          "descK_a", "descexpr1", "descexpr2", "descexpr3", "descexpr4", "descestimatedalpha",
                          "desctruthalpha", "desc_mloe_mmom", "descmloe", "descmmom")]
    + [(n, _D) for n in ("expr1", "expr2", "expr3", "expr4", "mloe", "mmom")]
    + [("mloe_mmom", _I), ("mloe_mmom_async", _I), ("mspe", _I), ("recovery_file", _CP),
       ("checkpoint_file", _CP), ("time_slots", _I), ("idw", _I), ("fisher", _I), ("descr", _VP),
       ("descrcpy", _VP), ("seed", _I)]
)


class MLEData(ctypes.Structure):
    _fields_ = _MLE_FIELDS


# error codes (include/exageostat_b200.h)
XG_OK, XG_ERR_NOT_INITIALIZED, XG_ERR_BAD_ARGUMENT, XG_ERR_CUDA, XG_ERR_NOT_SPD, XG_ERR_TIMEOUT, \
    XG_ERR_UNSUPPORTED, XG_ERR_NO_MEMORY = range(8)

EXPORTED_SYMBOLS = [
    "exageostat_init", "EXAGEOSTAT_init", "exageostat_finalize", "EXAGEOSTAT_dmle_Call", "MORSE_dmle_Call",
    "MLE_zvg", "MLE_alg", "EXAGEOSTAT_dmle_Tile", "MORSE_dmle_Tile", "MLE_get_zobs", "prediction_init",
    "EXAGEOSTAT_dmle_Predict_Allocate", "EXAGEOSTAT_dmle_Predict_Tile", "MORSE_dmle_Predict_Tile",
    "prediction_finalize", "MLE_Finalize", "GenerateXYLoc", "uniform_distribution", "shuffle",
    "locations_obs_zsort_inplace", "pick_random_points", "exageostat_b200_loglik", "exageostat_last_error",
    "exageostat_b200_abi_version", "exageostat_b200_sizeof_MLE_data", "exageostat_b200_sizeof_output",
    "exageostat_b200_offsetof_MLE_data", "exageostat_b200_dmle_host", "exageostat_b200_bessel_knu",
    "exageostat_b200_matern_pairs", "exageostat_b200_covariance_dense", "exageostat_b200_set_data",
    "exageostat_b200_set_profiling", "exageostat_b200_get_profile", "exageostat_b200_dmle_device_noalloc",
    "exageostat_b200_bobyqa", "EXAGEOSTAT_sdmle_Tile", "exageostat_b200_set_mixed",
    "exageostat_b200_dmle_host_mixed", "exageostat_b200_mixed_factor_dense", "exageostat_b200_batch_create",
    "exageostat_b200_batch_loglik", "exageostat_b200_batch_destroy", "exageostat_b200_set_sliced",
    "exageostat_b200_dmle_host_sliced", "exageostat_b200_sliced_factor_dense", "exageostat_b200_autotune",
    "exageostat_b200_batch_autotune", "EXAGEOSTAT_Fisher_Tile", "exageostat_b200_fisher",
    "exageostat_b200_fisher_host", "mloe_mmom_init", "EXAGEOSTAT_dmle_mloe_mmom_Allocate",
    "EXAGEOSTAT_dmle_mloe_mmom_Tile", "EXAGEOSTAT_dmle_mloe_mmom_Tile_Async", "mloe_mmom_finalize",
    "MLOE_MMOM_Finalize", "exageostat_b200_mloe_mmom_host", "countlines", "readLocsFile", "readLocsFile3d",
    "readObsFile", "readTimeFile", "shuffle2", "pick_random_points2", "results",
]

_lib = None


class XgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("exageostat_b200 error %d: %s" % (code, msg))
        self.code = code


def lib():
    """Load the compiled library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("%s is missing: build it with `python -m exageostat_b200.build` "
                           "(there is no CPU fallback)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    PM = ctypes.POINTER(MLEData)
    sig = {
        "exageostat_init": (None, [ctypes.POINTER(_I)] * 4),
        "exageostat_finalize": (None, []),
        "EXAGEOSTAT_dmle_Call": (None, [PM, _I, _I, _I, _I, _I, _I, _I, _I]),
        "MLE_zvg": (None, [PM, _PD, _PD, _I, _I, _I, _I, _I]),
        "MLE_alg": (_D, [ctypes.c_uint, _PD, _PD, _VP]),
        "EXAGEOSTAT_dmle_Tile": (_D, [ctypes.c_uint, _PD, _PD, _VP]),
        "MLE_get_zobs": (None, [PM, _PD, _I]),
        "prediction_init": (None, [PM, _I, _I, _I, _I, _I, _I]),
        "EXAGEOSTAT_dmle_Predict_Tile": (_D, [PM, _PD, _I, _I, _PD, _PD, _PD, _I]),
        "prediction_finalize": (None, [PM]),
        "MLE_Finalize": (None, [PM]),
        "GenerateXYLoc": (ctypes.POINTER(Location), [_I, _I]),
        "uniform_distribution": (_D, [_D, _D]),
        "locations_obs_zsort_inplace": (_I, [_I, ctypes.POINTER(Location), _PD]),
        "pick_random_points": (None, [PM, _PD, _PD, _I, _I, _I]),
        "pick_random_points2": (None, [PM, _PD, _PD, _I, _I, _I]),
        "exageostat_b200_loglik": (_I, [PM, _PD, _PD, _PD]),
        "exageostat_last_error": (_CP, []),
        "exageostat_b200_abi_version": (_I, []),
        "exageostat_b200_sizeof_MLE_data": (ctypes.c_size_t, []),
        "exageostat_b200_sizeof_output": (ctypes.c_size_t, []),
        "exageostat_b200_offsetof_MLE_data": (ctypes.c_long, [_CP]),
        "exageostat_b200_dmle_host": (_I, [_I, _PD, _PD, _PD, _PD, _I, _I, _I, _PD]),
        "exageostat_b200_bessel_knu": (_I, [_I, _PD, _PD, _PD]),
        "exageostat_b200_matern_pairs": (_I, [_I, _PD, _PD, _PD, _PD, _PD, _I, _I, _PD]),
        "exageostat_b200_covariance_dense": (_I, [_I, _PD, _PD, _PD, _I, _I, _I, _I, _PD]),
        "exageostat_b200_set_data": (_I, [PM, _PD, _PD, _PD]),
        "exageostat_b200_set_profiling": (_I, [PM, _I]),
        "exageostat_b200_get_profile": (_I, [PM, _PD, _I]),
        "exageostat_b200_diag_wait_timeout": (_I, [_D, _PD]),
        "exageostat_b200_dmle_device_noalloc": (_I, [_I, _PD, _PD, _PD, _PD, _I, _I, _PD, _VP]),
        "exageostat_b200_bobyqa": (_I, [_I, _PD, _PD, _PD, _D, _D, _D, _I, _VP, _VP, _PD]),
        "EXAGEOSTAT_sdmle_Tile": (_D, [ctypes.c_uint, _PD, _PD, _VP]),
        "exageostat_b200_set_mixed": (_I, [PM, _I, _I]),
        "exageostat_b200_dmle_host_mixed": (_I, [_I, _PD, _PD, _PD, _PD, _I, _I, _I, _I, _I, _PD]),
        "exageostat_b200_mixed_factor_dense": (_I, [_I, _PD, _PD, _PD, _I, _I, _I, _I, _I, _PD]),
        "exageostat_b200_batch_create": (_I, [_I, ctypes.POINTER(_I), _PD, _PD, _PD, _I, _I, _I,
                                              ctypes.POINTER(_VP)]),
        "exageostat_b200_batch_loglik": (_I, [_VP, _PD, _PD]),
        "exageostat_b200_batch_destroy": (_I, [_VP]),
        "exageostat_b200_batch_loglik_grad": (_I, [_VP, _PD, _PD, _PD]),
        "exageostat_b200_set_sliced": (_I, [PM]),
        "exageostat_b200_dmle_host_sliced": (_I, [_I, _PD, _PD, _PD, _PD, _I, _I, _I, _PD]),
        "exageostat_b200_sliced_factor_dense": (_I, [_I, _PD, _PD, _PD, _I, _I, _I, _PD]),
        "exageostat_b200_autotune": (_I, [PM, _PD, _D, ctypes.POINTER(_I), ctypes.POINTER(_I), _PD]),
        "exageostat_b200_batch_autotune": (_I, [_I, ctypes.POINTER(_I), _PD, _PD, _PD, _I, _I, _PD,
                                                ctypes.POINTER(_I), _PD, ctypes.POINTER(_VP)]),
        "EXAGEOSTAT_Fisher_Tile": (_PD, [PM, _I, _PD, _I, _I, _I]),
        "countlines": (_I, [_CP]),
        "readLocsFile": (ctypes.POINTER(Location), [_CP, _I]),
        "readLocsFile3d": (ctypes.POINTER(Location), [_CP, _I]),
        "readObsFile": (_PD, [_CP, _I]),
        "readTimeFile": (_PD, [_CP, _I]),
        "exageostat_b200_fisher": (_I, [PM, _PD, _PD, _PD]),
        "exageostat_b200_fisher_host": (_I, [_I, _PD, _PD, _PD, _I, _I, _I, _PD]),
        "mloe_mmom_init": (None, [PM, _I, _I, _I, _I, _I]),
        "EXAGEOSTAT_dmle_mloe_mmom_Tile": (None, [PM, _PD, _PD, _I, _I, _I]),
        "EXAGEOSTAT_dmle_mloe_mmom_Tile_Async": (None, [PM, _PD, _PD, _I, _I, _I]),
        "mloe_mmom_finalize": (None, [PM]),
        "exageostat_b200_mloe_mmom_host": (_I, [_I, _PD, _PD, _I, _PD, _PD, _PD, _PD, _I, _I, _I, _PD, _PD, _PD,
                                                _PD]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _p(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def last_error() -> str:
    return lib().exageostat_last_error().decode()


def diag_wait_timeout(limit_us: float):
    """Runs a kernel whose bounded wait must run out: returns (rc, waited
    microseconds); rc is XG_ERR_TIMEOUT when the wait gave up as designed."""
    w = _D(0.0)
    rc = lib().exageostat_b200_diag_wait_timeout(float(limit_us), ctypes.byref(w))
    return rc, w.value


def _check(rc: int):
    if rc != XG_OK:
        raise XgError(rc, last_error())


def check_abi() -> None:
    """Raise if the ctypes mirrors disagree with the compiled structures."""
    L = lib()
    if L.exageostat_b200_sizeof_MLE_data() != ctypes.sizeof(MLEData):
        raise RuntimeError("sizeof(MLE_data) %d != ctypes %d" % (L.exageostat_b200_sizeof_MLE_data(),
                                                                 ctypes.sizeof(MLEData)))
    if L.exageostat_b200_sizeof_output() != ctypes.sizeof(Output):
        raise RuntimeError("sizeof(output) mismatch")
    for name, _ in _MLE_FIELDS:
        off = L.exageostat_b200_offsetof_MLE_data(name.encode())
        if off >= 0 and off != getattr(MLEData, name).offset:
            raise RuntimeError("offsetof(MLE_data, %s) %d != ctypes %d" % (name, off, getattr(MLEData, name).offset))


def init(dts: int = 0) -> None:
    """exageostat_init(ncores=1, gpus=1, dts, lts=0)."""
    a, b, c, d = _I(1), _I(1), _I(int(dts)), _I(0)
    lib().exageostat_init(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))


def finalize() -> None:
    lib().exageostat_finalize()


KERNELS = {0: b"univariate_matern_stationary", 1: b"univariate_matern_nuggets_stationary",
           2: b"bivariate_matern_parsimonious", 3: b"bivariate_matern_flexible"}
NPARAMS = {0: 3, 1: 4, 2: 6, 3: 11}


def _dim(x, kernel) -> int:
    """Matrix dimension: the locations, times 2 for the bivariate kernel."""
    return x.size * (2 if kernel in (2, 3) else 1)


def bessel_knu(nu, x) -> np.ndarray:
    nu, x = _f64(nu), _f64(x)
    nu, x = np.broadcast_arrays(nu, x)
    nu, x = _f64(nu), _f64(x)
    out = np.empty(x.size)
    _check(lib().exageostat_b200_bessel_knu(x.size, _p(nu), _p(x), _p(out)))
    return out


def matern_pairs(x1, y1, x2, y2, theta, kernel=0, metric=0) -> np.ndarray:
    a = [_f64(v) for v in (x1, y1, x2, y2)]
    out = np.empty(a[0].size)
    _check(lib().exageostat_b200_matern_pairs(a[0].size, *[_p(v) for v in a], _p(_f64(theta)), kernel, metric,
                                              _p(out)))
    return out


def covariance_dense(x, y, theta, kernel=0, metric=0, ts=0, factor=False) -> np.ndarray:
    x, y = _f64(x), _f64(y)
    n = _dim(x, kernel)
    out = np.empty((n, n))
    _check(lib().exageostat_b200_covariance_dense(n, _p(x), _p(y), _p(_f64(theta)), kernel, metric, ts,
                                                  1 if factor else 0, _p(out)))
    return out


def dmle_host_mixed(x, y, z, theta, kernel=0, metric=0, ts=512, band=1, passes=3):
    """One-shot banded mixed-precision log-likelihood: (loglik, logdet, dotp)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.empty(3)
    _check(lib().exageostat_b200_dmle_host_mixed(x.size, _p(x), _p(y), _p(z), _p(_f64(theta)), kernel, metric, ts,
                                                 band, passes, _p(out)))
    return tuple(out)


def mixed_factor_dense(x, y, theta, kernel=0, metric=0, ts=512, band=1, passes=3) -> np.ndarray:
    x, y = _f64(x), _f64(y)
    n = x.size
    out = np.empty((n, n))
    _check(lib().exageostat_b200_mixed_factor_dense(n, _p(x), _p(y), _p(_f64(theta)), kernel, metric, ts, band,
                                                    passes, _p(out)))
    return out


def dmle_host_sliced(x, y, z, theta, kernel=0, metric=0, ts=0):
    """One-shot log-likelihood with FP64 tiles and INT8-sliced trailing
    updates: (loglik, logdet, dotp)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.empty(3)
    _check(lib().exageostat_b200_dmle_host_sliced(z.size, _p(x), _p(y), _p(z), _p(_f64(theta)), kernel, metric, ts,
                                                  _p(out)))
    return tuple(out)


def sliced_factor_dense(x, y, theta, kernel=0, metric=0, ts=0) -> np.ndarray:
    x, y = _f64(x), _f64(y)
    n = _dim(x, kernel)
    out = np.empty((n, n))
    _check(lib().exageostat_b200_sliced_factor_dense(n, _p(x), _p(y), _p(_f64(theta)), kernel, metric, ts,
                                                     _p(out)))
    return out


def _take_malloced(p, n) -> np.ndarray:
    """Copies n doubles from a library-malloc'd array and frees it."""
    out = np.ctypeslib.as_array(p, shape=(n,)).copy()
    _libc().free(ctypes.cast(p, ctypes.c_void_p))
    return out


_libc_handle = None


def _libc():
    global _libc_handle
    if _libc_handle is None:
        _libc_handle = ctypes.CDLL(None)
        _libc_handle.free.argtypes = [ctypes.c_void_p]
        _libc_handle.free.restype = None
    return _libc_handle


def countlines(path: str) -> int:
    """countlines (misc/compute/MLE_misc.c:965-985): '\n' characters in the file."""
    return int(lib().countlines(os.fsencode(path)))


def read_locs_file(path: str, n: int | None = None, dims: int = 2):
    """readLocsFile / readLocsFile3d (misc/compute/flat_file.c:23-111): n rows
    (default countlines(path)) of "x,y" (dims 2) or "x,y,z" (dims 3); returns
    (x, y) or (x, y, z)."""
    n = countlines(path) if n is None else int(n)
    fn = lib().readLocsFile3d if dims == 3 else lib().readLocsFile
    p = fn(os.fsencode(path), n)
    if not p:
        raise XgError(XG_ERR_BAD_ARGUMENT, "cannot read %d locations from %s" % (n, path))
    loc = p.contents
    cols = [_take_malloced(loc.x, n), _take_malloced(loc.y, n)]
    if dims == 3:
        cols.append(_take_malloced(loc.z, n))
    _libc().free(ctypes.cast(p, ctypes.c_void_p))
    return tuple(cols)


def read_obs_file(path: str, n: int | None = None, time: bool = False) -> np.ndarray:
    """readObsFile / readTimeFile (misc/compute/flat_file.c:115-171): n values,
    one per line (default countlines(path))."""
    n = countlines(path) if n is None else int(n)
    p = (lib().readTimeFile if time else lib().readObsFile)(os.fsencode(path), n)
    if not p:
        raise XgError(XG_ERR_BAD_ARGUMENT, "cannot read %d values from %s" % (n, path))
    return _take_malloced(p, n)


def fisher_host(x, y, theta, kernel=0, metric=0, ts=0) -> np.ndarray:
    """Fisher information 1/2 tr(Sigma^-1 dSigma_j Sigma^-1 dSigma_k) of the
    locations at theta: 3 x 3 (kernel 0) or 4 x 4 with the nugget (kernel 1)."""
    x, y = _f64(x), _f64(y)
    np_ = 4 if kernel == 1 else 3
    out = np.empty((np_, np_))
    _check(lib().exageostat_b200_fisher_host(x.size, _p(x), _p(y), _p(_f64(theta)), kernel, metric, ts, _p(out)))
    return out


def mloe_mmom_host(x_miss, y_miss, x_obs, y_obs, truth_theta, estimated_theta, kernel=0, metric=0, ts=0):
    """MLOE and MMOM of kriging the missing locations from the observed ones
    with estimated_theta when truth_theta is the truth.  Returns (mloe, mmom,
    terms, times): terms[m] = (expr1, expr2, expr3, expr4, loe, mom) of
    missing point m, times = (generation, factorisations, solves, total) s."""
    xm, ym, xo, yo = (_f64(a) for a in (x_miss, y_miss, x_obs, y_obs))
    mloe, mmom = ctypes.c_double(), ctypes.c_double()
    terms = np.empty((xm.size, 6))
    times = np.empty(4)
    _check(lib().exageostat_b200_mloe_mmom_host(xm.size, _p(xm), _p(ym), xo.size, _p(xo), _p(yo),
                                                _p(_f64(truth_theta)), _p(_f64(estimated_theta)), kernel, metric, ts,
                                                ctypes.byref(mloe), ctypes.byref(mmom), _p(terms), _p(times)))
    return mloe.value, mmom.value, terms, times


def dmle_host(x, y, z, theta, kernel=0, metric=0, ts=0):
    """One-shot log-likelihood on host arrays: (loglik, logdet, dotp)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.empty(3)
    _check(lib().exageostat_b200_dmle_host(z.size, _p(x), _p(y), _p(z), _p(_f64(theta)), kernel, metric, ts,
                                           _p(out)))
    return tuple(out)


class Session:
    """One MLE_data driven through the reference entry points, as the
    reference driver (examples/synthetic_dmle_test.c) does."""

    def __init__(self, x, y, kernel: int = 0, dm: str = "ed", dts: int = 0, precision: int = 0,
                 diag_thick: int = 1):
        self.L = lib()
        self.x, self.y = _f64(x).copy(), _f64(y).copy()
        self.N = _dim(self.x, kernel)
        self.kernel = kernel
        self.nparams = NPARAMS[kernel]
        d = MLEData()
        d.computation = b"exact"
        d.kernel_fun = KERNELS[kernel]
        d.dm = dm.encode()
        d.precision = precision
        d.diag_thick = diag_thick
        d.recovery_file = b""
        d.checkpoint_file = b""
        d.l1.x = _p(self.x)
        d.l1.y = _p(self.y)
        self._keep = []
        self.data = d
        self.L.EXAGEOSTAT_dmle_Call(ctypes.byref(d), 1, 1, dts, 1, 1, self.N, self.N, 0)
        if not d.descC:
            raise XgError(XG_ERR_CUDA, last_error())

    def zvg(self, theta0, nrand) -> None:
        t = _f64(theta0)
        e = _f64(nrand)
        self.L.MLE_zvg(ctypes.byref(self.data), _p(e), _p(t), self.N, 0, 0, 1, 1)

    def z(self) -> np.ndarray:
        out = np.empty(self.N)
        self.L.MLE_get_zobs(ctypes.byref(self.data), _p(out), self.N)
        return out

    def loglik(self, theta, grad: bool = False):
        t = _f64(theta)
        ll = _D()
        g = np.empty(self.nparams) if grad else None
        _check(self.L.exageostat_b200_loglik(ctypes.byref(self.data), _p(t), ctypes.byref(ll),
                                             _p(g) if grad else None))
        return (ll.value, g) if grad else ll.value

    def fit_bobyqa(self, lb, ub, x0=None, ftol_abs=1e-9, maxeval=0, rhobeg=0.0):
        """MLE with the derivative-free maximiser driving MLE_alg through the C
        ABI, as the reference driver does with NLopt (start = lower bounds,
        examples/examples.c:263-264).  Returns (theta_hat, loglik, evals)."""
        x0 = _f64(lb).copy() if x0 is None else _f64(x0)
        return bobyqa_maximize(None, x0, lb, ub, rhobeg=rhobeg, ftol_abs=ftol_abs, maxeval=maxeval,
                               c_objective=self.L.MLE_alg, c_data=ctypes.cast(ctypes.byref(self.data), _VP))

    def mle_alg(self, theta) -> float:
        t = _f64(theta)
        return self.L.MLE_alg(self.nparams, _p(t), None, ctypes.cast(ctypes.byref(self.data), _VP))

    def predict(self, theta, x_miss, y_miss, x_obs, y_obs, z_obs, z_actual=None):
        """EXAGEOSTAT_dmle_Predict_Tile: returns (mse, zmiss)."""
        xm, ym, xo, yo, zo = (_f64(a).copy() for a in (x_miss, y_miss, x_obs, y_obs, z_obs))
        za = None if z_actual is None else _f64(z_actual).copy()
        self._keep = [xm, ym, xo, yo]
        d = self.data
        d.lmiss.x, d.lmiss.y = _p(xm), _p(ym)
        d.lobs.x, d.lobs.y = _p(xo), _p(yo)
        nm, no = _dim(xm, self.kernel), _dim(xo, self.kernel)  # rows: 2 per location when bivariate
        zmiss = np.empty(nm)
        t = _f64(theta)
        mse = self.L.EXAGEOSTAT_dmle_Predict_Tile(ctypes.byref(d), _p(t), nm, no, _p(zo),
                                                  None if za is None else _p(za), _p(zmiss), self.N)
        return mse, zmiss

    def fisher(self, theta):
        """exageostat_b200_fisher: (F, F^-1) for the session's kernel."""
        np_ = 4 if self.kernel == 1 else 3
        F, Finv = np.empty((np_, np_)), np.empty((np_, np_))
        _check(self.L.exageostat_b200_fisher(ctypes.byref(self.data), _p(_f64(theta)), _p(F), _p(Finv)))
        return F, Finv

    def fisher_tile(self, theta) -> np.ndarray:
        """EXAGEOSTAT_Fisher_Tile: the inverse Fisher matrix (3 x 3, from the
        reference's 10-double column-major result)."""
        t = _f64(theta)
        r = self.L.EXAGEOSTAT_Fisher_Tile(ctypes.byref(self.data), self.N, _p(t), 0, 1, 1)
        if not r:
            raise XgError(-1, last_error())
        out = np.array([r[i] for i in range(9)]).reshape(3, 3).T.copy()
        _libc().free(ctypes.cast(r, ctypes.c_void_p))
        return out

    def mloe_mmom(self, truth_theta, estimated_theta, x_miss, y_miss, x_obs, y_obs, asynchronous=False):
        """mloe_mmom_init + EXAGEOSTAT_dmle_mloe_mmom_Tile(_Async) +
        mloe_mmom_finalize on the given locations: (data.mloe, data.mmom)."""
        xm, ym, xo, yo = (_f64(a).copy() for a in (x_miss, y_miss, x_obs, y_obs))
        self._keep = [xm, ym, xo, yo]
        d = self.data
        d.lmiss.x, d.lmiss.y = _p(xm), _p(ym)
        d.lobs.x, d.lobs.y = _p(xo), _p(yo)
        tt, te = _f64(truth_theta), _f64(estimated_theta)
        self.L.mloe_mmom_init(ctypes.byref(d), xm.size, xo.size, 0, 1, 1)
        fn = self.L.EXAGEOSTAT_dmle_mloe_mmom_Tile_Async if asynchronous else self.L.EXAGEOSTAT_dmle_mloe_mmom_Tile
        fn(ctypes.byref(d), _p(tt), _p(te), xm.size, xo.size, self.N)
        self.L.mloe_mmom_finalize(ctypes.byref(d))
        if not np.isfinite(d.mloe):
            raise XgError(-1, last_error())
        return d.mloe, d.mmom

    def set_data(self, x=None, y=None, z=None) -> None:
        arrs = [None if a is None else _f64(a) for a in (x, y, z)]
        _check(self.L.exageostat_b200_set_data(ctypes.byref(self.data),
                                               *[None if a is None else _p(a) for a in arrs]))

    def set_mixed(self, band: int = 1, passes: int = 3) -> None:
        """Switch MLE_alg / loglik to the banded mixed-precision path."""
        _check(self.L.exageostat_b200_set_mixed(ctypes.byref(self.data), band, passes))
        self.data.precision = 2

    def set_sliced(self) -> None:
        """Switch MLE_alg / loglik to FP64 tiles with INT8-sliced trailing
        updates (precision 3)."""
        _check(self.L.exageostat_b200_set_sliced(ctypes.byref(self.data)))

    def set_fp64(self) -> None:
        self.data.precision = 0

    def autotune(self, theta, tol: float = 1e-6):
        """exageostat_b200_autotune: tile size (and band width, precision 2)
        chosen by timing; the descriptors are rebuilt with them.  Returns
        (ts, band, [(ts, seconds), ...])."""
        ts, band = _I(), _I()
        rep = np.zeros(8)
        _check(self.L.exageostat_b200_autotune(ctypes.byref(self.data), _p(_f64(theta)), tol, ctypes.byref(ts),
                                               ctypes.byref(band), _p(rep)))
        pairs = [(int(rep[2 * i]), float(rep[2 * i + 1])) for i in range(4) if rep[2 * i] > 0]
        return ts.value, band.value, pairs

    def set_profiling(self, on: bool = True) -> None:
        _check(self.L.exageostat_b200_set_profiling(ctypes.byref(self.data), 1 if on else 0))

    def profile(self) -> dict:
        out = np.zeros(15)
        _check(self.L.exageostat_b200_get_profile(ctypes.byref(self.data), _p(out), 15))
        keys = ["t_gen", "t_potrf", "t_trsm", "t_gemm", "gemm_flops", "launches", "evals", "t_total", "ts", "nt",
                "N", "t_offband", "offband_flops", "t_band", "band_flops"]
        return dict(zip(keys, out.tolist()))

    def close(self) -> None:
        if self.data.descC22:
            self.L.prediction_finalize(ctypes.byref(self.data))
        if self.data.descC:
            self.L.MLE_Finalize(ctypes.byref(self.data))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Batch:
    """Many independent fields evaluated together (one graph launch per call)."""

    def __init__(self, xs, ys, zs, kernel: int = 0, metric: int = 0, ts: int = 256, autotune_theta=None):
        """ts: tile size; with autotune_theta (one parameter row per field) the
        tile size is chosen by exageostat_b200_batch_autotune instead
        (self.ts, self.autotune_report)."""
        self.L = lib()
        self.n = np.array([len(a) for a in xs], dtype=np.int32)
        self.kernel = kernel
        self.nparams = 4 if kernel == 1 else 3
        x, y, z = (_f64(np.concatenate(a)) for a in (xs, ys, zs))
        h = _VP()
        nptr = self.n.ctypes.data_as(ctypes.POINTER(_I))
        self.autotune_report = []
        if autotune_theta is None:
            _check(self.L.exageostat_b200_batch_create(len(xs), nptr, _p(x), _p(y), _p(z), kernel, metric, ts,
                                                       ctypes.byref(h)))
            self.ts = ts
        else:
            th = _f64(autotune_theta).reshape(len(self.n), self.nparams)
            t, rep = _I(), np.zeros(8)
            _check(self.L.exageostat_b200_batch_autotune(len(xs), nptr, _p(x), _p(y), _p(z), kernel, metric, _p(th),
                                                         ctypes.byref(t), _p(rep), ctypes.byref(h)))
            self.ts = t.value
            self.autotune_report = [(int(rep[2 * i]), float(rep[2 * i + 1])) for i in range(4) if rep[2 * i] > 0]
        self.h = h

    def loglik(self, thetas, grad: bool = False):
        """Log-likelihood of every field (one row of parameters per field);
        with grad=True also the gradients, an array of the same shape as the
        parameters: (loglik, grad)."""
        th = _f64(thetas).reshape(len(self.n), self.nparams)
        out = np.empty(len(self.n))
        if grad:
            g = np.empty_like(th)
            _check(self.L.exageostat_b200_batch_loglik_grad(self.h, _p(th), _p(out), _p(g)))
            return out, g
        _check(self.L.exageostat_b200_batch_loglik(self.h, _p(th), _p(out)))
        return out

    def close(self) -> None:
        if self.h:
            self.L.exageostat_b200_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


NLOPT_FUNC = ctypes.CFUNCTYPE(_D, ctypes.c_uint, _PD, _PD, _VP)


def bobyqa_maximize(fun, x0, lb, ub, rhobeg=0.0, rhoend=0.0, ftol_abs=1e-9, maxeval=0, c_objective=None,
                    c_data=None):
    """Maximise with the library's bound-constrained derivative-free method.

    ``fun(x) -> float`` is a Python objective; alternatively pass a C function
    pointer (``c_objective``, e.g. ``lib().MLE_alg``) and its ``c_data``.
    Returns (x_max, f_max, evaluations)."""
    x = _f64(x0).copy()
    lb, ub = _f64(lb), _f64(ub)
    if c_objective is None:
        def _cb(n, xp, gp, data):
            return float(fun(np.ctypeslib.as_array(xp, shape=(n,)).copy()))

        cfun = NLOPT_FUNC(_cb)
        fptr = ctypes.cast(cfun, _VP)
    else:
        cfun = None
        fptr = ctypes.cast(c_objective, _VP)
    fmax = _D()
    ev = lib().exageostat_b200_bobyqa(x.size, _p(x), _p(lb), _p(ub), rhobeg, rhoend, ftol_abs, maxeval, fptr,
                                      c_data, ctypes.byref(fmax))
    if ev < 0:
        raise XgError(-ev, "bobyqa: bad arguments")
    return x, fmax.value, ev


def generate_xy_loc(n: int, seed: int):
    """GenerateXYLoc through the library (host code; consumes libc rand())."""
    L = lib()
    p = L.GenerateXYLoc(int(n), int(seed))
    x = np.ctypeslib.as_array(p.contents.x, shape=(n,)).copy()
    y = np.ctypeslib.as_array(p.contents.y, shape=(n,)).copy()
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [_VP]
    libc.free(ctypes.cast(p.contents.x, _VP))
    libc.free(ctypes.cast(p.contents.y, _VP))
    libc.free(ctypes.cast(p, _VP))
    return x, y
