"""CPU oracle for the exact Matern log-likelihood path (TEST INFRASTRUCTURE).

Only the tests, the smoke check and the benchmark's CPU-baseline leg use this
package, and only as the checker.  The product library never imports it.

It wraps ``oracle/_build/liboracle.so`` (built from ``oracle.c`` by
``oracle/Makefile``), a C restatement of the reference algorithm with the
reference file:line of every function in its header comment.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_D = ctypes.c_double
_I = ctypes.c_int
_PD = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + numpy's OpenBLAS)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.ora_bessel_knu.restype = _D
        L.ora_bessel_knu.argtypes = [_D, _D]
        L.ora_generate_xy_loc.argtypes = [_I, _I, _PD, _PD]
        L.ora_rand_replay.argtypes = [_I, ctypes.c_long]
        L.ora_pick_random_points.argtypes = [_I, _PD, _PD, _PD, _I, _PD, _PD, _PD, _PD, _PD, _PD]
        L.ora_locations_obs_zsort_inplace.argtypes = [_I, _PD, _PD, _PD]
        L.ora_pick_random_points2.argtypes = [_I, _PD, _PD, _PD, _I, _PD, _PD, _PD, _PD, _PD, _PD]
        L.ora_core_dcmg.argtypes = [_PD, _I, _I, _I, _I, _PD, _PD, _PD, _PD, _PD, _I]
        L.ora_gen_lower_dense.argtypes = [_PD, _I, _PD, _PD, _PD, _I]
        L.ora_dcmg_deriv.argtypes = [_PD, _I, _I, _I, _I, _PD, _PD, _PD, _PD, _PD, _I]
        L.ora_set_metric.argtypes = [_I]
        L.ora_dlarnv.argtypes = [_I, _I, _PD]
        L.ora_dzvg.argtypes = [_I, _PD, _PD, _PD, _I, _PD, _PD]
        L.ora_dmle.argtypes = [_I, _PD, _PD, _PD, _PD, _I, _PD, _PD, _PD, _PD]
        L.ora_dpredict.restype = _D
        L.ora_dpredict.argtypes = [_I, _I, _PD, _PD, _PD, _PD, _PD, _PD, _PD, _I, _PD]
        L.ora_set_threads.argtypes = [_I]
        L.ora_get_max_threads.restype = _I
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_PD)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def max_threads() -> int:
    return int(lib().ora_get_max_threads())


def bessel_knu(nu: float, x: float) -> float:
    return float(lib().ora_bessel_knu(float(nu), float(x)))


def generate_xy_loc(n: int, seed: int):
    x = np.empty(n)
    y = np.empty(n)
    lib().ora_generate_xy_loc(int(n), int(seed), _p(x), _p(y))
    return x, y


def rand_replay(seed: int, skip: int) -> None:
    lib().ora_rand_replay(int(seed), int(skip))


def pick_random_points(x, y, z, n_miss: int, seed: int | None = None, skip: int | None = None):
    """Hold-out split.  With ``seed`` the libc stream is first replayed to the
    state GenerateXYLoc(N, seed) leaves it in (2 N draws)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    N = x.size
    if seed is not None:
        rand_replay(seed, 2 * N if skip is None else skip)
    n_obs = N - n_miss
    out = [np.empty(n_miss), np.empty(n_miss), np.empty(n_miss), np.empty(n_obs), np.empty(n_obs), np.empty(n_obs)]
    lib().ora_pick_random_points(N, _p(x), _p(y), _p(z), int(n_miss), *[_p(a) for a in out])
    xm, ym, za, xo, yo, zo = out
    return dict(x_miss=xm, y_miss=ym, z_actual=za, x_obs=xo, y_obs=yo, z_obs=zo)


def pick_random_points2(x, y, z, n_miss: int):
    """Bivariate hold-out (pick_random_points2): x, y hold the locations, z
    the interleaved values (2 per location); the libc stream is used as it
    stands (replay it first with rand_replay)."""
    x, y, z = _f64(x), _f64(y), _f64(z)
    nloc = x.size
    n_obs = nloc - n_miss
    out = [np.empty(n_miss), np.empty(n_miss), np.empty(2 * n_miss), np.empty(n_obs), np.empty(n_obs),
           np.empty(2 * n_obs)]
    lib().ora_pick_random_points2(nloc, _p(x), _p(y), _p(z), int(n_miss), *[_p(a) for a in out])
    xm, ym, za, xo, yo, zo = out
    return dict(x_miss=xm, y_miss=ym, z_actual=za, x_obs=xo, y_obs=yo, z_obs=zo)


def core_dcmg(m, n, m0, n0, x1, y1, x2, y2, theta, kernel=0, metric=0) -> np.ndarray:
    """Column-major m x n tile, returned as an (m, n) array (metric 1: great
    circle on (lat, lon) in degrees, km)."""
    lib().ora_set_metric(int(metric))
    A = np.empty((n, m))  # column-major storage == C-order (n, m)
    x1, y1, x2, y2, th = _f64(x1), _f64(y1), _f64(x2), _f64(y2), _f64(theta)
    lib().ora_core_dcmg(_p(A), m, n, m0, n0, _p(x1), _p(y1), _p(x2), _p(y2), _p(th), int(kernel))
    return A.T.copy()


def covariance_lower(x, y, theta, kernel=0, metric=0) -> np.ndarray:
    """Lower triangle of Sigma(theta) (upper part left as zeros); for the
    bivariate kernel 2 the matrix is 2 n x 2 n (index 2 l + v)."""
    lib().ora_set_metric(int(metric))
    x, y, th = _f64(x), _f64(y), _f64(theta)
    N = x.size * (2 if kernel in (2, 3) else 1)
    C = np.zeros((N, N))  # column-major buffer; transposed on return
    lib().ora_gen_lower_dense(_p(C), N, _p(x), _p(y), _p(th), int(kernel))
    return C.T.copy()


def dcmg_deriv(m, n, m0, n0, x1, y1, x2, y2, theta, which, metric=0) -> np.ndarray:
    """dSigma/dtheta_which (0 sigma^2, 1 beta, 2 nu) of the Matern part, an
    (m, n) block (core_dcmg_matern_dsigma_square / _dbeta / _dnu,
    exageostat_exact/cpu_core/compute/core_zcmg.c:315-488)."""
    A = np.empty((n, m))
    x1, y1, x2, y2, th = _f64(x1), _f64(y1), _f64(x2), _f64(y2), _f64(theta)
    lib().ora_set_metric(int(metric))
    lib().ora_dcmg_deriv(_p(A), m, n, m0, n0, _p(x1), _p(y1), _p(x2), _p(y2), _p(th), int(which))
    return A.T.copy()


def covariance_full(x, y, theta, kernel=0, metric=0) -> np.ndarray:
    C = covariance_lower(x, y, theta, kernel, metric)
    return C + np.tril(C, -1).T


def _spd_inverse_as_reference(A):
    """LAPACKE_dpotrf('L') then two dtrsm on the identity
    (exageostat_exact/src/compute/MLE_dexact.c:1893-1916)."""
    from scipy.linalg import solve_triangular

    L = np.linalg.cholesky(A)
    Y = solve_triangular(L, np.eye(A.shape[0]), lower=True)
    return solve_triangular(L, Y, lower=True, trans="T")


def fisher(x, y, theta, kernel=0, metric=0):
    """EXAGEOSTAT_Fisher_Tile (exageostat_exact/src/compute/MLE_dexact.c:1777-1934):
    C = Sigma(theta) factored; for j <= k: CJ = L^-T L^-1 dSigma_j, CK likewise
    (two dtrsm each, :1846-1847, :1866-1867), A[k + 3 j] = 1/2 trace(CJ CK) (:1870-1879);
    then the inverse of A.  kernel 1 adds tau^2 (dSigma = I) as a fourth
    parameter, which the reference does not have.  Returns (F, F^-1), both
    symmetric np x np."""
    from scipy.linalg import solve_triangular

    x, y = _f64(x), _f64(y)
    N = x.size
    C = covariance_full(x, y, theta, kernel, metric)
    L = np.linalg.cholesky(C)
    D = [dcmg_deriv(N, N, 0, 0, x, y, x, y, theta, j, metric) for j in range(3)]
    if kernel == 1:
        D.append(np.eye(N))
    M = []
    for Dj in D:
        T = solve_triangular(L, Dj, lower=True)
        M.append(solve_triangular(L, T, lower=True, trans="T"))
    n = len(D)
    F = np.empty((n, n))
    for j in range(n):
        for k in range(j, n):
            F[j, k] = F[k, j] = 0.5 * np.sum(M[j] * M[k].T)
    return F, _spd_inverse_as_reference(F)


def mloe_mmom(x_miss, y_miss, x_obs, y_obs, truth_theta, estimated_theta, kernel=0, metric=0):
    """EXAGEOSTAT_dmle_mloe_mmom_Tile (exageostat_exact/src/compute/MLE_dexact.c:1109-1434)
    restated with the missing points as columns: K_a, K_t (:1239-1245) and
    their factors (:1252, :1261); per point k_t, k_a (:1283-1286), the four
    triangular solves (:1302-1326), expr1 = k_t^T k_a, expr4 = k_a^T k_a,
    expr3 = k_t^T k_t on the solved vectors (:1334-1350), k_a <- L_t^T k_a and
    expr2 = k_a^T k_a (:1357-1362), the geadd steps (:1371-1375) and the
    accumulation of CORE_dmloe_mmom_starpu
    (exageostat_exact/runtime/starpu/codelets/codelet_zmloe_mmom.c:42-60).
    Returns (mloe, mmom, terms) with terms[m] = (k_t^T K_a^-1 k_a, expr2,
    expr3, expr4, loe, mom)."""
    from scipy.linalg import solve_triangular

    xm, ym, xo, yo = (_f64(a) for a in (x_miss, y_miss, x_obs, y_obs))
    nobs, nmiss = xo.size, xm.size
    La = np.linalg.cholesky(covariance_full(xo, yo, estimated_theta, kernel, metric))
    Lt = np.linalg.cholesky(covariance_full(xo, yo, truth_theta, kernel, metric))
    kt = core_dcmg(nobs, nmiss, 0, 0, xo, yo, xm, ym, truth_theta, kernel, metric)
    ka = core_dcmg(nobs, nmiss, 0, 0, xo, yo, xm, ym, estimated_theta, kernel, metric)
    kttmp, katmp = kt.copy(), ka.copy()
    ka = solve_triangular(La, ka, lower=True)
    kt = solve_triangular(Lt, kt, lower=True)
    ka = solve_triangular(La, ka, lower=True, trans="T")
    kt = solve_triangular(Lt, kt, lower=True, trans="T")
    e1 = np.sum(kttmp * ka, axis=0)
    e4 = np.sum(katmp * ka, axis=0)
    e3 = np.sum(kttmp * kt, axis=0)
    ka = Lt.T @ ka
    e2 = np.sum(ka * ka, axis=0)
    t0, a0 = float(truth_theta[0]), float(estimated_theta[0])
    expr1 = t0 - 2.0 * e1
    expr2 = expr1 + e2
    expr3 = t0 - e3
    expr4 = a0 - e4
    terms = np.empty((nmiss, 6))
    mloe = mmom = 0.0
    for p in range(nmiss):
        loe = -1.0 if expr3[p] == 0.0 else expr2[p] / expr3[p] - 1.0
        mom = -1.0 if expr2[p] == 0.0 else expr4[p] / expr2[p] - 1.0
        mloe += loe
        mmom += mom
        terms[p] = (e1[p], expr2[p], expr3[p], expr4[p], loe, mom)
    return mloe / nmiss, mmom / nmiss, terms


def dlarnv(seed: int, n: int) -> np.ndarray:
    out = np.empty(n)
    info = lib().ora_dlarnv(int(seed), int(n), _p(out))
    if info != 0:
        raise RuntimeError("dlarnv failed: %d" % info)
    return out


def dzvg(x, y, theta, nrand, kernel=0, metric=0) -> np.ndarray:
    lib().ora_set_metric(int(metric))
    x, y, th, e = _f64(x), _f64(y), _f64(theta), _f64(nrand)
    z = np.empty(e.size)  # 2 x the locations for the bivariate kernel
    info = lib().ora_dzvg(e.size, _p(x), _p(y), _p(th), int(kernel), _p(e), _p(z))
    if info != 0:
        raise RuntimeError("oracle dzvg: dpotrf info=%d" % info)
    return z


def dmle(x, y, z, theta, kernel=0, metric=0):
    """Returns (loglik, logdet, dotp, (t_gen, t_chol, t_solve))."""
    lib().ora_set_metric(int(metric))
    x, y, z, th = _f64(x), _f64(y), _f64(z), _f64(theta)
    ll, ld, dp = _D(), _D(), _D()
    times = np.zeros(3)
    info = lib().ora_dmle(z.size, _p(x), _p(y), _p(z), _p(th), int(kernel), ctypes.byref(ll), ctypes.byref(ld),
                          ctypes.byref(dp), _p(times))
    if info != 0:
        raise RuntimeError("oracle dmle: dpotrf info=%d" % info)
    return ll.value, ld.value, dp.value, tuple(times)


def dpredict(x_miss, y_miss, x_obs, y_obs, z_obs, z_actual, theta, kernel=0, metric=0):
    """Returns (mse, zmiss)."""
    lib().ora_set_metric(int(metric))
    xm, ym, xo, yo, zo, th = (_f64(a) for a in (x_miss, y_miss, x_obs, y_obs, z_obs, theta))
    za = None if z_actual is None else _f64(z_actual)
    nm = xm.size * (2 if kernel in (2, 3) else 1)  # matrix rows: two per location for the bivariate kernel
    zmiss = np.empty(nm)
    mse = lib().ora_dpredict(nm, zo.size, _p(xm), _p(ym), _p(xo), _p(yo), _p(zo),
                             None if za is None else _p(za), _p(th), int(kernel), _p(zmiss))
    return float(mse), zmiss


def synthetic_field(N: int, seed: int, theta, kernel=0, metric=0, locations=None):
    """The reference's synthetic workflow (synthetic_dmle_test.c:103-147,278):
    e = dlarnv(3, {seed,seed,seed,1}), locations = GenerateXYLoc(N, seed),
    z = L(theta) e."""
    e = dlarnv(seed, N)
    nloc = N // 2 if kernel in (2, 3) else N  # N = p x locations (synthetic_dmle_test.c:134, 153)
    x, y = generate_xy_loc(nloc, seed) if locations is None else (_f64(locations[0]), _f64(locations[1]))
    z = dzvg(x, y, theta, e, kernel, metric)
    return x, y, z, e


def maximise(x, y, z, lb, ub, starts, kernel=0, metric=0):
    """Maximiser of the oracle log-likelihood on the box [lb, ub] (lb > 0):
    scipy's L-BFGS-B in log-parameters with a 4th-order central-difference
    gradient (h = 1e-5 in log theta), from each start; the best is returned
    as (theta_hat, loglik).  The reference's own driver is derivative-free
    (NLopt BOBYQA, synthetic_dmle_test.c:140-142), which is not available
    here, so the oracle's maximiser is defined by this independent method."""
    from scipy.optimize import minimize

    x, y, z = _f64(x), _f64(y), _f64(z)
    lb, ub = _f64(lb), _f64(ub)
    n = lb.size

    def negll(phi):
        try:
            return -dmle(x, y, z, np.exp(phi), kernel, metric)[0]
        except RuntimeError:
            return 1e30

    def grad(phi, h=1e-5):
        g = np.zeros(n)
        for k in range(n):
            e = np.zeros(n)
            e[k] = h
            g[k] = (8 * (negll(phi + e) - negll(phi - e)) - (negll(phi + 2 * e) - negll(phi - 2 * e))) / (12 * h)
        return g

    best = None
    for start in starts:
        r = minimize(negll, np.log(_f64(start)), jac=grad, method="L-BFGS-B",
                     bounds=list(zip(np.log(lb), np.log(ub))), options=dict(ftol=1e-15, gtol=1e-9, maxiter=500))
        if best is None or r.fun < best.fun:
            best = r
    return np.exp(best.x), -best.fun
