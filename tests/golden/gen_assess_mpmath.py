"""Golden Fisher matrices and MLOE / MMOM values computed entirely in mpmath
(30 digits), for small fields.

Locations follow GenerateXYLoc (restated in gen_loglik_mpmath.py).  The
covariance is the Matern formula of core_zcmg.c:963-994 with mpmath besselk.

* Fisher (EXAGEOSTAT_Fisher_Tile, MLE_dexact.c:1777-1934):
  F_jk = 1/2 tr(Sigma^-1 dSigma_j Sigma^-1 dSigma_k) over (sigma^2, beta, nu)
  (+ tau^2 for the nugget kernel, dSigma = I), with the element derivatives
  taken by mpmath differentiation of the element itself (d/d sigma^2 exact);
  zero distance gives 1, 0, 0 as core_zcmg.c:331-332, 394-395, 471-472.
* MLOE / MMOM (EXAGEOSTAT_dmle_mloe_mmom_Tile, MLE_dexact.c:1109-1434 and
  codelet_zmloe_mmom.c:22-60): per missing point
  expr1 = k_t' K_a^-1 k_a, expr2 = s_t - 2 expr1 + k_a' K_a^-1 K_t K_a^-1 k_a,
  expr3 = s_t - k_t' K_t^-1 k_t, expr4 = s_a - k_a' K_a^-1 k_a,
  loe = expr2 / expr3 - 1, mom = expr4 / expr2 - 1, then the means.

Usage: python tests/golden/gen_assess_mpmath.py   (writes assess_mpmath.json)
"""
import json
import math
import os
import sys

import mpmath as mp

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from gen_loglik_mpmath import generate_xy_loc, matern  # noqa: E402

mp.mp.dps = 30


def _dist(x1, y1, x2, y2):
    return math.sqrt((x2 - x1) ** 2 + (y2 - y1) ** 2)


def _cov(xa, ya, xb, yb, theta, kernel):
    S = mp.matrix(len(xa), len(xb))
    for i in range(len(xa)):
        for j in range(len(xb)):
            S[i, j] = matern(_dist(xa[i], ya[i], xb[j], yb[j]), theta, kernel)
    return S


def _deriv(d, theta, which):
    """d Sigma / d theta_which of one element (Matern part)."""
    s2, beta, nu = (mp.mpf(t) for t in theta[:3])
    if d == 0:
        return mp.mpf(1) if which == 0 else mp.mpf(0)
    if which == 0:
        return matern(d, [1.0, theta[1], theta[2]], 0)
    if which == 1:
        return mp.diff(lambda b: matern(d, [s2, b, nu], 0), beta)
    return mp.diff(lambda v: matern(d, [s2, beta, v], 0), nu)


def fisher(x, y, theta, kernel):
    n = len(x)
    S = mp.inverse(_cov(x, y, x, y, theta, kernel))
    D = []
    for which in range(3):
        M = mp.matrix(n, n)
        for i in range(n):
            for j in range(i + 1):
                M[i, j] = M[j, i] = _deriv(_dist(x[i], y[i], x[j], y[j]), theta, which)
        D.append(M)
    if kernel == 1:
        D.append(mp.eye(n))
    G = [S * Dj for Dj in D]
    npar = len(D)
    F = [[None] * npar for _ in range(npar)]
    for j in range(npar):
        for k in range(j, npar):
            t = mp.fsum(G[j][a, b] * G[k][b, a] for a in range(n) for b in range(n))
            F[j][k] = F[k][j] = t / 2
    return F


def mloe_mmom(xm, ym, xo, yo, truth, est, kernel):
    Ka = _cov(xo, yo, xo, yo, est, kernel)
    Kt = _cov(xo, yo, xo, yo, truth, kernel)
    Kai, Kti = mp.inverse(Ka), mp.inverse(Kt)
    kt = _cov(xo, yo, xm, ym, truth, kernel)
    ka = _cov(xo, yo, xm, ym, est, kernel)
    st, sa = mp.mpf(truth[0]), mp.mpf(est[0])
    terms = []
    for p in range(len(xm)):
        a = ka[:, p]
        t = kt[:, p]
        w = Kai * a
        e1 = (t.T * w)[0]
        e2 = st - 2 * e1 + (w.T * Kt * w)[0]
        e3 = st - (t.T * (Kti * t))[0]
        e4 = sa - (a.T * w)[0]
        loe = -1 if e3 == 0 else e2 / e3 - 1
        mom = -1 if e2 == 0 else e4 / e2 - 1
        terms.append([e1, e2, e3, e4, loe, mom])
    m = len(xm)
    return mp.fsum(r[4] for r in terms) / m, mp.fsum(r[5] for r in terms) / m, terms


FISHER_CASES = [
    {"name": "matern_nu0.5", "n": 25, "seed": 0, "theta": [1.0, 0.1, 0.5], "kernel": 0},
    {"name": "matern_nu0.73", "n": 30, "seed": 1, "theta": [1.3, 0.07, 0.73], "kernel": 0},
    {"name": "matern_nu1.5", "n": 20, "seed": 2, "theta": [0.8, 0.1, 1.5], "kernel": 0},
    {"name": "nugget_nu1.0", "n": 24, "seed": 4, "theta": [1.0, 0.1, 1.0, 0.01], "kernel": 1},
]

MLOE_CASES = [
    {"name": "matern", "n": 36, "nmiss": 6, "seed": 5, "truth": [1.0, 0.1, 0.5], "est": [0.9, 0.12, 0.6],
     "kernel": 0},
    {"name": "nugget", "n": 30, "nmiss": 5, "seed": 6, "truth": [1.0, 0.1, 1.0, 0.01],
     "est": [1.2, 0.08, 0.8, 0.02], "kernel": 1},
]


def _s(v):
    return mp.nstr(v, 25)


def main():
    out = {"generator": "mpmath %s, dps=30" % mp.__version__, "fisher": [], "mloe_mmom": []}
    for c in FISHER_CASES:
        x, y = generate_xy_loc(c["n"], c["seed"])
        F = fisher(x, y, c["theta"], c["kernel"])
        out["fisher"].append(dict(c, x=x, y=y, F=[[_s(v) for v in row] for row in F]))
        print("fisher", c["name"], mp.nstr(F[0][0], 15), mp.nstr(F[-1][-1], 15))
    for c in MLOE_CASES:
        x, y = generate_xy_loc(c["n"], c["seed"])
        k = c["nmiss"]
        ml, mm, terms = mloe_mmom(x[:k], y[:k], x[k:], y[k:], c["truth"], c["est"], c["kernel"])
        out["mloe_mmom"].append(dict(c, x=x, y=y, mloe=_s(ml), mmom=_s(mm),
                                     terms=[[_s(v) for v in r] for r in terms]))
        print("mloe", c["name"], mp.nstr(ml, 15), mp.nstr(mm, 15))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "assess_mpmath.json")
    with open(path, "w") as f:
        json.dump(out, f)
    print("wrote", path)


if __name__ == "__main__":
    main()
