"""Golden log-likelihoods computed entirely in mpmath (30 digits).

Locations follow GenerateXYLoc (misc/compute/MLE_misc.c:763-792: libc
rand() jitter of a ceil(sqrt n)^2 grid, Morton sort, uint16 quantisation),
restated here in Python with libc's rand() through ctypes.  z is a fixed
N(0,1) vector from numpy (stored in the file).  Sigma uses the Matern formula
of core_zcmg.c:963-994 with mpmath besselk; loglik = -0.5 z^T Sigma^-1 z -
0.5 log|Sigma| - (N/2) log(2 pi) (MLE_dexact.c:426) via an mpmath Cholesky.

Usage: python tests/golden/gen_loglik_mpmath.py   (writes loglik_mpmath.json)
"""
import ctypes
import json
import math
import os

import mpmath as mp
import numpy as np

mp.mp.dps = 30
libc = ctypes.CDLL(None)
RAND_MAX = 2147483647


def spread(v):
    v &= 0xFFFF
    out = 0
    for b in range(16):
        out |= ((v >> b) & 1) << (2 * b)
    return out


def compact(v):
    out = 0
    for b in range(16):
        out |= ((v >> (2 * b)) & 1) << b
    return out


def generate_xy_loc(n, seed):
    libc.srand(seed)
    side = int(math.ceil(math.sqrt(n)))
    xs, ys = [], []
    for i in range(side):
        for j in range(side):
            if len(xs) >= n:
                break
            u = libc.rand() / (1.0 + RAND_MAX)
            xs.append(((i + 1) - 0.5 + (u * 0.8 + -0.4)) / side)
            u = libc.rand() / (1.0 + RAND_MAX)
            ys.append(((j + 1) - 0.5 + (u * 0.8 + -0.4)) / side)
    codes = sorted((spread(int(y * 65535.0 + .5)) << 1) + spread(int(x * 65535.0 + .5)) for x, y in zip(xs, ys))
    x = [compact(c) / 65535.0 for c in codes]
    y = [compact(c >> 1) / 65535.0 for c in codes]
    return x, y


def matern(d, theta, kernel):
    s2, beta, nu = (mp.mpf(t) for t in theta[:3])
    r = mp.mpf(d) / beta
    if r == 0:
        return s2 + (mp.mpf(theta[3]) if kernel == 1 else 0)
    return s2 / (mp.power(2, nu - 1) * mp.gamma(nu)) * mp.power(r, nu) * mp.besselk(nu, r)


def loglik(x, y, z, theta, kernel):
    n = len(x)
    S = mp.matrix(n, n)
    for i in range(n):
        for j in range(i + 1):
            d = math.sqrt((x[j] - x[i]) ** 2 + (y[j] - y[i]) ** 2)
            S[i, j] = S[j, i] = matern(d, theta, kernel)
    L = mp.cholesky(S)
    # forward substitution
    w = [mp.mpf(0)] * n
    for i in range(n):
        s = mp.mpf(z[i])
        for k in range(i):
            s -= L[i, k] * w[k]
        w[i] = s / L[i, i]
    dot = mp.fsum(t * t for t in w)
    logdet = 2 * mp.fsum(mp.log(L[i, i]) for i in range(n))
    ll = -dot / 2 - logdet / 2 - mp.mpf(n) / 2 * mp.log(2 * mp.pi)
    return ll, logdet, dot


CASES = [
    {"name": "matern_nu0.5", "n": 60, "seed": 0, "theta": [1.0, 0.1, 0.5], "kernel": 0},
    {"name": "matern_nu0.73", "n": 60, "seed": 1, "theta": [1.3, 0.07, 0.73], "kernel": 0},
    {"name": "matern_nu1.5", "n": 49, "seed": 2, "theta": [0.8, 0.3, 1.5], "kernel": 0},
    {"name": "matern_nu2.5", "n": 36, "seed": 3, "theta": [1.0, 0.05, 2.5], "kernel": 0},
    {"name": "nugget_nu1.0", "n": 50, "seed": 4, "theta": [1.0, 0.1, 1.0, 0.01], "kernel": 1},
]


def main():
    out = []
    for c in CASES:
        x, y = generate_xy_loc(c["n"], c["seed"])
        z = np.random.default_rng(100 + c["seed"]).standard_normal(c["n"]).tolist()
        ll, ld, dot = loglik(x, y, z, c["theta"], c["kernel"])
        out.append(dict(c, x=x, y=y, z=z, loglik=mp.nstr(ll, 25), logdet=mp.nstr(ld, 25), dotp=mp.nstr(dot, 25)))
        print(c["name"], mp.nstr(ll, 20))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "loglik_mpmath.json")
    with open(path, "w") as f:
        json.dump({"generator": "mpmath %s, dps=30" % mp.__version__, "cases": out}, f)
    print("wrote", path)


if __name__ == "__main__":
    main()
