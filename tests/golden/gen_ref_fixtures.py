"""Writes tests/golden/ref_fixtures.npz and ref_fixtures.json from the
reference's OWN C code, compiled unchanged from the reference tree into
oracle/_ref (``make -C oracle ref``; see oracle/Makefile and oracle/ref.py).
Run where the reference tree is present:

    python tests/golden/gen_ref_fixtures.py

ref_fixtures.json: SHA-256 of the float64 bytes of the locations that
GenerateXYLoc(n, seed) returns (misc/compute/MLE_misc.c:763-792, with the
Morton sort and uint16 quantisation of :297-319) at the sizes of the
benchmark configurations, and of the six arrays of pick_random_points
(:1700-1741: shuffle :1238-1259 on libc rand() continuing after
GenerateXYLoc's 2 N draws, then locations_obs_zsort_inplace :453-534) with z
= the dlarnv draws of the same seed.

ref_fixtures.npz: 24 x 24 covariance tiles of core_dcmg (core_zcmg.c:963-994),
core_dcmg_nuggets (core_zcmg_nuggets.c:107-156),
core_dcmg_bivariate_parsimonious (core_zcmg.c:1628-1726),
core_dcmg_bivariate_flexible (core_zcmg.c:1514-1580), the great-circle
metric (distanceEarth, core_zcmg.c:51-60) and the derivative tiles
core_dcmg_matern_dsigma_square / _dbeta / _dnu (core_zcmg.c:315-488) on the
GenerateXYLoc(1600, 0) locations, and core_dmdet (core_zmdet.c:50-59) of a
factor tile.  K_nu inside the kernels is the oracle's (GSL is absent).
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from oracle import ref  # noqa: E402

LOC_CASES = [(37, 3), (400, 2), (1600, 0), (6400, 0), (20000, 0), (40000, 0), (100000, 0)]
PICK_CASES = [(1600, 0, 100), (40000, 0, 1000)]
TILE = 24
# (name, kernel, theta, metric); the tile positions are row/column offsets
COV_CASES = [
    ("matern_nu0.5", "matern", [1.0, 0.1, 0.5], 0),
    ("matern_nu0.73", "matern", [1.0, 0.1, 0.73], 0),
    ("matern_nu1.5", "matern", [1.0, 0.1, 1.5], 0),
    ("matern_nu2.5", "matern", [1.0, 0.05, 2.5], 0),
    ("matern_nu3.3", "matern", [2.0, 0.2, 3.3], 0),
    ("matern_edge", "matern", [0.7, 4.9, 0.011], 0),
    ("nuggets", "nuggets", [1.0, 0.1, 1.0, 0.01], 0),
    ("bivariate", "bivariate_parsimonious", [1.0, 1.5, 0.1, 0.5, 1.2, 0.3], 0),
    ("bivariate_flexible", "bivariate_flexible", [0.1, 0.15, 0.5, 0.5, 0.8, 1.2, 0.3, 0.5, 1.0, 1.1, 0.3], 0),
    ("great_circle", "matern", [1.0, 150.0, 0.73], 1),
    ("dsigma_square", "dsigma_square", [1.0, 0.1, 0.73], 0),
    ("dbeta", "dbeta", [1.0, 0.1, 0.73], 0),
    ("dnu", "dnu", [1.0, 0.1, 0.73], 0),
]
# even offsets: the bivariate kernel fills 2 x 2 blocks from an even corner
OFFSETS = [(0, 0), (320, 0), (1302, 976)]


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def latlon(x, y):
    """(latitude, longitude) in degrees for the great-circle tiles."""
    return 20.0 + 10.0 * x, 40.0 + 10.0 * y


def main():
    oracle.build()
    if ref.build() is None:
        raise SystemExit("the reference tree is absent: cannot compile oracle/_ref")
    meta = {"locations": {}, "pick_random_points": {}}
    for n, seed in LOC_CASES:
        x, y = ref.generate_xy_loc(n, seed)
        meta["locations"]["%d_%d" % (n, seed)] = {"x": sha(x), "y": sha(y), "x_first": x[:4].tolist(),
                                                  "y_last": y[-4:].tolist()}
    for n, seed, nmiss in PICK_CASES:
        x, y = ref.generate_xy_loc(n, seed)  # leaves libc rand() after 2 n draws
        z = oracle.dlarnv(seed, n)
        split = ref.pick_random_points(x, y, z, nmiss)
        meta["pick_random_points"]["%d_%d_%d" % (n, seed, nmiss)] = {k: sha(v) for k, v in split.items()}
    x, y = ref.generate_xy_loc(1600, 0)
    tiles = {}
    for name, kern, theta, metric in COV_CASES:
        a, b = latlon(x, y) if metric else (x, y)
        for m0, n0 in OFFSETS:
            tiles["%s_%d_%d" % (name, m0, n0)] = ref.cmg(kern, TILE, TILE, m0, n0, a, b, a, b, theta, metric)
    C = oracle.covariance_full(x[:64], y[:64], [1.0, 0.1, 0.73])
    L = np.linalg.cholesky(C)
    tiles["dmdet_factor"] = L
    meta["dmdet"] = ref.dmdet(L)
    meta["cov_cases"] = [[name, kern, theta, metric] for name, kern, theta, metric in COV_CASES]
    meta["offsets"] = OFFSETS
    meta["tile"] = TILE
    np.savez_compressed(os.path.join(HERE, "ref_fixtures.npz"), **tiles)
    with open(os.path.join(HERE, "ref_fixtures.json"), "w") as f:
        json.dump(meta, f, indent=1)


if __name__ == "__main__":
    main()
