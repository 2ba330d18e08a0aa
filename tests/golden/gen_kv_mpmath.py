"""Generate K_nu(x) golden values with mpmath (40 significant digits).

The reference evaluates the Matern kernel with GSL's gsl_sf_bessel_Knu
(exageostat_exact/cpu_core/compute/core_zcmg.c:987).  GSL is not available,
so both the CPU oracle and the GPU kernels are pinned to mpmath's besselk
over the (nu, x) range the MLE explores: nu in [0.01, 5] (the optimizer
bounds of the reference's tests) and x = d / beta in [1e-6, 700].

Usage: python tests/golden/gen_kv_mpmath.py   (writes kv_mpmath.json beside it)
"""
import json
import os

import mpmath as mp

mp.mp.dps = 40

NUS = [0.01, 0.1, 0.25, 0.333, 0.5, 0.73, 0.999, 1.0, 1.25, 1.5, 1.77, 2.0, 2.5, 2.9, 3.5, 4.0, 4.49, 5.0]
XS = [1e-6, 1e-4, 1e-3, 0.01, 0.05, 0.1, 0.3, 0.5, 0.9, 1.0, 1.5, 1.9, 1.999, 2.0, 2.001, 2.5, 3.0, 4.0, 5.5,
      8.0, 12.0, 20.0, 35.0, 60.0, 100.0, 200.0, 400.0, 700.0]


def main():
    rows = []
    for nu in NUS:
        for x in XS:
            k = mp.besselk(nu, x)
            dk = mp.diff(lambda v: mp.besselk(v, x), nu)
            rows.append({"nu": nu, "x": x, "k": mp.nstr(k, 25), "dk_dnu": mp.nstr(dk, 25)})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kv_mpmath.json")
    with open(out, "w") as f:
        json.dump({"generator": "mpmath %s besselk, dps=40" % mp.__version__, "rows": rows}, f, indent=0)
    print("wrote", out, len(rows))


if __name__ == "__main__":
    main()
