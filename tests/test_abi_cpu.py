"""C-ABI library: loads, exports every declared symbol, layout matches (no GPU)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    with open(os.path.join(ROOT, "include", "exageostat_b200.h")) as f:
        src = f.read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = set(re.findall(r"^\s*(?:[A-Za-z_][\w\s\*]*?[\s\*])([A-Za-z_]\w*)\s*\(", src, flags=re.M))
    return sorted(n for n in names if n not in ("if", "while", "for", "return", "sizeof"))


def test_library_exports_every_declared_symbol(xg):
    L = xg.lib()
    declared = _declared_functions()
    assert "MLE_alg" in declared and "EXAGEOSTAT_dmle_Predict_Tile" in declared
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing
    assert hasattr(L, "results")
    for n in xg.EXPORTED_SYMBOLS:
        assert hasattr(L, n), n


def test_struct_layout_matches_library(xg):
    xg.check_abi()
    L = xg.lib()
    assert L.exageostat_b200_offsetof_MLE_data(b"seed") == xg.MLEData.seed.offset
    assert L.exageostat_b200_offsetof_MLE_data(b"no_such_field") == -1


def test_host_generate_xy_loc_matches_oracle(xg, ora):
    for n, seed in ((1600, 0), (1000, 7), (37, 3)):
        x1, y1 = xg.generate_xy_loc(n, seed)
        x2, y2 = ora.generate_xy_loc(n, seed)
        assert np.array_equal(x1, x2) and np.array_equal(y1, y2)


def test_host_zsort_and_shuffle_match_oracle(xg, ora):
    """locations_obs_zsort_inplace and the libc-rand shuffle of the library
    reproduce the oracle bit for bit."""
    L = xg.lib()
    rng = np.random.default_rng(0)
    n = 500
    x, y, z = rng.random(n), rng.random(n), rng.standard_normal(n)
    loc = xg.Location()
    xa, ya, za = x.copy(), y.copy(), z.copy()
    loc.x, loc.y = xa.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ya.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    L.locations_obs_zsort_inplace(n, ctypes.byref(loc), za.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    xb, yb, zb = x.copy(), y.copy(), z.copy()
    ora.lib().ora_locations_obs_zsort_inplace(n, *(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in (xb, yb, zb)))
    assert np.array_equal(xa, xb) and np.array_equal(ya, yb) and np.array_equal(za, zb)


def test_device_bessel_code_compiled_for_host_matches_mpmath(tmp_path):
    """The device K_nu source (kbessel.cuh) is host/device code; compile it
    with g++ and check it against the mpmath golden values."""
    import json

    src = tmp_path / "kv.cpp"
    src.write_text('#include <cstdio>\n#include "kbessel.cuh"\nint main(){double a,b;'
                   'while(scanf("%lf %lf",&a,&b)==2)printf("%.17g\\n",xg_bessel_knu(a,b));}\n')
    exe = tmp_path / "kv"
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "exageostat_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    rows = json.load(open(os.path.join(ROOT, "tests", "golden", "kv_mpmath.json")))["rows"]
    inp = "\n".join("%r %r" % (r["nu"], r["x"]) for r in rows)
    out = subprocess.run([str(exe)], input=inp, capture_output=True, text=True, check=True).stdout.split()
    rel = [abs(float(v) - float(r["k"])) / float(r["k"]) for r, v in zip(rows, out)]
    assert max(rel) < 1e-14, max(rel)


def test_device_matern_element_compiled_for_host_matches_mpmath(tmp_path):
    """The Matern element of the covariance generators (xg_matern_general:
    Temme's series with the order constants and r^nu from its own power for
    r <= 2, the trapezoidal rule, the asymptotic expansion for r >= 20),
    compiled for the host, against mpmath's r^nu K_nu(r) on a grid of orders
    and distances that crosses every branch boundary."""
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.dps = 30
    src = tmp_path / "m.cpp"
    src.write_text('#include <cstdio>\n#include "kbessel.cuh"\nint main(){double a,b;'
                   'while(scanf("%lf %lf",&a,&b)==2)printf("%.17g\\n",xg_matern_general(b,a,1.0));}\n')
    exe = tmp_path / "m"
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "exageostat_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    pts = [(nu, float(r)) for nu in (0.01, 0.3, 0.5, 0.73, 1.0, 1.37, 2.5, 3.3, 4.99, 5.0, 5.5)
           for r in list(np.geomspace(1e-4, 2.0, 9)) + [2.0000001, 3.0, 7.0, 12.5, 19.99, 20.0, 20.01, 25.0, 40.0,
                                                         80.0, 200.0]]
    out = subprocess.run([str(exe)], input="\n".join("%r %r" % p for p in pts), capture_output=True, text=True,
                         check=True).stdout.split()
    rel = [abs(float(v) / float(mpmath.power(r, nu) * mpmath.besselk(nu, r)) - 1.0) for (nu, r), v in zip(pts, out)]
    assert len(rel) == len(pts) and max(rel) < 2e-14, max(rel)


def test_branch_grouped_generation_gives_the_same_bits(tmp_path):
    """The generators that group elements by K_nu branch (xg_matern_branch,
    then xg_matern_small_c / _trap / _asym) must give the same bits as the
    one-call element (xg_matern_general_c) for every r and order."""
    src = tmp_path / "b.cpp"
    src.write_text('#include <cstdio>\n#include <cstring>\n#include "kbessel.cuh"\n'
                   'int main(){double nu,r;int bad=0,n=0;while(scanf("%lf %lf",&nu,&r)==2){++n;'
                   'XgTemme tc=xg_temme_consts(nu);double con=1.7;double a=xg_matern_general_c(r,nu,con,tc);'
                   'int q=xg_matern_branch(r,nu);double b=q==0?xg_matern_small_c(r,con,tc):'
                   'q==3?xg_matern_asym(r,nu,con):xg_matern_trap(r,nu,con);'
                   'if(memcmp(&a,&b,8))++bad;}printf("%d %d\\n",n,bad);}\n')
    exe = tmp_path / "b"
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "exageostat_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    pts = ["%r %r" % (nu, float(r)) for nu in (0.01, 0.37, 0.5, 0.73, 1.0, 2.2, 4.99, 5.0, 5.5)
           for r in np.concatenate([np.geomspace(1e-5, 2.0, 40), [2.0, 6.0, 19.999, 20.0]], axis=None).tolist()
           + np.geomspace(2.0001, 600.0, 60).tolist()]
    out = subprocess.run([str(exe)], input="\n".join(pts), capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == len(pts) and int(out[1]) == 0


def test_product_fails_loudly_without_library(xg, monkeypatch):
    monkeypatch.setattr(xg, "_lib", None)
    monkeypatch.setattr(xg, "LIB_PATH", "/nonexistent/libexageostat_b200.so")
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        xg.lib()
