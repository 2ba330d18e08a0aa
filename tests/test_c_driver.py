"""The C driver in tests/c_driver (the reference driver's call sequence,
written against include/exageostat_b200.h only) compiles with -Wall -Werror
and links against the library (CPU); on the GPU it runs the C1 workflow
(N = 1600, tile 320, 100 held out) end to end with the reference's dlarnv
draws read from a file, and its values are checked against the oracle
running the same workflow: l(theta0) and the checksums of z to 1e-10,
theta-hat against the oracle's maximiser to 1e-3, and the kriging MSE and
predictions at the driver's theta-hat to 1e-9."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(xg, tmp_path):
    exe = tmp_path / "synthetic_dmle"
    libdir = os.path.dirname(xg.LIB_PATH)
    subprocess.run(["gcc", "-std=c11", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_driver", "synthetic_dmle.c"), "-o", str(exe), "-L", libdir,
                    "-lexageostat_b200", "-Wl,-rpath," + libdir, "-lm"], check=True)
    return exe


def test_c_driver_compiles_and_links(xg, tmp_path):
    exe = _build(xg, tmp_path)
    assert exe.exists()


@pytest.mark.gpu
def test_c_driver_runs_the_reference_workflow(xg, ora, tmp_path):
    N, dts, nmiss, seed = 1600, 320, 100, 0
    theta0 = [1.0, 0.1, 0.5]
    exe = _build(xg, tmp_path)
    e = ora.dlarnv(seed, N)
    nrand = tmp_path / "nrand.txt"
    nrand.write_text("".join("%.17g\n" % v for v in e))
    env = dict(os.environ, EXAGEOSTAT_B200_SILENT="1")
    r = subprocess.run([str(exe), str(N), str(dts), str(nmiss), str(seed), str(nrand)], capture_output=True,
                       text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    kv = dict(item.split("=", 1) for item in r.stdout.strip().splitlines()[-1].split())
    theta = np.array([float(v) for v in kv["theta"].split(",")])
    assert int(kv["evals"]) > 10
    # the oracle workflow on the same locations and draws
    x, y = ora.generate_xy_loc(N, seed)
    z = ora.dzvg(x, y, theta0, e)
    assert float(kv["zsum"]) == pytest.approx(z.sum(), rel=1e-10, abs=1e-10 * np.abs(z).sum())
    assert float(kv["zsq"]) == pytest.approx((z * z).sum(), rel=1e-10)
    assert float(kv["loglik0"]) == pytest.approx(ora.dmle(x, y, z, theta0)[0], rel=1e-10)
    lb, ub = np.full(3, 0.01), np.full(3, 5.0)
    th_ora, ll_ora = ora.maximise(x, y, z, lb, ub, [[0.5, 0.5, 0.5], theta0])
    assert np.all(np.abs(theta - th_ora) <= 1e-3 * th_ora), (theta, th_ora)
    assert float(kv["loglik"]) == pytest.approx(ll_ora, abs=1e-6)
    # kriging at the driver's theta-hat, hold-out drawn after GenerateXYLoc's 2 N draws
    split = ora.pick_random_points(x, y, z, nmiss, seed=seed)
    mse, zm = ora.dpredict(split["x_miss"], split["y_miss"], split["x_obs"], split["y_obs"], split["z_obs"],
                           split["z_actual"], theta)
    assert float(kv["mse"]) == pytest.approx(mse, rel=1e-9)
    assert float(kv["pred_sum"]) == pytest.approx(zm.sum(), rel=1e-9, abs=1e-9 * np.abs(zm).sum())
