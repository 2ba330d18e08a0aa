"""The C driver in tests/c_driver (the reference driver's call sequence,
written against include/exageostat_b200.h only) compiles with -Wall -Werror
and links against the library (CPU); on the GPU it runs the C1 workflow
(N = 1600, tile 320, 100 held out) end to end."""
import os
import subprocess

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
def test_c_driver_runs_the_reference_workflow(xg, tmp_path):
    exe = _build(xg, tmp_path)
    env = dict(os.environ, EXAGEOSTAT_B200_SILENT="1")
    r = subprocess.run([str(exe), "1600", "320", "100", "0"], capture_output=True, text=True, env=env, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    kv = dict(item.split("=", 1) for item in r.stdout.strip().splitlines()[-1].split())
    theta = [float(v) for v in kv["theta"].split(",")]
    assert all(0.01 <= t <= 5 for t in theta) and int(kv["evals"]) > 10
    assert 0 <= float(kv["mse"]) < 1.0
