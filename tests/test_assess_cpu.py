"""Assessment oracle (Fisher information, MLOE / MMOM) pinned on CPU, and the
device element derivatives compiled for the host against it (no GPU).

Pins (the reference has no tests for these routines):
  * dSigma/dtheta element kernels == central differences of the covariance
    generator, itself pinned to mpmath through K_nu;
  * F_{sigma^2 sigma^2} = N / (2 sigma^4) exactly for the Matern kernel
    (dSigma/dsigma^2 = Sigma / sigma^2);
  * MLOE = MMOM = 0 when the estimate equals the truth; with only the variance
    scaled by c, the kriging weights are unchanged, so MLOE = 0 and MMOM = c - 1.
"""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("theta", [[1.3, 0.1, 0.7], [0.8, 0.05, 1.5], [1.0, 0.2, 0.5]])
def test_oracle_derivatives_match_covariance_differences(ora, theta):
    n = 150
    x, y = ora.generate_xy_loc(n, 1)
    for j in range(3):
        D = ora.dcmg_deriv(n, n, 0, 0, x, y, x, y, theta, j)
        h = 1e-5 * theta[j]
        tp, tm = list(theta), list(theta)
        tp[j] += h
        tm[j] -= h
        fd = (ora.covariance_full(x, y, tp) - ora.covariance_full(x, y, tm)) / (2 * h)
        assert np.abs(D - fd).max() / np.abs(D).max() < 1e-8, j


def test_oracle_fisher_identities(ora):
    n = 250
    x, y = ora.generate_xy_loc(n, 2)
    theta = [1.3, 0.1, 0.7]
    F, Finv = ora.fisher(x, y, theta)
    assert F[0, 0] == pytest.approx(n / (2 * theta[0] ** 2), rel=1e-12)
    assert np.allclose(F, F.T)
    assert np.allclose(Finv @ F, np.eye(3), atol=1e-10)
    F4, F4inv = ora.fisher(x, y, [1.3, 0.1, 0.7, 0.05], kernel=1)
    assert F4.shape == (4, 4) and np.all(np.linalg.eigvalsh(F4) > 0)
    assert np.allclose(F4inv @ F4, np.eye(4), atol=1e-9)


def test_oracle_mloe_mmom_identities(ora):
    x, y = ora.generate_xy_loc(300, 4)
    xo, yo, xm, ym = x[:240], y[:240], x[240:], y[240:]
    theta = [1.3, 0.1, 0.7]
    mloe, mmom, terms = ora.mloe_mmom(xm, ym, xo, yo, theta, theta)
    assert abs(mloe) < 1e-12 and abs(mmom) < 1e-12
    c = 2.5
    mloe, mmom, _ = ora.mloe_mmom(xm, ym, xo, yo, theta, [c * theta[0], theta[1], theta[2]])
    assert abs(mloe) < 1e-12 and mmom == pytest.approx(c - 1, abs=1e-12)
    mloe, mmom, terms = ora.mloe_mmom(xm, ym, xo, yo, theta, [1.0, 0.05, 0.5])
    assert mloe > 0 and terms.shape == (60, 6)
    assert np.all(terms[:, 2] > 0) and np.all(terms[:, 1] >= terms[:, 2] * (1 - 1e-12))


def test_device_element_derivatives_match_oracle(ora, tmp_path):
    """xg_matern_grad (kbessel.cuh, host/device code) compiled with g++ against
    the oracle's restatement of the reference derivative kernels."""
    from scipy.special import digamma

    src = tmp_path / "dm.cpp"
    src.write_text('#include <cstdio>\n#include <cmath>\n#include "kbessel.cuh"\n'
                   'int main(){double r,nu,s2,b,dl;while(scanf("%lf %lf %lf %lf %lf",&r,&nu,&s2,&b,&dl)==5){'
                   'double con=s2/(pow(2.0,nu-1)*tgamma(nu));double m,ds,db,dn;'
                   'xg_matern_grad(r,nu,con,s2,b,dl,&m,&ds,&db,&dn);printf("%.17g %.17g %.17g\\n",ds,db,dn);}}\n')
    exe = tmp_path / "dm"
    subprocess.run(["g++", "-O2", "-I", os.path.join(ROOT, "exageostat_b200", "csrc"), str(src), "-o", str(exe)],
                   check=True)
    rows, ref = [], []
    for nu in (0.3, 0.5, 0.73, 1.0, 1.5, 2.5, 4.0):
        for beta in (0.05, 0.1, 0.3):
            th = [1.3, beta, nu]
            d = np.geomspace(1e-4, 3.0, 25)
            x1, y1 = np.zeros(1), np.zeros(1)
            for j in range(3):
                ref.append(ora.dcmg_deriv(1, d.size, 0, 0, x1, y1, d, np.zeros(d.size), th, j)[0])
            dl = -(np.log(2.0) + digamma(nu))
            rows += ["%r %r %r %r %r" % (float(dd / beta), nu, th[0], beta, float(dl)) for dd in d]
    out = subprocess.run([str(exe)], input="\n".join(rows), capture_output=True, text=True, check=True).stdout
    got = np.array(out.split(), dtype=float).reshape(-1, 3)
    want = np.concatenate([np.stack(ref[i:i + 3], axis=1) for i in range(0, len(ref), 3)])
    scale = np.abs(want).max(axis=0)
    err = np.abs(got - want).max(axis=0) / scale
    # the oracle's nu derivative (the reference's psi series, a central
    # difference of K_nu) is good to ~7e-10 of the largest entry; the device
    # function agrees with mpmath to ~1e-13
    assert np.all(err < 2e-9), err


def _golden():
    import json

    with open(os.path.join(ROOT, "tests", "golden", "assess_mpmath.json")) as f:
        return json.load(f)


def test_oracle_fisher_matches_mpmath(ora):
    """tests/golden/assess_mpmath.json (tests/golden/gen_assess_mpmath.py):
    30-digit Fisher matrices of small fields; the oracle's locations are the
    golden ones bit for bit and its F agrees to 1e-8 of sqrt(F_jj F_kk) (its
    nu derivative uses the reference's psi series and a difference quotient)."""
    for c in _golden()["fisher"]:
        x, y = ora.generate_xy_loc(c["n"], c["seed"])
        assert np.array_equal(x, c["x"]) and np.array_equal(y, c["y"])
        F, _ = ora.fisher(x, y, c["theta"], c["kernel"])
        G = np.array([[float(v) for v in row] for row in c["F"]])
        scale = np.sqrt(np.outer(np.diag(G), np.diag(G)))
        assert (np.abs(F - G) / scale).max() < 1e-8, (c["name"], F, G)


def test_oracle_mloe_mmom_matches_mpmath(ora):
    for c in _golden()["mloe_mmom"]:
        x, y = ora.generate_xy_loc(c["n"], c["seed"])
        k = c["nmiss"]
        mloe, mmom, terms = ora.mloe_mmom(x[:k], y[:k], x[k:], y[k:], c["truth"], c["est"], c["kernel"])
        G = np.array([[float(v) for v in r] for r in c["terms"]])
        assert np.abs(terms[:, :4] - G[:, :4]).max() < 1e-12 * c["truth"][0], c["name"]
        assert np.abs(terms[:, 4:] - G[:, 4:]).max() < 1e-10, c["name"]
        assert mloe == pytest.approx(float(c["mloe"]), abs=1e-11) and mmom == pytest.approx(float(c["mmom"]), abs=1e-11)


def test_device_formulations_equal_the_reference_sequences(ora):
    """The GPU computes MLOE / MMOM as A = L_a^-1 k_a, U = L_a^-1 k_t,
    T = L_t^-1 k_t, W = L_a^-T A, V = L_t^T W with expr1 = U.A,
    expr2 = s_t - 2 expr1 + V.V, expr3 = s_t - T.T, expr4 = s_a - A.A, and the
    Fisher matrix as tr(G_j G_k) with G_j = Sigma^-1 dSigma_j; restated here in
    numpy, both equal the oracle's restatement of the reference's own sequence
    (per-point TRSM/TRMM/GEMM, MLE_dexact.c:1300-1375; CJ CK products,
    :1846-1879) to rounding."""
    from scipy.linalg import solve_triangular

    x, y = ora.generate_xy_loc(400, 11)
    xo, yo, xm, ym = x[:340], y[:340], x[340:], y[340:]
    truth, est = [1.3, 0.1, 0.7], [1.0, 0.08, 0.9]
    La = np.linalg.cholesky(ora.covariance_full(xo, yo, est))
    Lt = np.linalg.cholesky(ora.covariance_full(xo, yo, truth))
    ka = ora.core_dcmg(340, 60, 0, 0, xo, yo, xm, ym, est)
    kt = ora.core_dcmg(340, 60, 0, 0, xo, yo, xm, ym, truth)
    A = solve_triangular(La, ka, lower=True)
    U = solve_triangular(La, kt, lower=True)
    T = solve_triangular(Lt, kt, lower=True)
    W = solve_triangular(La, A, lower=True, trans="T")
    V = Lt.T @ W
    e1 = np.sum(U * A, axis=0)
    e2 = (truth[0] - 2 * e1) + np.sum(V * V, axis=0)
    e3 = truth[0] - np.sum(T * T, axis=0)
    e4 = est[0] - np.sum(A * A, axis=0)
    _, _, ref = ora.mloe_mmom(xm, ym, xo, yo, truth, est)
    assert np.abs(np.stack([e1, e2, e3, e4], axis=1) - ref[:, :4]).max() < 1e-13
    # Fisher: traces of S dSigma_j S dSigma_k
    n = 200
    theta = [1.3, 0.1, 0.7]
    S = np.linalg.inv(ora.covariance_full(x[:n], y[:n], theta))
    G = [S @ ora.dcmg_deriv(n, n, 0, 0, x[:n], y[:n], x[:n], y[:n], theta, j) for j in range(3)]
    F = np.array([[0.5 * np.sum(G[j] * G[k].T) for k in range(3)] for j in range(3)])
    Fo, _ = ora.fisher(x[:n], y[:n], theta)
    assert np.abs(F - Fo).max() / np.abs(Fo).max() < 1e-10
