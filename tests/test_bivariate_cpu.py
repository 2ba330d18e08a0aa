"""Bivariate parsimonious Matern (kernel 2) in the oracle, pinned against an
independent scipy restatement of the model (Gneiting, Kleiber & Schlather,
JASA 2010, parsimonious bivariate Matern) and against the univariate kernel
(no GPU)."""
import numpy as np
from scipy.special import gamma, kv


def _matern(d, sigma2, beta, nu):
    r = d / beta
    out = np.full(r.shape, sigma2, dtype=float)
    nz = r > 0
    out[nz] = sigma2 * 2 ** (1 - nu) / gamma(nu) * r[nz] ** nu * kv(nu, r[nz])
    return out


def _bivariate(x, y, theta):
    s1, s2, beta, nu1, nu2, rho = theta
    nu12 = 0.5 * (nu1 + nu2)
    rho_eff = rho * np.sqrt(gamma(nu1 + 1) * gamma(nu2 + 1) / (gamma(nu1) * gamma(nu2))) * gamma(nu12) / gamma(nu12 + 1)
    d = np.hypot(x[:, None] - x[None, :], y[:, None] - y[None, :])
    n = x.size
    C = np.empty((2 * n, 2 * n))
    C[0::2, 0::2] = _matern(d, s1, beta, nu1)
    C[1::2, 1::2] = _matern(d, s2, beta, nu2)
    cross = _matern(d, 1.0, beta, nu12) * rho_eff * np.sqrt(s1 * s2)
    C[0::2, 1::2] = cross
    C[1::2, 0::2] = cross
    return C


def test_oracle_bivariate_matches_scipy(ora):
    x, y = ora.generate_xy_loc(150, 3)
    for theta in ([1.0, 2.0, 0.1, 0.5, 1.2, 0.4], [0.7, 1.3, 0.05, 1.0, 0.6, -0.3]):
        C = ora.covariance_full(x, y, theta, kernel=2)
        ref = _bivariate(x, y, theta)
        assert C.shape == (300, 300)
        assert np.abs(C - ref).max() < 1e-13 * np.abs(ref).max()
        assert np.linalg.eigvalsh(C).min() > 0


def test_oracle_bivariate_uncorrelated_is_two_univariate_fields(ora):
    """rho = 0: Sigma is block diagonal after de-interleaving, so the
    log-likelihood is the sum of the two univariate ones."""
    theta = [1.3, 0.8, 0.1, 0.7, 1.1, 0.0]
    N = 600
    x, y, z, _ = ora.synthetic_field(N, 5, theta, kernel=2)
    assert x.size == N // 2 and z.size == N
    ll = ora.dmle(x, y, z, theta, kernel=2)[0]
    l0 = ora.dmle(x, y, z[0::2], [theta[0], theta[2], theta[3]])[0]
    l1 = ora.dmle(x, y, z[1::2], [theta[1], theta[2], theta[4]])[0]
    assert ll == __import__("pytest").approx(l0 + l1, rel=1e-12)
