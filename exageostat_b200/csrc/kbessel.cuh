/*
 * Modified Bessel function of the second kind K_nu(x) and the Matern
 * covariance element, for host and device code.
 *
 * The reference evaluates every covariance element with GSL's
 * gsl_sf_bessel_Knu (exageostat_exact/cpu_core/compute/core_zcmg.c:987) on the
 * CPU.  This header is the project's own K_nu, written for the GPU from two
 * published methods:
 *
 *   x <= 2 : Temme's series for K_mu, K_{mu+1} with |mu| <= 1/2
 *            (N. M. Temme, J. Comput. Phys. 19 (1975) 324-337), then forward
 *            recurrence in the order up to nu = mu + n.
 *   x >  2 : the trapezoidal rule on the integral representation
 *              e^x K_nu(x) = int_0^inf exp(-2 x sinh^2(t/2)) cosh(nu t) dt
 *            (DLMF 10.32.9).  The integrand is even and analytic in a strip,
 *            so the trapezoidal rule converges geometrically (Trefethen &
 *            Weideman, SIAM Rev. 56 (2014) 385-458).  The step
 *            h = min(0.1615, 0.57 / sqrt(x)) keeps the quadrature error below
 *            3e-16 for 0 <= nu <= 5, 2 <= x <= 700 (measured against mpmath);
 *            with rounding the whole evaluation stays within 7e-15 relative
 *            (worst near nu = 5, x = 2).  Larger orders shrink h by
 *            sqrt(5 / nu).  The same nodes give
 *            d/dnu K_nu and K_{nu-1}, which the gradient kernels use.
 *
 * Both branches run a short loop with no table lookups, so a warp whose
 * lanes hold different x stays mostly converged.
 */
#ifndef EXAGEOSTAT_B200_KBESSEL_CUH
#define EXAGEOSTAT_B200_KBESSEL_CUH

#include <math.h>

#include "rgamma_taylor.cuh"

#ifndef XG_HD
#ifdef __CUDACC__
#define XG_HD __host__ __device__
#else
#define XG_HD
#endif
#endif

#define XG_PI 3.141592653589793
#define XG_EPS 2.220446049250313e-16

/* Temme's series: K_mu(x) and K_{mu+1}(x) for |mu| <= 1/2, 0 < x <= 2. */
XG_HD inline void xg_k_temme(double mu, double x, double *k_mu, double *k_mu1)
{
    const double m2 = mu * mu;
    const double even = xg_rgamma_even(m2);
    const double odd = xg_rgamma_odd(m2);
    const double gamma1 = -odd;               /* (1/G(1-mu) - 1/G(1+mu)) / (2 mu) */
    const double gamma2 = even;               /* (1/G(1-mu) + 1/G(1+mu)) / 2 */
    const double rgamma_plus = even + mu * odd;  /* 1/G(1+mu) */
    const double rgamma_minus = even - mu * odd; /* 1/G(1-mu) */
    const double half_x = 0.5 * x;
    const double ln_two_over_x = -log(half_x);
    const double sigma = mu * ln_two_over_x;
    const double pimu = XG_PI * mu;
    const double pimu_over_sin = (pimu == 0.0) ? 1.0 : pimu / sin(pimu);
    const double shc = (sigma == 0.0) ? 1.0 : sinh(sigma) / sigma;
    const double pow_two_over_x = exp(sigma);
    double f = pimu_over_sin * (gamma1 * cosh(sigma) + gamma2 * shc * ln_two_over_x);
    double p = 0.5 * pow_two_over_x / rgamma_plus;
    double q = 0.5 / (pow_two_over_x * rgamma_minus);
    const double qx2 = half_x * half_x;
    double ck = 1.0, s0 = f, s1 = p;
    for (int k = 1; k < 200; ++k) {
        const double dk = (double)k;
        f = (dk * f + p + q) / (dk * dk - m2);
        ck *= qx2 / dk;
        p /= (dk - mu);
        q /= (dk + mu);
        const double t0 = ck * f;
        s0 += t0;
        s1 += ck * (p - dk * f);
        if (fabs(t0) < 0.25 * XG_EPS * fabs(s0)) break;
    }
    *k_mu = s0;
    *k_mu1 = s1 / half_x;
}

/* K_nu(x) for nu >= 0, 0 < x <= 2, by Temme's series and forward recurrence.
 * Also returns K_{nu-1}(x) (= K_{1-nu} by symmetry when nu < 1). */
XG_HD inline double xg_knu_small(double nu, double x, double *k_num1)
{
    const int n = (int)(nu + 0.5);
    const double mu = nu - n;
    double k0, k1;
    xg_k_temme(mu, x, &k0, &k1);
    if (n == 0) {
        /* K_{nu-1} = K_{mu-1} = K_{mu+1} - 2 mu / x K_mu */
        if (k_num1) *k_num1 = k1 - 2.0 * mu / x * k0;
        return k0;
    }
    for (int j = 1; j < n; ++j) {
        const double k2 = 2.0 * (mu + j) / x * k1 + k0;
        k0 = k1;
        k1 = k2;
    }
    if (k_num1) *k_num1 = k0;
    return k1;
}

/* Trapezoidal step for the integral representation (see the header). */
XG_HD inline double xg_trap_step(double nu, double x)
{
    double h = 0.57 / sqrt(x);
    h = h < 0.1615 ? h : 0.1615;
    if (nu > 5.0) h *= sqrt(5.0 / nu);
    return h;
}

/* e^x K_nu(x) for x > 2 by the trapezoidal rule. */
XG_HD inline double xg_knu_scaled_trap(double nu, double x)
{
    const double h = xg_trap_step(nu, x);
    /* (s_k, q_k) = (sinh, cosh)(k h / 2) advance by the hyperbolic addition
     * formulas (relative error grows only linearly in k); c_k = cosh(nu k h)
     * by its three-term recurrence (a growing sequence, so stable). */
    const double sh = sinh(0.5 * h), chh = cosh(0.5 * h);
    const double two_cnh = 2.0 * cosh(nu * h);
    double s = sh, q = chh;
    double c_prev = 1.0, c = 0.5 * two_cnh;
    double sum = 0.5;
    for (int k = 1; k < 400; ++k) {
        const double g = exp(-2.0 * x * s * s) * c;
        sum += g;
        /* past the maximum of the integrand (x sinh t > nu) and negligible */
        if (g < 1e-17 * sum && 2.0 * x * s * q > nu) break;
        const double s_next = s * chh + q * sh;
        q = q * chh + s * sh;
        s = s_next;
        const double c_next = two_cnh * c - c_prev;
        c_prev = c;
        c = c_next;
    }
    return h * sum;
}

/* K_nu(x), nu >= 0, x > 0. */
XG_HD inline double xg_bessel_knu(double nu, double x)
{
    if (x <= 2.0) return xg_knu_small(nu, x, nullptr);
    return xg_knu_scaled_trap(nu, x) * exp(-x);
}

/* Matern element con * r^nu * K_nu(r), r = d / beta > 0, for general nu
 * (core_zcmg.c:987).  The large-r branch folds r^nu e^-r into one exp so it
 * neither overflows nor underflows early. */
XG_HD inline double xg_matern_general(double r, double nu, double con)
{
    if (r <= 2.0) return con * pow(r, nu) * xg_knu_small(nu, r, nullptr);
    return con * exp(nu * log(r) - r) * xg_knu_scaled_trap(nu, r);
}

/* e^x K_nu(x), e^x K_{nu-1}(x) and e^x dK_nu/dnu(x) for all x > 0 from one
 * trapezoidal sum over the integral representation (DLMF 10.32.9 and its nu
 * derivative, int t sinh(nu t) e^{-x cosh t} dt).  For x <= 2 the step is
 * 0.145 and the sum runs to where the integrand has decayed (at most ~130
 * nodes for x >= 1e-6); measured against mpmath the nu derivative stays
 * within 1.2e-12 of K_nu(x) for 0 <= nu <= 5.  Used by the gradient kernels. */
XG_HD inline void xg_knu_trap3(double nu, double x, double *k, double *km1, double *dk)
{
    double h = (x > 2.0) ? xg_trap_step(nu, x) : 0.145;
    if (x <= 2.0 && nu > 5.0) h *= sqrt(5.0 / nu);
    const double sh = sinh(0.5 * h), chh = cosh(0.5 * h);
    double s = sh, q = chh;
    const double e_nu = exp(nu * h), e_m1 = exp((nu - 1.0) * h);
    double pn = e_nu, pm = e_m1; /* e^{nu t}, e^{(nu-1) t} at t = k h */
    double s0 = 0.5, s1 = 0.5, s2 = 0.0;
    for (int kk = 1; kk < 2000; ++kk) {
        const double t = kk * h;
        const double w = exp(-2.0 * x * s * s);
        const double ipn = 1.0 / pn, ipm = 1.0 / pm;
        const double g0 = w * 0.5 * (pn + ipn);
        s0 += g0;
        s1 += w * 0.5 * (pm + ipm);
        const double g2 = w * t * 0.5 * (pn - ipn);
        s2 += g2;
        if (g0 < 1e-17 * s0 && fabs(g2) < 1e-17 * (fabs(s2) + s0) && 2.0 * x * s * q > nu + 1.0) break;
        const double s_next = s * chh + q * sh;
        q = q * chh + s * sh;
        s = s_next;
        pn *= e_nu;
        pm *= e_m1;
    }
    *k = h * s0;
    *km1 = h * s1;
    *dk = h * s2;
}

/* Derivatives of the Matern element M = con r^nu K_nu(r), r = d / beta > 0,
 * con = sigma2 / (2^(nu-1) Gamma(nu)), with respect to sigma2, beta and nu
 * (the math of core_dcmg_matern_dsigma_square / _dbeta / _dnu,
 * core_zcmg.c:315-488, with an exact nu derivative of K_nu instead of the
 * reference's 1e-9 forward difference, core_zcmg.c:228-235):
 *   dM/dsigma2 = M / sigma2
 *   dM/dbeta   = con r^(nu+1) K_{nu-1}(r) / beta
 *   dM/dnu     = M (log r - log 2 - psi(nu)) + con r^nu dK_nu/dnu
 * dlogcon = -(log 2 + psi(nu)) is passed in (one digamma per evaluation). */
XG_HD inline void xg_matern_grad(double r, double nu, double con, double sigma2, double beta, double dlogcon,
                                 double *m, double *d_sigma2, double *d_beta, double *d_nu)
{
    double ek, ekm1, edk;
    xg_knu_trap3(nu, r, &ek, &ekm1, &edk);
    const double f = exp(nu * log(r) - r); /* r^nu e^-r (the trapezoid sums carry e^r) */
    const double M = con * f * ek;
    *m = M;
    *d_sigma2 = M / sigma2;
    *d_beta = con * f * r * ekm1 / beta;
    *d_nu = M * (log(r) + dlogcon) + con * f * edk;
}

/* Half-integer orders in closed form: for nu = p + 1/2 the Matern element is
 * sigma^2 e^-r P_p(r) with P_0 = 1, P_1 = 1 + r, P_2 = 1 + r + r^2/3. */
XG_HD inline double xg_matern_half_integer(double r, double sigma2, int p)
{
    const double e = exp(-r);
    if (p == 0) return sigma2 * e;
    if (p == 1) return sigma2 * (1.0 + r) * e;
    return sigma2 * (1.0 + r + r * r * (1.0 / 3.0)) * e;
}

#endif
