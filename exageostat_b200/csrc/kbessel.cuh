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
   x >= 20 (nu <= 5): the asymptotic expansion
 *              K_nu(x) = sqrt(pi / (2x)) e^-x sum_k a_k(nu) / x^k   (DLMF 10.40.2),
 *            summed until the terms fall below 1e-17 of the sum: for
 *            0 <= nu <= 5 and x >= 20 at most 22 terms and a truncation
 *            error below 2e-16 relative (measured against mpmath), with one
 *            exponential where the trapezoidal rule takes one per node.
 *
 * The terms of Temme's series that depend on the order only (the 1/Gamma
 * values, pi mu / sin(pi mu), 2^mu) are computed once per order (XgTemme);
 * the covariance generators pass them in with the Matern parameters.  Each
 * branch runs a short loop; the reciprocals 1/k of the loops come from a
 * table in constant memory on the device.
 */
#ifndef EXAGEOSTAT_B200_KBESSEL_CUH
#define EXAGEOSTAT_B200_KBESSEL_CUH

#include <math.h>

#include "rgamma_taylor.cuh"
#include "xg_temme.h"

#ifndef XG_HD
#ifdef __CUDACC__
#define XG_HD __host__ __device__
#else
#define XG_HD
#endif
#endif

#define XG_PI 3.141592653589793
#define XG_EPS 2.220446049250313e-16

/* 1 / k for the series loops: on the device from a constant-memory table
 * (every lane of a converged warp reads the same entry), on the host by
 * division; both are the correctly rounded value. */
#ifdef __CUDACC__
static __constant__ double xg_inv_int_tab[64] = {1.0 / 1, 1.0 / 2, 1.0 / 3, 1.0 / 4, 1.0 / 5, 1.0 / 6, 1.0 / 7, 1.0 / 8, 1.0 / 9, 1.0 / 10, 1.0 / 11, 1.0 / 12, 1.0 / 13, 1.0 / 14, 1.0 / 15, 1.0 / 16, 1.0 / 17, 1.0 / 18, 1.0 / 19, 1.0 / 20, 1.0 / 21, 1.0 / 22, 1.0 / 23, 1.0 / 24, 1.0 / 25, 1.0 / 26, 1.0 / 27, 1.0 / 28, 1.0 / 29, 1.0 / 30, 1.0 / 31, 1.0 / 32, 1.0 / 33, 1.0 / 34, 1.0 / 35, 1.0 / 36, 1.0 / 37, 1.0 / 38, 1.0 / 39, 1.0 / 40, 1.0 / 41, 1.0 / 42, 1.0 / 43, 1.0 / 44, 1.0 / 45, 1.0 / 46, 1.0 / 47, 1.0 / 48, 1.0 / 49, 1.0 / 50, 1.0 / 51, 1.0 / 52, 1.0 / 53, 1.0 / 54, 1.0 / 55, 1.0 / 56, 1.0 / 57, 1.0 / 58, 1.0 / 59, 1.0 / 60, 1.0 / 61, 1.0 / 62, 1.0 / 63, 1.0 / 64};
#endif
XG_HD inline double xg_inv_int(int k)
{
#ifdef __CUDA_ARCH__
    return k <= 64 ? xg_inv_int_tab[k - 1] : 1.0 / k;
#else
    return 1.0 / k;
#endif
}


XG_HD inline XgTemme xg_temme_consts(double nu)
{
    XgTemme c;
    c.n = (int)(nu + 0.5);
    c.mu = nu - c.n;
    c.m2 = c.mu * c.mu;
    const double even = xg_rgamma_even(c.m2);
    const double odd = xg_rgamma_odd(c.m2);
    c.gamma1 = -odd;                     /* (1/G(1-mu) - 1/G(1+mu)) / (2 mu) */
    c.gamma2 = even;                     /* (1/G(1-mu) + 1/G(1+mu)) / 2 */
    c.grp = 1.0 / (even + c.mu * odd);   /* G(1+mu) */
    c.grm = 1.0 / (even - c.mu * odd);   /* G(1-mu) */
    const double pimu = XG_PI * c.mu;
    c.pimu_sin = (pimu == 0.0) ? 1.0 : pimu / sin(pimu);
    c.two_mu = pow(2.0, c.mu);
    return c;
}

/* Temme's series: K_mu(x) and K_{mu+1}(x), 0 < x <= 2; *pw = (2 / x)^mu.
 * One division per term: 1 / (k^2 - mu^2) also gives 1 / (k -+ mu). */
XG_HD inline void xg_k_temme(const XgTemme &c, double x, double *k_mu, double *k_mu1, double *pw)
{
    const double mu = c.mu, m2 = c.m2;
    const double half_x = 0.5 * x;
    const double ln_two_over_x = -log(half_x);
    const double sigma = mu * ln_two_over_x;
    const double e = exp(sigma), ie = 1.0 / e; /* (2/x)^mu and its inverse */
    const double shc = (sigma == 0.0) ? 1.0 : sinh(sigma) / sigma;
    double f = c.pimu_sin * (c.gamma1 * 0.5 * (e + ie) + c.gamma2 * shc * ln_two_over_x);
    double p = 0.5 * e * c.grp;
    double q = 0.5 * ie * c.grm;
    const double qx2 = half_x * half_x;
    double ck = 1.0, s0 = f, s1 = p;
    for (int k = 1; k < 200; ++k) {
        const double dk = (double)k;
        const double inv = 1.0 / (dk * dk - m2);
        f = (dk * f + p + q) * inv;
        ck *= qx2 * xg_inv_int(k);
        p *= (dk + mu) * inv;
        q *= (dk - mu) * inv;
        const double t0 = ck * f;
        s0 += t0;
        s1 += ck * (p - dk * f);
        if (fabs(t0) < 0.25 * XG_EPS * fabs(s0)) break;
    }
    *k_mu = s0;
    *k_mu1 = s1 / half_x;
    *pw = e;
}

/* K_nu(x) for nu >= 0, 0 < x <= 2, by Temme's series and forward recurrence
 * from the order's constants; also K_{nu-1}(x) (= K_{1-nu} by symmetry when
 * nu < 1) and (2 / x)^mu. */
XG_HD inline double xg_knu_small_c(const XgTemme &c, double x, double *k_num1, double *pw)
{
    double k0, k1;
    xg_k_temme(c, x, &k0, &k1, pw);
    const double tx = 2.0 / x;
    if (c.n == 0) {
        /* K_{nu-1} = K_{mu-1} = K_{mu+1} - 2 mu / x K_mu */
        if (k_num1) *k_num1 = k1 - c.mu * tx * k0;
        return k0;
    }
    for (int j = 1; j < c.n; ++j) {
        const double k2 = (c.mu + j) * tx * k1 + k0;
        k0 = k1;
        k1 = k2;
    }
    if (k_num1) *k_num1 = k0;
    return k1;
}

XG_HD inline double xg_knu_small(double nu, double x, double *k_num1)
{
    double pw;
    return xg_knu_small_c(xg_temme_consts(nu), x, k_num1, &pw);
}

/* sum_k a_k, a_0 = 1, a_k = a_{k-1} (4 nu^2 - (2k - 1)^2) / (8 k x): e^x K_nu(x)
 * sqrt(2 x / pi) for x >= XG_KNU_ASYM_X, 0 <= nu <= XG_KNU_ASYM_NU. */
#define XG_KNU_ASYM_X 20.0
#define XG_KNU_ASYM_NU 5.0
#define XG_SQRT_HALF_PI 1.2533141373155003
XG_HD inline double xg_knu_asym_sum(double nu, double x)
{
    const double m4 = 4.0 * nu * nu, i8x = 0.125 / x;
    double a = 1.0, s = 1.0;
    for (int k = 1; k <= 40; ++k) {
        const double t = 2.0 * k - 1.0;
        a *= (m4 - t * t) * i8x * xg_inv_int(k);
        s += a;
        if (fabs(a) < 1e-17 * fabs(s)) break;
    }
    return s;
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
    if (x >= XG_KNU_ASYM_X && nu <= XG_KNU_ASYM_NU)
        return XG_SQRT_HALF_PI / sqrt(x) * exp(-x) * xg_knu_asym_sum(nu, x);
    return xg_knu_scaled_trap(nu, x) * exp(-x);
}

/* Matern element con * r^nu * K_nu(r), r = d / beta > 0, for general nu
 * (core_zcmg.c:987), with the order's Temme constants tc.  For r <= 2,
 * r^nu = r^n 2^mu / (2/r)^mu reuses the series' own power; the large-r
 * branches fold r^nu e^-r into one exp so it neither overflows nor
 * underflows early. */
/* the three branches, also called one by one by the generators that group
 * elements by branch (xg_matern_branch) */
XG_HD inline double xg_matern_small_c(double r, double con, const XgTemme &tc) /* 0 < r <= 2 */
{
    double pw;
    const double k = xg_knu_small_c(tc, r, nullptr, &pw);
    double rn = 1.0;
    for (int j = 0; j < tc.n; ++j) rn *= r;
    return con * (rn * tc.two_mu / pw) * k;
}
XG_HD inline double xg_matern_asym(double r, double nu, double con) /* r >= 20, nu <= 5 */
{
    return con * XG_SQRT_HALF_PI * exp((nu - 0.5) * log(r) - r) * xg_knu_asym_sum(nu, r);
}
XG_HD inline double xg_matern_trap(double r, double nu, double con) /* r > 2 */
{
    return con * exp(nu * log(r) - r) * xg_knu_scaled_trap(nu, r);
}
/* branch of r > 0: 0 Temme (r <= 2), 1 and 2 the trapezoidal rule (r <= 6,
 * beyond: fewer nodes), 3 the asymptotic expansion */
XG_HD inline int xg_matern_branch(double r, double nu)
{
    if (r <= 2.0) return 0;
    if (r >= XG_KNU_ASYM_X && nu <= XG_KNU_ASYM_NU) return 3;
    return r <= 6.0 ? 1 : 2;
}

XG_HD inline double xg_matern_general_c(double r, double nu, double con, const XgTemme &tc)
{
    if (r <= 2.0) return xg_matern_small_c(r, con, tc);
    if (r >= XG_KNU_ASYM_X && nu <= XG_KNU_ASYM_NU) return xg_matern_asym(r, nu, con);
    return xg_matern_trap(r, nu, con);
}

XG_HD inline double xg_matern_general(double r, double nu, double con)
{
    return xg_matern_general_c(r, nu, con, xg_temme_consts(nu));
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

/* e^x K_nu(x), e^x K_{nu-1}(x) and e^x dK_nu/dnu(x) for x >= XG_KNU_ASYM_X,
 * 0 <= nu <= XG_KNU_ASYM_NU from the asymptotic expansion (DLMF 10.40.2) of
 * both orders and its term-by-term nu derivative: with c_k = (4 nu^2 -
 * (2k - 1)^2) / (8 k x), a_k = a_{k-1} c_k and a'_k = a'_{k-1} c_k + a_{k-1}
 * nu / (k x).  At most 30 terms; truncation below 2e-17 of K_nu for all
 * three (measured against mpmath, the derivative by mpmath's numerical
 * differentiation). */
XG_HD inline void xg_knu_asym3(double nu, double x, double *k, double *km1, double *dk)
{
    const double m4 = 4.0 * nu * nu, m4b = 4.0 * (nu - 1.0) * (nu - 1.0), i8x = 0.125 / x, ix = 1.0 / x;
    double a = 1.0, b = 1.0, ad = 0.0, s = 1.0, sb = 1.0, sd = 0.0;
    for (int kk = 1; kk <= 40; ++kk) {
        const double t = 2.0 * kk - 1.0, ik = xg_inv_int(kk);
        const double c = (m4 - t * t) * i8x * ik;
        ad = ad * c + a * (nu * ix * ik);
        a *= c;
        b *= (m4b - t * t) * i8x * ik;
        s += a;
        sb += b;
        sd += ad;
        if (fabs(a) < 1e-17 * fabs(s) && fabs(b) < 1e-17 * fabs(sb) && fabs(ad) < 1e-17 * (fabs(sd) + fabs(s)))
            break;
    }
    const double f = XG_SQRT_HALF_PI / sqrt(x);
    *k = f * s;
    *km1 = f * sb;
    *dk = f * sd;
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
    if (r >= XG_KNU_ASYM_X && nu <= XG_KNU_ASYM_NU)
        xg_knu_asym3(nu, r, &ek, &ekm1, &edk);
    else
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
