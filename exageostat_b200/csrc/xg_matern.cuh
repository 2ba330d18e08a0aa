/*
 * Location distance and the Matern covariance element, shared by every kernel
 * that generates covariance entries (core_dcmg, exageostat_exact/cpu_core/
 * compute/core_zcmg.c:963-994; core_dcmg_nuggets, core_zcmg_nuggets.c:107-156).
 */
#ifndef EXAGEOSTAT_B200_MATERN_CUH
#define EXAGEOSTAT_B200_MATERN_CUH

#include <math.h>

#include "kbessel.cuh"
#include "xg_kernels.h"

/* deg * PI / 180 in the reference's order of operations (core_zcmg.c:30-32) */
__device__ inline double xg_deg2rad(double d) { return d * XG_PI / 180.0; }

/* Distance between (x1, y1) [row location] and (x2, y2) [column location].
 * Euclidean: sqrt(pow(x2 - x1, 2) + pow(y2 - y1, 2)) as core_zcmg.c:84, with
 * explicit round-to-nearest products and sum so no FMA contraction changes
 * the rounding.  Great circle (dm = "gc"): haversine in km on (lat, lon) in
 * degrees, as distanceEarth (core_zcmg.c:51-60). */
__device__ inline double xg_distance(double x1, double y1, double x2, double y2, int metric)
{
    if (metric == 1) {
        const double lat1 = xg_deg2rad(x1), lon1 = xg_deg2rad(y1);
        const double lat2 = xg_deg2rad(x2), lon2 = xg_deg2rad(y2);
        const double u = sin((lat2 - lat1) / 2), v = sin((lon2 - lon1) / 2);
        return 2.0 * 6371.0 * asin(sqrt(u * u + cos(lat1) * cos(lat2) * v * v));
    }
    const double dx = x2 - x1, dy = y2 - y1;
    return sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
}

/* Covariance element at distance d: sigma^2 (+ tau^2 for the nugget kernel)
 * on the exact zero of d / beta (core_zcmg.c:983-984), else the Matern value. */
__device__ inline double xg_matern_value(double d, const XgMaternParams &p)
{
    const double r = d / p.beta;
    if (r == 0.0) return p.sigma2 + p.nugget;
    if (p.half_integer >= 0) return xg_matern_half_integer(r, p.sigma2, p.half_integer);
    return xg_matern_general_c(r, p.nu, p.con, p.tm);
}

/* Bivariate Matern element between variable a of one location and variable
 * b of another.  Parsimonious (core_dcmg_bivariate_parsimonious,
 * core_zcmg.c:1628-1726): Matern(sigma_a^2, beta, nu_a) on the diagonal
 * blocks, rho sqrt(sigma_1^2 sigma_2^2) Matern(1, beta, nu12) across.
 * Flexible (core_dcmg_bivariate_flexible, core_zcmg.c:1514-1580): a scale,
 * smoothness and constant per component.  The values at d / beta == 0 are the
 * reference's (sigma2, sigma2b, cross0 as the host set them). */
__device__ inline double xg_matern_value_biv(double d, const XgMaternParams &p, int a, int b)
{
    const double r = d / p.beta;
    if (r == 0.0) return a != b ? p.cross0 : (a == 0 ? p.sigma2 : p.sigma2b);
    if (a != b) return xg_matern_general(d / p.beta12, p.nu12, p.con12);
    if (a == 0) return xg_matern_general(r, p.nu, p.con);
    return xg_matern_general(d / p.beta2, p.nu2, p.con2);
}

#endif
