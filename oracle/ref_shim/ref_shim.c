/*
 * Link-time stand-ins for the reference functions compiled into
 * oracle/_ref/libexageostat_ref.so (test infrastructure only).
 *
 *  - gsl_sf_bessel_Knu: GSL is absent here.  The reference's Matern kernels
 *    (core_zcmg.c, core_zcmg_nuggets.c) call it for K_nu; this stand-in
 *    returns the oracle's K_nu (ora_bessel_knu in oracle/oracle.c: Temme's
 *    series for x <= 2, Steed's continued fraction above, pinned to mpmath
 *    besselk to 1e-14 relative by tests/golden/kv_mpmath.json).  Everything
 *    else in those kernels -- the distance, the exact zero-distance branch,
 *    the 2^(nu-1) Gamma(nu) constant, pow -- is the reference's own code.
 *  - results: the global that misc/include/MLE_misc.h declares extern (the
 *    reference's drivers define it).
 *  - MLE_get_zobs (src/compute/MLE.c:420-430 copies the device vector z
 *    out): here it copies the vector registered by ref_pick_random_points,
 *    the wrapper the tests call around the reference's pick_random_points.
 *  - nlopt_set_*: referenced by functions of misc/compute/MLE_misc.c that
 *    the tests never call; they abort.
 */
#include <stdio.h>
#include <stdlib.h>

#include "MLE_misc.h"

double ora_bessel_knu(double nu, double x);

double gsl_sf_bessel_Knu(const double nu, const double x) { return ora_bessel_knu(nu, x); }

output results;

static void ref_shim_unavailable(const char *name)
{
    fprintf(stderr, "oracle/_ref: %s is not part of the compiled reference subset\n", name);
    abort();
}

static const double *g_ref_z = NULL;
static int g_ref_n = 0;

void MLE_get_zobs(MLE_data *data, double *z, int n)
{
    (void)data;
    if (!g_ref_z || n > g_ref_n) ref_shim_unavailable("MLE_get_zobs without a registered z");
    for (int i = 0; i < n; ++i) z[i] = g_ref_z[i];
}

/* The reference's pick_random_points on locations (x, y) and values z of N
 * points: the libc rand() stream is used as it stands (the caller replays
 * it).  Outputs: the nmiss held-out points (xm, ym, zact) and the N - nmiss
 * observed ones (xo, yo, zobs), each set Morton-sorted as the reference
 * leaves them in data->lmiss / data->lobs. */
void ref_pick_random_points(int N, const double *x, const double *y, const double *z, int nmiss, double *xm,
                            double *ym, double *zact, double *xo, double *yo, double *zobs)
{
    MLE_data data = {0};
    double *lx = malloc(sizeof(double) * N), *ly = malloc(sizeof(double) * N);
    for (int i = 0; i < N; ++i) {
        lx[i] = x[i];
        ly[i] = y[i];
    }
    data.l1.x = lx;
    data.l1.y = ly;
    g_ref_z = z;
    g_ref_n = N;
    const int nobs = N - nmiss;
    pick_random_points(&data, zobs, zact, nmiss, nobs, N);
    g_ref_z = NULL;
    for (int i = 0; i < nmiss; ++i) {
        xm[i] = data.lmiss.x[i];
        ym[i] = data.lmiss.y[i];
    }
    for (int i = 0; i < nobs; ++i) {
        xo[i] = data.lobs.x[i];
        yo[i] = data.lobs.y[i];
    }
    free(data.lmiss.x); /* the reference allocates one array and splits it */
    free(data.lmiss.y);
    free(lx);
    free(ly);
}

int nlopt_set_ftol_abs(nlopt_opt opt, double tol)
{
    (void)opt, (void)tol;
    ref_shim_unavailable("nlopt_set_ftol_abs");
    return 0;
}

int nlopt_set_lower_bounds(nlopt_opt opt, const double *lb)
{
    (void)opt, (void)lb;
    ref_shim_unavailable("nlopt_set_lower_bounds");
    return 0;
}

int nlopt_set_upper_bounds(nlopt_opt opt, const double *ub)
{
    (void)opt, (void)ub;
    ref_shim_unavailable("nlopt_set_upper_bounds");
    return 0;
}
