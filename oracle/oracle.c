/*
 * CPU ORACLE for the exact univariate Matern maximum-likelihood path.
 *
 * This file is TEST INFRASTRUCTURE.  It is a plain-C restatement of the
 * reference (ExaGeoStat 1.2, exageostat_exact) CPU algorithm and is used only
 * by the tests, by the smoke check and by the timed CPU-baseline leg of the
 * benchmark.  The product library never links, loads or calls it.
 *
 * What it restates (paths are inside the reference project):
 *   - GenerateXYLoc / uniform_distribution / zsort_locations and the Morton
 *     helpers              misc/compute/MLE_misc.c:225-319, 753-792
 *   - shuffle, shuffle2, pick_random_points, pick_random_points2,
 *     locations_obs_zsort_inplace + radix sort
 *                          misc/compute/MLE_misc.c:405-534, 1238-1259, 1700-1741
 *   - core_dcmg (Matern) and core_dcmg_nuggets
 *                          exageostat_exact/cpu_core/compute/core_zcmg.c:71-92, 963-994
 *                          exageostat_exact/cpu_core/compute/core_zcmg_nuggets.c:107-156
 *   - core_dmdet           exageostat_exact/cpu_core/compute/core_zmdet.c:50-59
 *   - EXAGEOSTAT_MLE_dzvg_Tile (Z = L e)   exageostat_exact/src/compute/MLE_dexact.c:25-148
 *   - EXAGEOSTAT_dmle_Tile (log-likelihood) exageostat_exact/src/compute/MLE_dexact.c:231-489
 *   - core_dcmg_bivariate_parsimonious
 *                          exageostat_exact/cpu_core/compute/core_zcmg.c:1628-1726
 *   - core_dcmg_matern_dsigma_square / _dbeta / _dnu and psi
 *                          exageostat_exact/cpu_core/compute/core_zcmg.c:189-235, 315-488
 *   - EXAGEOSTAT_dmle_Predict_Tile + CORE_dmse_starpu
 *                          exageostat_exact/src/compute/MLE_dexact.c:688-874,
 *                          exageostat_exact/runtime/starpu/codelets/codelet_zmse.c:22-38
 *
 * Third-party arithmetic the reference takes from libraries that are not in
 * the reference tree:
 *   - gsl_sf_bessel_Knu (GSL 2.6).  Restated from the published method GSL
 *     documents: Temme's series (N. M. Temme, J. Comput. Phys. 19 (1975)
 *     324-337) for x < 2, Steed's continued fraction CF2 with Temme's
 *     normalisation (I. J. Thompson & A. R. Barnett, J. Comput. Phys. 64
 *     (1986) 490-509) for x >= 2, then forward recurrence in the order.
 *     Checked against mpmath besselk (tests/golden/kv_mpmath.json).
 *   - The Cholesky factorisation is the tile algorithm of the reference's
 *     CHAMELEON_dpotrf_Tile (MLE_dexact.c:372; its step structure is the one
 *     chameleon_psdpotrf spells out with an infinite band, psdportf.c:85-186):
 *     per block column k, POTRF of the diagonal block, TRSM of the blocks
 *     below it and the SYRK/GEMM update of the trailing matrix, with the
 *     block operations (dpotrf, dtrsm, dsyrk, dgemm) called from the OpenBLAS
 *     0.3.30 (ILP64, "scipy_" symbol prefix) bundled with numpy.  OpenBLAS's
 *     own one-call dpotrf is not used: it segfaults at N = 40 000 here.
 *   - dtrsv / dtrmv / dgemv / dlarnv: called from the same OpenBLAS, as the
 *     reference calls MKL/Chameleon for the same operations.
 *
 * Parity of the reference's GSL values themselves is unpinned (GSL is absent
 * here); this oracle is pinned to mpmath for K_nu and to the reference's own
 * formulas for everything else.
 */
#define _GNU_SOURCE
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "rgamma_taylor.h"

/* ---- OpenBLAS ILP64 entry points (numpy.libs/libscipy_openblas64_*.so) ---- */
typedef int64_t blasint64;
enum { ORA_COL_MAJOR = 102, ORA_NOTRANS = 111, ORA_TRANS = 112, ORA_UPPER = 121,
       ORA_LOWER = 122, ORA_NONUNIT = 131 };
extern blasint64 scipy_LAPACKE_dpotrf64_(int layout, char uplo, blasint64 n, double *a, blasint64 lda);
extern blasint64 scipy_LAPACKE_dlarnv64_(blasint64 idist, blasint64 *iseed, blasint64 n, double *x);
extern blasint64 scipy_LAPACKE_dposv64_(int layout, char uplo, blasint64 n, blasint64 nrhs, double *a,
                                       blasint64 lda, double *b, blasint64 ldb);
extern void scipy_cblas_dtrsv64_(int order, int uplo, int trans, int diag, blasint64 n, const double *a,
                                 blasint64 lda, double *x, blasint64 incx);
extern void scipy_cblas_dtrmv64_(int order, int uplo, int trans, int diag, blasint64 n, const double *a,
                                 blasint64 lda, double *x, blasint64 incx);
extern void scipy_cblas_dgemv64_(int order, int trans, blasint64 m, blasint64 n, double alpha, const double *a,
                                 blasint64 lda, const double *x, blasint64 incx, double beta, double *y,
                                 blasint64 incy);
extern double scipy_cblas_ddot64_(blasint64 n, const double *x, blasint64 incx, const double *y, blasint64 incy);
extern void scipy_openblas_set_num_threads64_(int n);
extern void scipy_cblas_dtrsm64_(int order, int side, int uplo, int trans, int diag, blasint64 m, blasint64 n,
                                 double alpha, const double *a, blasint64 lda, double *b, blasint64 ldb);
extern void scipy_cblas_dsyrk64_(int order, int uplo, int trans, blasint64 n, blasint64 k, double alpha,
                                 const double *a, blasint64 lda, double beta, double *c, blasint64 ldc);
extern void scipy_cblas_dgemm64_(int order, int transa, int transb, blasint64 m, blasint64 n, blasint64 k,
                                 double alpha, const double *a, blasint64 lda, const double *b, blasint64 ldb,
                                 double beta, double *c, blasint64 ldc);
enum { ORA_RIGHT = 142 };

/* Block size of the tile Cholesky (the reference's default dense tile size is
 * of this order; the factor does not depend on it beyond rounding). */
#define ORA_NB 512

/* Lower Cholesky factor in place of the column-major N x N array C (leading
 * dimension N), by block columns of ORA_NB (the tile algorithm):
 *   C_kk = chol(C_kk); C_ik = C_ik C_kk^-T (i > k);
 *   C_jj -= C_jk C_jk^T, C_ij -= C_ik C_jk^T (i > j > k).
 * Returns 0, or the 1-based column of the first non-positive pivot. */
static blasint64 ora_potrf_tiles(blasint64 N, double *C)
{
    for (blasint64 k = 0; k < N; k += ORA_NB) {
        const blasint64 kb = N - k < ORA_NB ? N - k : ORA_NB;
        double *Ckk = C + k + k * N;
        blasint64 info = scipy_LAPACKE_dpotrf64_(ORA_COL_MAJOR, 'L', kb, Ckk, N);
        if (info != 0) return info > 0 ? k + info : info;
        const blasint64 m = N - k - kb;
        if (m == 0) break;
        double *Cik = Ckk + kb;
        scipy_cblas_dtrsm64_(ORA_COL_MAJOR, ORA_RIGHT, ORA_LOWER, ORA_TRANS, ORA_NONUNIT, m, kb, 1.0, Ckk, N, Cik,
                             N);
        /* trailing update block column by block column: SYRK on the diagonal
         * block, GEMM on the blocks below it (one dsyrk over the whole
         * trailing matrix segfaults inside OpenBLAS at N = 40 000) */
        for (blasint64 j = k + kb; j < N; j += ORA_NB) {
            const blasint64 jb = N - j < ORA_NB ? N - j : ORA_NB;
            const double *Cjk = C + j + k * N;
            scipy_cblas_dsyrk64_(ORA_COL_MAJOR, ORA_LOWER, ORA_NOTRANS, jb, kb, -1.0, Cjk, N, 1.0, C + j + j * N, N);
            const blasint64 mb = N - j - jb;
            if (mb > 0)
                scipy_cblas_dgemm64_(ORA_COL_MAJOR, ORA_NOTRANS, ORA_TRANS, mb, jb, kb, -1.0, Cjk + jb, N, Cjk, N,
                                     1.0, C + (j + jb) + j * N, N);
        }
    }
    return 0;
}

#define ORA_PI 3.141592653589793 /* MLE_misc.h:64 */

static double ora_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

void ora_set_threads(int n)
{
    scipy_openblas_set_num_threads64_(n);
#ifdef _OPENMP
    omp_set_num_threads(n);
#endif
}

int ora_get_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ========================================================================== */
/* Modified Bessel function of the second kind K_nu(x), nu >= 0, x > 0.       */
/* ========================================================================== */

/* Gamma1(mu), Gamma2(mu) of Temme's series and 1/Gamma(1+mu), 1/Gamma(1-mu),
 * from the Taylor series 1/Gamma(z) = sum_k c_k z^k split into even/odd parts. */
static void ora_temme_gammas(double mu, double *g1, double *g2, double *rg_p, double *rg_m)
{
    const double m2 = mu * mu;
    double even = 0.0, odd = 0.0; /* even = sum_j c_{2j+1} m2^j, odd = sum_j c_{2j+2} m2^j */
    for (int j = (ORA_RGAMMA_C_COUNT - 2) / 2; j >= 0; --j) {
        even = even * m2 + ORA_RGAMMA_C[2 * j + 1];
        odd = odd * m2 + ((2 * j + 2 < ORA_RGAMMA_C_COUNT) ? ORA_RGAMMA_C[2 * j + 2] : 0.0);
    }
    *g1 = -odd;
    *g2 = even;
    *rg_p = even + mu * odd;
    *rg_m = even - mu * odd;
}

/* Temme's series: K_mu(x), K_{mu+1}(x) for |mu| <= 1/2, 0 < x <= 2 (unscaled). */
static void ora_k_temme(double mu, double x, double *k_mu, double *k_mu1)
{
    double g1, g2, rgp, rgm;
    ora_temme_gammas(mu, &g1, &g2, &rgp, &rgm);
    const double half_x = 0.5 * x;
    const double ln_2_over_x = -log(half_x);
    const double sigma = mu * ln_2_over_x;
    const double pimu = ORA_PI * mu;
    const double pimu_over_sin = (fabs(pimu) < 1e-300) ? 1.0 : pimu / sin(pimu);
    const double sinh_sigma_over_sigma = (fabs(sigma) < 1e-300) ? 1.0 : sinh(sigma) / sigma;
    const double two_over_x_pow_mu = exp(sigma);
    double f = pimu_over_sin * (g1 * cosh(sigma) + g2 * sinh_sigma_over_sigma * ln_2_over_x);
    double p = 0.5 * two_over_x_pow_mu / rgp;   /* (x/2)^-mu Gamma(1+mu) / 2 */
    double q = 0.5 / (two_over_x_pow_mu * rgm); /* (x/2)^+mu Gamma(1-mu) / 2 */
    const double quarter_x2 = half_x * half_x;
    double ck = 1.0;
    double sum0 = f, sum1 = p;
    for (int k = 1; k < 1000; ++k) {
        const double dk = (double)k;
        f = (dk * f + p + q) / (dk * dk - mu * mu);
        ck *= quarter_x2 / dk;
        p /= (dk - mu);
        q /= (dk + mu);
        const double t0 = ck * f;
        sum0 += t0;
        sum1 += ck * (p - dk * f);
        if (fabs(t0) < 0.5 * DBL_EPSILON * fabs(sum0)) break;
    }
    *k_mu = sum0;
    *k_mu1 = sum1 / half_x;
}

/* Steed's CF2 with Temme's normalisation: e^x K_mu(x), e^x K_{mu+1}(x) for
 * |mu| <= 1/2, x >= 2. */
static void ora_k_cf2_scaled(double mu, double x, double *k_mu, double *k_mu1)
{
    const double a1 = 0.25 - mu * mu;
    double bi = 2.0 * (1.0 + x);
    double di = 1.0 / bi;
    double delta_h = di, h = di;
    double q_prev = 0.0, q_cur = 1.0;
    double ai = -a1, ci = a1, qsum = a1;
    double s = 1.0 + qsum * delta_h;
    for (int i = 2; i < 100000; ++i) {
        ai -= 2.0 * (i - 1);
        ci = -ai * ci / i;
        const double q_next = (q_prev - bi * q_cur) / ai;
        q_prev = q_cur;
        q_cur = q_next;
        qsum += ci * q_next;
        bi += 2.0;
        di = 1.0 / (bi + ai * di);
        delta_h = (bi * di - 1.0) * delta_h;
        h += delta_h;
        const double ds = qsum * delta_h;
        s += ds;
        if (fabs(ds) < 0.5 * DBL_EPSILON * fabs(s)) break;
    }
    h *= a1;
    *k_mu = sqrt(ORA_PI / (2.0 * x)) / s;
    *k_mu1 = *k_mu * (mu + x + 0.5 - h) / x;
}

double ora_bessel_knu(double nu, double x)
{
    if (!(x > 0.0) || nu < 0.0) return NAN;
    const int n = (int)(nu + 0.5);
    const double mu = nu - n; /* in [-1/2, 1/2) */
    double k0, k1;
    double scale = 1.0;
    if (x < 2.0) {
        ora_k_temme(mu, x, &k0, &k1);
    } else {
        ora_k_cf2_scaled(mu, x, &k0, &k1);
        scale = exp(-x);
    }
    /* forward recurrence K_{m+1} = K_{m-1} + 2 m / x K_m, m = mu+1 .. nu-1 */
    for (int j = 1; j < n; ++j) {
        const double k2 = 2.0 * (mu + j) / x * k1 + k0;
        k0 = k1;
        k1 = k2;
    }
    return scale * (n == 0 ? k0 : k1);
}

/* ========================================================================== */
/* Synthetic locations: GenerateXYLoc (MLE_misc.c:763-792)                    */
/* ========================================================================== */

/* uniform_distribution, MLE_misc.c:753-761 */
static double ora_uniform(double lo, double hi)
{
    double r = (double)rand() / (double)(1.0 + RAND_MAX);
    double range = hi - lo;
    return r * range + lo;
}

/* Morton helpers, MLE_misc.c:225-296 */
static uint32_t ora_spread_bits(uint32_t v)
{
    v &= 0x0000ffffu;
    v = (v ^ (v << 8)) & 0x00ff00ffu;
    v = (v ^ (v << 4)) & 0x0f0f0f0fu;
    v = (v ^ (v << 2)) & 0x33333333u;
    v = (v ^ (v << 1)) & 0x55555555u;
    return v;
}

static uint32_t ora_gather_bits(uint32_t v)
{
    v &= 0x55555555u;
    v = (v ^ (v >> 1)) & 0x33333333u;
    v = (v ^ (v >> 2)) & 0x0f0f0f0fu;
    v = (v ^ (v >> 4)) & 0x00ff00ffu;
    v = (v ^ (v >> 8)) & 0x0000ffffu;
    return v;
}

static int ora_cmp_u32(const void *a, const void *b)
{
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}

/* zsort_locations, MLE_misc.c:297-319: Morton sort + uint16 quantisation. */
static void ora_zsort_locations(int n, double *x, double *y)
{
    uint32_t *code = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) {
        uint16_t qx = (uint16_t)(x[i] * (double)UINT16_MAX + .5);
        uint16_t qy = (uint16_t)(y[i] * (double)UINT16_MAX + .5);
        code[i] = (ora_spread_bits(qy) << 1) + ora_spread_bits(qx);
    }
    qsort(code, (size_t)n, sizeof(uint32_t), ora_cmp_u32);
    for (int i = 0; i < n; ++i) {
        uint16_t qx = (uint16_t)ora_gather_bits(code[i]);
        uint16_t qy = (uint16_t)ora_gather_bits(code[i] >> 1);
        x[i] = (double)qx / (double)UINT16_MAX;
        y[i] = (double)qy / (double)UINT16_MAX;
    }
    free(code);
}

/* GenerateXYLoc(n, seed): seeds libc rand() with `seed`, jitters a
 * ceil(sqrt(n))^2 grid (row-major over x then y, truncated at n) and Morton
 * sorts.  Leaves the libc rand() stream where the reference leaves it. */
void ora_generate_xy_loc(int n, int seed, double *x, double *y)
{
    srand((unsigned)seed);
    int sqrtn = (int)ceil(sqrt((double)n));
    int index = 0;
    for (int i = 0; i < sqrtn && index < n; ++i)
        for (int j = 0; j < sqrtn && index < n; ++j) {
            x[index] = ((i + 1) - 0.5 + ora_uniform(-0.4, 0.4)) / sqrtn;
            y[index] = ((j + 1) - 0.5 + ora_uniform(-0.4, 0.4)) / sqrtn;
            ++index;
        }
    ora_zsort_locations(n, x, y);
}

/* Replays the libc rand() stream: srand(seed) then `skip` draws. */
void ora_rand_replay(int seed, long skip)
{
    srand((unsigned)seed);
    for (long i = 0; i < skip; ++i) (void)rand();
}

/* ========================================================================== */
/* Hold-out selection: shuffle + pick_random_points (MLE_misc.c)             */
/* ========================================================================== */

/* radix_sort_recursive, MLE_misc.c:405-441 */
static void ora_radix_rec(const uint32_t *data, int count, int ndim, int *order, int *tmp, int sdim, int sbit,
                          int lo, int hi)
{
    int lo_last = lo, hi_last = hi;
    const uint32_t *sdata = data + (size_t)sdim * count;
    uint32_t check = 1u << sbit;
    for (int i = lo; i <= hi; ++i) {
        if ((sdata[order[i]] & check) == 0)
            tmp[lo_last++] = order[i];
        else
            tmp[hi_last--] = order[i];
    }
    for (int i = lo; i <= hi; ++i) order[i] = tmp[i];
    if (sdim > 0) {
        if (lo_last - lo > 1) ora_radix_rec(data, count, ndim, order, tmp, sdim - 1, sbit, lo, lo_last - 1);
        if (hi - hi_last > 1) ora_radix_rec(data, count, ndim, order, tmp, sdim - 1, sbit, hi_last + 1, hi);
    } else if (sbit > 0) {
        if (lo_last - lo > 1) ora_radix_rec(data, count, ndim, order, tmp, ndim - 1, sbit - 1, lo, lo_last - 1);
        if (hi - hi_last > 1) ora_radix_rec(data, count, ndim, order, tmp, ndim - 1, sbit - 1, hi_last + 1, hi);
    }
}

/* locations_obs_zsort_inplace, MLE_misc.c:453-534 */
int ora_locations_obs_zsort_inplace(int n, double *x, double *y, double *z)
{
    const int ndim = 2;
    if (n <= 0) return 0;
    double *point = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        point[i] = x[i];
        point[i + n] = y[i];
    }
    double minmax[4];
    for (int d = 0; d < ndim; ++d) {
        const double *p = point + (size_t)d * n;
        minmax[d] = p[0];
        minmax[d + ndim] = minmax[d];
        for (int j = 1; j < n; ++j) {
            if (minmax[d] > p[j])
                minmax[d] = p[j];
            else if (minmax[d + ndim] < p[j])
                minmax[d + ndim] = p[j];
        }
    }
    uint32_t *up = (uint32_t *)malloc(sizeof(uint32_t) * 2 * (size_t)n);
    for (int d = 0; d < ndim; ++d) {
        const double mn = minmax[d], range = minmax[d + ndim] - mn;
        for (int j = 0; j < n; ++j) up[(size_t)d * n + j] = (uint32_t)((point[(size_t)d * n + j] - mn) / range * UINT32_MAX);
    }
    int *order = (int *)malloc(sizeof(int) * (size_t)n);
    int *tmp = (int *)malloc(sizeof(int) * (size_t)n);
    for (int j = 0; j < n; ++j) order[j] = j;
    ora_radix_rec(up, n, ndim, order, tmp, ndim - 1, 31, 0, n - 1);
    double *nz = (double *)malloc(sizeof(double) * (size_t)n);
    for (int j = 0; j < n; ++j) {
        x[j] = point[order[j]];
        y[j] = point[(size_t)n + order[j]];
        nz[j] = z[order[j]];
    }
    memcpy(z, nz, sizeof(double) * (size_t)n);
    free(nz);
    free(tmp);
    free(order);
    free(up);
    free(point);
    return 0;
}

/* shuffle (MLE_misc.c:1238-1259) + pick_random_points (MLE_misc.c:1700-1741).
 * Continues the current libc rand() stream.  Outputs: the first nZmiss
 * shuffled points are the missing set, the rest the observed set; each set
 * is then Morton re-sorted with its values. */
void ora_pick_random_points(int N, const double *x, const double *y, const double *z, int nZmiss,
                            double *xmiss, double *ymiss, double *zactual, double *xobs, double *yobs, double *zobs)
{
    double *Z = (double *)malloc(sizeof(double) * (size_t)N);
    double *lx = (double *)malloc(sizeof(double) * (size_t)N);
    double *ly = (double *)malloc(sizeof(double) * (size_t)N);
    memcpy(Z, z, sizeof(double) * (size_t)N);
    memcpy(lx, x, sizeof(double) * (size_t)N);
    memcpy(ly, y, sizeof(double) * (size_t)N);
    size_t n = (size_t)N;
    if (n > 1) {
        for (size_t i = 0; i < n - 1; ++i) {
            size_t j = i + (size_t)rand() / (RAND_MAX / (n - i) + 1);
            double t = Z[j]; Z[j] = Z[i]; Z[i] = t;
            t = lx[j]; lx[j] = lx[i]; lx[i] = t;
            t = ly[j]; ly[j] = ly[i]; ly[i] = t;
        }
    }
    const int nZobs = N - nZmiss;
    for (int i = 0; i < nZobs; ++i) {
        zobs[i] = Z[nZmiss + i];
        xobs[i] = lx[nZmiss + i];
        yobs[i] = ly[nZmiss + i];
    }
    for (int i = 0; i < nZmiss; ++i) {
        zactual[i] = Z[i];
        xmiss[i] = lx[i];
        ymiss[i] = ly[i];
    }
    ora_locations_obs_zsort_inplace(nZobs, xobs, yobs, zobs);
    ora_locations_obs_zsort_inplace(nZmiss, xmiss, ymiss, zactual);
    free(ly);
    free(lx);
    free(Z);
}

/* pick_random_points2 + shuffle2 (MLE_misc.c:1261-1285, 1744-1810): the
 * bivariate hold-out over nloc locations, z interleaved (2 nloc values); the
 * first nZmiss shuffled locations are missing, outputs interleaved again. */
void ora_pick_random_points2(int nloc, const double *x, const double *y, const double *z, int nZmiss,
                             double *xmiss, double *ymiss, double *zactual, double *xobs, double *yobs, double *zobs)
{
    double *Z1 = (double *)malloc(sizeof(double) * (size_t)nloc);
    double *Z2 = (double *)malloc(sizeof(double) * (size_t)nloc);
    double *lx = (double *)malloc(sizeof(double) * (size_t)nloc);
    double *ly = (double *)malloc(sizeof(double) * (size_t)nloc);
    for (int i = 0; i < nloc; ++i) {
        Z1[i] = z[2 * (size_t)i];
        Z2[i] = z[2 * (size_t)i + 1];
        lx[i] = x[i];
        ly[i] = y[i];
    }
    size_t n = (size_t)nloc;
    if (n > 1) {
        for (size_t i = 0; i < n - 1; ++i) {
            size_t j = i + (size_t)rand() / (RAND_MAX / (n - i) + 1);
            double t = Z1[j]; Z1[j] = Z1[i]; Z1[i] = t;
            t = Z2[j]; Z2[j] = Z2[i]; Z2[i] = t;
            t = lx[j]; lx[j] = lx[i]; lx[i] = t;
            t = ly[j]; ly[j] = ly[i]; ly[i] = t;
        }
    }
    const int nZobs = nloc - nZmiss;
    for (int i = 0; i < nZmiss; ++i) {
        zactual[2 * i] = Z1[i];
        zactual[2 * i + 1] = Z2[i];
        xmiss[i] = lx[i];
        ymiss[i] = ly[i];
    }
    for (int i = 0; i < nZobs; ++i) {
        zobs[2 * i] = Z1[nZmiss + i];
        zobs[2 * i + 1] = Z2[nZmiss + i];
        xobs[i] = lx[nZmiss + i];
        yobs[i] = ly[nZmiss + i];
    }
    free(ly);
    free(lx);
    free(Z2);
    free(Z1);
}

/* ========================================================================== */
/* Covariance generation: core_dcmg / core_dcmg_nuggets                       */
/* ========================================================================== */

/* Distance metric of the generators: 0 Euclidean (core_zcmg.c:84), 1 great
 * circle (distanceEarth, core_zcmg.c:51-60: haversine in km on (lat, lon) in
 * degrees, deg2rad :30-32, earthRadiusKm MLE_misc.h:68).  Set with
 * ora_set_metric; not thread-safe, like the reference's own globals. */
static int ora_metric = 0;

void ora_set_metric(int metric) { ora_metric = metric; }

static double ora_deg2rad(double deg) { return (deg * 3.141592653589793 / 180); }

static inline double ora_distance(double x1, double y1, double x2, double y2)
{
    if (ora_metric == 1) {
        const double lat1r = ora_deg2rad(x1), lon1r = ora_deg2rad(y1);
        const double lat2r = ora_deg2rad(x2), lon2r = ora_deg2rad(y2);
        const double u = sin((lat2r - lat1r) / 2), v = sin((lon2r - lon1r) / 2);
        return 2.0 * 6371.0 * asin(sqrt(u * u + cos(lat1r) * cos(lat2r) * v * v));
    }
    return sqrt(pow(x2 - x1, 2) + pow(y2 - y1, 2));
}

/* One Matern element (core_zcmg.c:975-990): distance with pow(.,2) and sqrt,
 * an exact compare with zero, then con * expr^nu * K_nu(expr). kernel 1 adds
 * the nugget theta[3] on the zero-distance branch (core_zcmg_nuggets.c:131). */
static inline double ora_matern_elem(double x1, double y1, double x2, double y2, const double *theta, double con,
                                     int kernel)
{
    double expr = ora_distance(x1, y1, x2, y2) / theta[1];
    if (expr == 0) return kernel == 1 ? theta[0] + theta[3] : theta[0];
    return con * pow(expr, theta[2]) * ora_bessel_knu(theta[2], expr);
}

static double ora_matern_con(const double *theta)
{
    double con = pow(2, (theta[2] - 1)) * tgamma(theta[2]);
    con = 1.0 / con;
    return theta[0] * con;
}

/* Bivariate Matern kernels, rows and columns interleaving the two variables.
 * Per component (0: variable 1, 1: variable 2, 2: the cross covariance) the
 * constant con, smoothness nu, scale and the value at zero distance.
 *   kernel 2, parsimonious, theta = (sigma_1^2, sigma_2^2, beta, nu_1, nu_2,
 *     rho): core_dcmg_bivariate_parsimonious (core_zcmg.c:1637-1651), one
 *     scale beta for all three;
 *   kernel 3, flexible, theta = (a_1, a_2, ., ., nu_1, nu_2, ., ., ., ., .):
 *     core_dcmg_bivariate_flexible (core_zcmg.c:1524-1556), a scale per
 *     component.  At zero distance the reference stores theta[0], theta[1] and
 *     rho (:1565-1568) -- the scales, not the variances sigma_11, sigma_22 that
 *     the Matern terms tend to -- and this restatement keeps that. */
typedef struct {
    double con[3], nu[3], scale[3], zero[3];
} ora_biv_t;

static void ora_biv_consts(const double *theta, int kernel, ora_biv_t *c)
{
    if (kernel == 3) {
        const double scale1 = theta[0], scale2 = theta[1], nu1 = theta[4], nu2 = theta[5];
        const double scale12 = pow(0.5 * (pow(scale1, -2) + pow(scale2, -2)) + theta[2] * (1 - theta[3]), -0.5);
        const double nu12 = 0.5 * (nu1 + nu2) + theta[6] * (1 - theta[7]);
        const double rho = theta[8] * theta[9] * theta[10] * pow(scale12, 2 * theta[6] + (nu1 + nu2)) *
                           tgamma(0.5 * (nu1 + nu2) + 1) * tgamma(nu12) / tgamma(nu12 + 1);
        const double s11 = theta[8] * theta[8] * pow(scale1, 2 * theta[6] + nu1 + nu1) * tgamma(nu1);
        const double s22 = theta[9] * theta[9] * pow(scale2, 2 * theta[6] + nu2 + nu2) * tgamma(nu2);
        double con1 = pow(2, (nu1 - 1)) * tgamma(nu1);
        con1 = 1.0 / con1;
        con1 = s11 * con1;
        double con2 = pow(2, (nu2 - 1)) * tgamma(nu2);
        con2 = 1.0 / con2;
        con2 = s22 * con2;
        double con12 = pow(2, (nu12 - 1)) * tgamma(nu12);
        con12 = 1.0 / con12;
        con12 = rho * con12;
        const double con[3] = {con1, con2, con12}, nu[3] = {nu1, nu2, nu12};
        const double sc[3] = {scale1, scale2, scale12}, zero[3] = {theta[0], theta[1], rho};
        for (int t = 0; t < 3; ++t) {
            c->con[t] = con[t];
            c->nu[t] = nu[t];
            c->scale[t] = sc[t];
            c->zero[t] = zero[t];
        }
        return;
    }
    double con1 = pow(2, (theta[3] - 1)) * tgamma(theta[3]);
    con1 = 1.0 / con1;
    con1 = theta[0] * con1;
    double con2 = pow(2, (theta[4] - 1)) * tgamma(theta[4]);
    con2 = 1.0 / con2;
    con2 = theta[1] * con2;
    const double nu12 = 0.5 * (theta[3] + theta[4]);
    const double rho = theta[5] * sqrt((tgamma(theta[3] + 1) * tgamma(theta[4] + 1)) /
                                       (tgamma(theta[3]) * tgamma(theta[4]))) *
                       tgamma(nu12) / tgamma(nu12 + 1);
    double con12 = pow(2, (nu12 - 1)) * tgamma(nu12);
    con12 = 1.0 / con12;
    con12 = rho * sqrt(theta[0] * theta[1]) * con12;
    const double con[3] = {con1, con2, con12}, nu[3] = {theta[3], theta[4], nu12};
    const double zero[3] = {theta[0], theta[1], rho * sqrt(theta[0] * theta[1])};
    for (int t = 0; t < 3; ++t) {
        c->con[t] = con[t];
        c->nu[t] = nu[t];
        c->scale[t] = theta[2];
        c->zero[t] = zero[t];
    }
}

/* Element between variable a of (x1, y1) and variable b of (x2, y2)
 * (core_zcmg.c:1656-1671 and :1561-1576: the 2 x 2 block of one location
 * pair; the zero-distance test is on the first component's scaled distance). */
static inline double ora_biv_elem(double x1, double y1, double x2, double y2, int a, int b, const ora_biv_t *c)
{
    const double d = ora_distance(x1, y1, x2, y2);
    const int t = a != b ? 2 : a;
    if (d / c->scale[0] == 0) return c->zero[t];
    const double expr = d / c->scale[t];
    return c->con[t] * pow(expr, c->nu[t]) * ora_bessel_knu(c->nu[t], expr);
}

/* core_dcmg: A (column-major, lda = m) = Sigma(l1[m0:m0+m], l2[n0:n0+n]).
 * Bivariate (kernel 2): rows and columns are matrix indices 2 l + v (location
 * l, variable v), as the reference's i0 = m0 / 2 loop (core_zcmg.c:1652-1673). */
void ora_core_dcmg(double *A, int m, int n, int m0, int n0, const double *x1, const double *y1, const double *x2,
                   const double *y2, const double *theta, int kernel)
{
    if (kernel == 2 || kernel == 3) {
        ora_biv_t c;
        ora_biv_consts(theta, kernel, &c);
#pragma omp parallel for schedule(static)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < m; ++i) {
                const int gi = m0 + i, gj = n0 + j;
                A[i + (size_t)j * m] = ora_biv_elem(x1[gi / 2], y1[gi / 2], x2[gj / 2], y2[gj / 2], gi % 2, gj % 2,
                                                    &c);
            }
        return;
    }
    const double con = ora_matern_con(theta);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i)
            A[i + (size_t)j * m] = ora_matern_elem(x1[m0 + i], y1[m0 + i], x2[n0 + j], y2[n0 + j], theta, con, kernel);
}

/* ========================================================================== */
/* Covariance derivatives: core_dcmg_matern_dsigma_square / _dbeta / _dnu      */
/* ========================================================================== */

/* psi (digamma) as the reference's series (core_zcmg.c:199-211): upward
 * recurrence to x >= 7, then the asymptotic expansion of psi(t + 1/2) at
 * t = x - 1/2 (absolute error below 1e-10). */
static double ora_psi(double x)
{
    double result = 0.0;
    for (; x < 7; ++x) result -= 1 / x;
    x -= 1.0 / 2.0;
    const double xx = 1.0 / x, xx2 = xx * xx, xx4 = xx2 * xx2;
    return result + log(x) + (1. / 24.) * xx2 - (7.0 / 960.0) * xx4 + (31.0 / 8064.0) * xx4 * xx2 -
           (127.0 / 30720.0) * xx4 * xx4;
}

/* dK_nu(x)/dnu.  The reference takes a forward difference with h = 1e-9
 * (dbessel_nu, core_zcmg.c:228-235), good to ~1e-7 relative; the oracle takes
 * the 4th-order central difference with h = 2e-4 (truncation ~h^4 log(2/x)^5
 * and rounding ~eps / h, both near 1e-12 relative for x >= 1e-4).  K_nu is
 * even in nu, so orders below zero are taken at |nu|. */
static double ora_dknu_dnu(double nu, double x)
{
    const double h = 2e-4;
    const double kp1 = ora_bessel_knu(nu + h, x), km1 = ora_bessel_knu(fabs(nu - h), x);
    const double kp2 = ora_bessel_knu(nu + 2 * h, x), km2 = ora_bessel_knu(fabs(nu - 2 * h), x);
    return (8.0 * (kp1 - km1) - (kp2 - km2)) / (12.0 * h);
}

/* Derivative `which` (0 sigma^2, 1 beta, 2 nu) of one Matern element,
 * core_zcmg.c:315-342 (dsigma_square), 453-488 (dbeta, with dbessel_input
 * :189-191), 380-416 (dnu); zero distance gives 1, 0, 0. */
static double ora_dmatern_elem(double x1, double y1, double x2, double y2, const double *theta, int which)
{
    const double expr = ora_distance(x1, y1, x2, y2) / theta[1];
    if (expr == 0) return which == 0 ? 1.0 : 0.0;
    const double nu = theta[2], beta = theta[1], sigma2 = theta[0];
    const double con = 1.0 / (pow(2, (nu - 1)) * tgamma(nu));
    const double knu = ora_bessel_knu(nu, expr);
    if (which == 0) return con * pow(expr, nu) * knu;
    if (which == 1) {
        const double dk = nu / expr * knu - ora_bessel_knu(nu + 1, expr);
        const double beta_expr = -nu / beta * pow(expr, nu) * knu - pow(expr, nu) * dk * expr / beta;
        return sigma2 * con * beta_expr;
    }
    const double g = tgamma(nu);
    const double nu_expr =
        -2 * log(2.0) * pow(2, -nu) * 1 / g * pow(expr, nu) * knu +
        pow(2, 1 - nu) * (-1 / g * ora_psi(nu) * pow(expr, nu) * knu +
                          1 / g * (pow(expr, nu) * log(expr) * knu + pow(expr, nu) * ora_dknu_dnu(nu, expr)));
    return sigma2 * nu_expr;
}

/* A (column-major, lda = m) = dSigma/dtheta_which (l1[m0:m0+m], l2[n0:n0+n]). */
void ora_dcmg_deriv(double *A, int m, int n, int m0, int n0, const double *x1, const double *y1, const double *x2,
                    const double *y2, const double *theta, int which)
{
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i)
            A[i + (size_t)j * m] = ora_dmatern_elem(x1[m0 + i], y1[m0 + i], x2[n0 + j], y2[n0 + j], theta, which);
}

/* Lower triangle (with the diagonal) of the N x N covariance, column-major.
 * The reference generates the lower tiles and the full diagonal tiles
 * (codelet_zcmg.c:316-342); LAPACK dpotrf reads only the lower triangle. */
static void ora_gen_lower(double *C, int N, const double *x, const double *y, const double *theta, int kernel)
{
    if (kernel == 2 || kernel == 3) {
        ora_biv_t c;
        ora_biv_consts(theta, kernel, &c);
#pragma omp parallel for schedule(dynamic, 16)
        for (int j = 0; j < N; ++j)
            for (int i = j; i < N; ++i)
                C[i + (size_t)j * N] = ora_biv_elem(x[i / 2], y[i / 2], x[j / 2], y[j / 2], i % 2, j % 2, &c);
        return;
    }
    const double con = ora_matern_con(theta);
#pragma omp parallel for schedule(dynamic, 16)
    for (int j = 0; j < N; ++j)
        for (int i = j; i < N; ++i)
            C[i + (size_t)j * N] = ora_matern_elem(x[i], y[i], x[j], y[j], theta, con, kernel);
}

/* ========================================================================== */
/* Likelihood, synthetic Z, prediction                                        */
/* ========================================================================== */

int ora_dlarnv(int seed, int n, double *out)
{
    blasint64 iseed[4] = {seed, seed, seed, 1};
    return (int)scipy_LAPACKE_dlarnv64_(3, iseed, n, out);
}

/* EXAGEOSTAT_MLE_dzvg_Tile: z = chol(Sigma(theta0)) * nrand. */
int ora_dzvg(int N, const double *x, const double *y, const double *theta, int kernel, const double *nrand,
             double *z)
{
    double *C = (double *)malloc(sizeof(double) * (size_t)N * N);
    if (!C) return -100;
    ora_gen_lower(C, N, x, y, theta, kernel);
    blasint64 info = ora_potrf_tiles(N, C);
    if (info != 0) {
        free(C);
        return (int)info;
    }
    memcpy(z, nrand, sizeof(double) * (size_t)N);
    scipy_cblas_dtrmv64_(ORA_COL_MAJOR, ORA_LOWER, ORA_NOTRANS, ORA_NONUNIT, N, C, N, z, 1);
    free(C);
    return 0;
}

/* EXAGEOSTAT_dmle_Tile: loglik = -0.5 dotp - 0.5 logdet - (N/2.0) log(2 pi),
 * logdet = 2 sum log L_ii over positive pivots (core_zmdet.c:55),
 * dotp = |L^-1 z|^2.  times[0..2] = generation, factorisation, solve (s). */
int ora_dmle(int N, const double *x, const double *y, const double *z, const double *theta, int kernel,
             double *loglik, double *logdet_out, double *dotp_out, double *times)
{
    double t0 = ora_now();
    double *C = (double *)malloc(sizeof(double) * (size_t)N * N);
    double *v = (double *)malloc(sizeof(double) * (size_t)N);
    if (!C || !v) {
        free(C);
        free(v);
        return -100;
    }
    ora_gen_lower(C, N, x, y, theta, kernel);
    double t1 = ora_now();
    blasint64 info = ora_potrf_tiles(N, C);
    double t2 = ora_now();
    if (info != 0) {
        free(C);
        free(v);
        return (int)info;
    }
    double det = 0.0;
    for (int i = 0; i < N; ++i) {
        double d = C[i + (size_t)i * N];
        if (d > 0) det += log(d);
    }
    double logdet = 2 * det;
    memcpy(v, z, sizeof(double) * (size_t)N);
    scipy_cblas_dtrsv64_(ORA_COL_MAJOR, ORA_LOWER, ORA_NOTRANS, ORA_NONUNIT, N, C, N, v, 1);
    double dotp = scipy_cblas_ddot64_(N, v, 1, v, 1);
    double t3 = ora_now();
    *loglik = -0.5 * dotp - 0.5 * logdet - (double)(N / 2.0) * log(2.0 * ORA_PI);
    if (logdet_out) *logdet_out = logdet;
    if (dotp_out) *dotp_out = dotp;
    if (times) {
        times[0] = t1 - t0;
        times[1] = t2 - t1;
        times[2] = t3 - t2;
    }
    free(C);
    free(v);
    return 0;
}

/* Dense covariance (lower triangle, column-major) for element-wise checks. */
void ora_gen_lower_dense(double *C, int N, const double *x, const double *y, const double *theta, int kernel)
{
    ora_gen_lower(C, N, x, y, theta, kernel);
}

/* EXAGEOSTAT_dmle_Predict_Tile: C22 = Sigma(obs, obs) (lower), C12 =
 * Sigma(miss, obs) (full), dposv, zmiss = C12 alpha, MSE = sum (zactual -
 * zmiss)^2 / nZmiss, or -1 when zactual is NULL.  Returns -2 on a
 * factorisation failure. */
double ora_dpredict(int nmiss, int nobs, const double *xmiss, const double *ymiss, const double *xobs,
                    const double *yobs, const double *zobs, const double *zactual, const double *theta, int kernel,
                    double *zmiss)
{
    double *C22 = (double *)malloc(sizeof(double) * (size_t)nobs * nobs);
    double *C12 = (double *)malloc(sizeof(double) * (size_t)nmiss * nobs);
    double *alpha = (double *)malloc(sizeof(double) * (size_t)nobs);
    ora_gen_lower(C22, nobs, xobs, yobs, theta, kernel);
    ora_core_dcmg(C12, nmiss, nobs, 0, 0, xmiss, ymiss, xobs, yobs, theta, kernel);
    memcpy(alpha, zobs, sizeof(double) * (size_t)nobs);
    /* dposv: the tile Cholesky, then L y = b and L^T alpha = y */
    blasint64 info = ora_potrf_tiles(nobs, C22);
    if (info == 0) {
        scipy_cblas_dtrsv64_(ORA_COL_MAJOR, ORA_LOWER, ORA_NOTRANS, ORA_NONUNIT, nobs, C22, nobs, alpha, 1);
        scipy_cblas_dtrsv64_(ORA_COL_MAJOR, ORA_LOWER, ORA_TRANS, ORA_NONUNIT, nobs, C22, nobs, alpha, 1);
    }
    double mse = -1;
    if (info != 0) {
        mse = -2;
    } else {
        scipy_cblas_dgemv64_(ORA_COL_MAJOR, ORA_NOTRANS, nmiss, nobs, 1.0, C12, nmiss, alpha, 1, 0.0, zmiss, 1);
        if (zactual) {
            double s = 0.0;
            for (int i = 0; i < nmiss; ++i) s += pow((zactual[i] - zmiss[i]), 2);
            mse = s / nmiss;
        }
    }
    free(alpha);
    free(C12);
    free(C22);
    return mse;
}
