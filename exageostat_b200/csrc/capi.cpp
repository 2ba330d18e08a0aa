/*
 * The reference's C API (include/exageostat_b200.h) on top of the engine.
 *
 * Argument meaning, side effects on MLE_data / results and the per-iterate
 * log line follow the cited reference functions; where the reference calls
 * exit() this layer returns an error value instead.
 */
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/exageostat_b200.h"
#include "xg_engine.h"

/* misc/include/MLE_misc.h:350 / examples/examples.c:24 */
__attribute__((weak)) output results;

static bool xg_quiet()
{
    const char *s = getenv("EXAGEOSTAT_B200_SILENT");
    return s && *s && strcmp(s, "0") != 0;
}

/* kernel_fun -> (kernel id, number of parameters); the exact path of this
 * library covers the two univariate stationary Matern kernels
 * (MLE_dexact.c:272-298 lists the reference's set). */
static int xg_kernel_of(const MLE_data *data, int *kernel, int *nparams)
{
    const char *k = data->kernel_fun ? data->kernel_fun : "univariate_matern_stationary";
    if (strcmp(k, "univariate_matern_stationary") == 0) {
        *kernel = 0;
        *nparams = 3;
        return XG_OK;
    }
    if (strcmp(k, "univariate_matern_nuggets_stationary") == 0) {
        *kernel = 1;
        *nparams = 4;
        return XG_OK;
    }
    if (strcmp(k, "bivariate_matern_parsimonious") == 0) {
        /* N is 2 x the number of locations in data->l1 (synthetic_dmle_test.c:67-69, 134, 153) */
        *kernel = 2;
        *nparams = 6;
        return XG_OK;
    }
    if (strcmp(k, "bivariate_matern_flexible") == 0) {
        /* 11 parameters (examples/examples.c:221-223), N = 2 x the locations */
        *kernel = 3;
        *nparams = 11;
        return XG_OK;
    }
    return xg_fail(XG_ERR_UNSUPPORTED, "kernel_fun \"%s\" is not supported (univariate_matern_stationary, "
                                       "univariate_matern_nuggets_stationary, bivariate_matern_parsimonious and "
                                       "bivariate_matern_flexible are)",
                   k);
}

static int xg_metric_of(const MLE_data *data)
{
    return (data->dm && (strcmp(data->dm, "gc") == 0 || strcmp(data->dm, "gcd") == 0)) ? 1 : 0;
}

static bool xg_is_exact(const MLE_data *data)
{
    return data->computation == NULL || strcmp(data->computation, "exact") == 0;
}

/* ------------------------------------------------------------------------- */
/* init / finalize                                                           */
/* ------------------------------------------------------------------------- */

extern "C" void exageostat_init(int *ncores, int *gpus, int *dts, int *lts)
{
    (void)ncores;
    (void)lts;
    if (g_xg.initialized) {
        printf("Another instance of Chameleon is already running...!");
        return;
    }
    if (gpus && *gpus > 1) fprintf(stderr, "exageostat_b200: one GPU per field; using the current device only\n");
    int rc = xg_context_start(dts ? *dts : 0);
    if (rc) fprintf(stderr, "exageostat_b200: init failed: %s\n", exageostat_last_error());
}

extern "C" void EXAGEOSTAT_init(int *ncores, int *gpus, int *dts, int *lts) { exageostat_init(ncores, gpus, dts, lts); }

extern "C" void exageostat_finalize(void)
{
    if (!g_xg.initialized) {
        printf("No active instance oh Chameleon...please use exageostat_init() function to initiate a new instance!\n");
        return;
    }
    cudaStreamSynchronize(g_xg.stream);
    cudaStreamDestroy(g_xg.stream);
    g_xg.stream = nullptr;
    g_xg.initialized = false;
}

/* ------------------------------------------------------------------------- */
/* descriptors                                                               */
/* ------------------------------------------------------------------------- */

static XgField *xg_field_of(MLE_data *data) { return data ? (XgField *)data->descC : nullptr; }

extern "C" void EXAGEOSTAT_dmle_Call(MLE_data *data, int ncores, int gpus, int dts, int p_grid, int q_grid, int N,
                                     int nZobs, int nZmiss)
{
    (void)ncores;
    (void)gpus;
    (void)p_grid;
    (void)q_grid;
    (void)nZobs;
    (void)nZmiss;
    int kernel = 0, np = 0;
    if (xg_kernel_of(data, &kernel, &np)) {
        fprintf(stderr, "EXAGEOSTAT_dmle_Call: %s\n", exageostat_last_error());
        return;
    }
    if (data->descC) MLE_Finalize(data);
    XgField *f = nullptr;
    const int ts = dts > 0 ? dts : g_xg.dts;
    if (xg_field_create(&f, N, ts, data->l1.x, data->l1.y, kernel, xg_metric_of(data))) {
        fprintf(stderr, "EXAGEOSTAT_dmle_Call: %s\n", exageostat_last_error());
        return;
    }
    data->descC = f;
    data->descZ = f;
    data->descZcpy = f;
    data->descdet = &data->det;
    data->descproduct = &data->dotp;
    data->sequence = NULL;
    data->request = NULL;
}

extern "C" void MORSE_dmle_Call(MLE_data *data, int ncores, int gpus, int dts, int p_grid, int q_grid, int N,
                                int nZobs, int nZmiss)
{
    EXAGEOSTAT_dmle_Call(data, ncores, gpus, dts, p_grid, q_grid, N, nZobs, nZmiss);
}

extern "C" void MLE_Finalize(MLE_data *data)
{
    if (!data) return;
    XgField *f = xg_field_of(data);
    if (f) xg_field_destroy(f);
    data->descC = data->descZ = data->descZcpy = NULL;
    data->descdet = data->descproduct = NULL;
}

/* ------------------------------------------------------------------------- */
/* synthetic z                                                               */
/* ------------------------------------------------------------------------- */

extern "C" void MLE_zvg(MLE_data *data, double *Nrand, double *initial_theta, int n, int ts, int log, int p_grid,
                        int q_grid)
{
    (void)ts;
    (void)log;
    (void)p_grid;
    (void)q_grid;
    data->iter_count = 0;
    XgField *f = xg_field_of(data);
    if (!f) {
        xg_fail(XG_ERR_NOT_INITIALIZED, "MLE_zvg before EXAGEOSTAT_dmle_Call");
        fprintf(stderr, "MLE_zvg: %s\n", exageostat_last_error());
        return;
    }
    if (!xg_is_exact(data) || (data->precision != 0 && data->precision != 2 && data->precision != 3)) {
        xg_fail(XG_ERR_UNSUPPORTED, "MLE_zvg: computation=%s precision=%d", data->computation, data->precision);
        fprintf(stderr, "%s\n", exageostat_last_error());
        return;
    }
    if (n != f->N) {
        xg_fail(XG_ERR_BAD_ARGUMENT, "MLE_zvg: n = %d but the descriptors hold N = %d", n, f->N);
        fprintf(stderr, "%s\n", exageostat_last_error());
        return;
    }
    double times[2] = {0, 0};
    if (xg_field_zvg(f, initial_theta, Nrand, times)) {
        fprintf(stderr, "MLE_zvg: %s\n", exageostat_last_error());
        return;
    }
    data->avg_exec_time_gen_stage = times[1];
    const double flops = (double)n * n * n / 3.0;
    data->avg_flops_gen_stage = times[1] > 0 ? flops / 1e9 / times[1] : 0.0;
}

extern "C" void MLE_get_zobs(MLE_data *data, double *z, int n)
{
    XgField *f = xg_field_of(data);
    if (!f || xg_field_get_z(f, z, n)) fprintf(stderr, "MLE_get_zobs: %s\n", exageostat_last_error());
}

/* ------------------------------------------------------------------------- */
/* the likelihood                                                            */
/* ------------------------------------------------------------------------- */

/* recover(), misc/compute/MLE_misc.c:2037-2074: a line "iter theta... loglik"
 * of the recovery file replays that iteration's value. */
static bool xg_recover(const char *path, int iter, int np, double *loglik)
{
    FILE *fp = fopen(path, "r");
    if (!fp) return false;
    char line[4096];
    bool found = false;
    while (fgets(line, sizeof line, fp)) {
        char *save = NULL;
        char *tok = strtok_r(line, " \n", &save);
        if (!tok || atoi(tok) != iter) continue;
        int i = 0;
        for (; i < np && (tok = strtok_r(NULL, " \n", &save)); ++i) {
        }
        tok = strtok_r(NULL, " \n", &save);
        if (i == np && tok) {
            *loglik = atof(tok);
            found = true;
        }
        break;
    }
    fclose(fp);
    return found;
}

/* checkpointing(), misc/compute/MLE_misc.c:2014-2035 */
static void xg_checkpoint(const char *path, int iter, const double *theta, int np, double loglik)
{
    FILE *fp = fopen(path, "a");
    if (!fp) return;
    fprintf(fp, "%d ", iter);
    for (int i = 0; i < np; ++i) fprintf(fp, "%.17g ", theta[i]);
    fprintf(fp, "%.17g \n", loglik);
    fclose(fp);
}

extern "C" int exageostat_b200_loglik(MLE_data *data, const double *theta, double *loglik, double *grad)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    int kernel = 0, np = 0;
    int rc = xg_kernel_of(data, &kernel, &np);
    if (rc) return rc;
    if (!xg_is_exact(data)) return xg_fail(XG_ERR_UNSUPPORTED, "computation \"%s\"", data->computation);
    if (data->precision != 0 && data->precision != 2 && data->precision != 3)
        return xg_fail(XG_ERR_UNSUPPORTED,
                       "precision %d (0 = FP64, 2 = banded mixed, 3 = FP64 with INT8-sliced updates are supported)",
                       data->precision);
    const bool mixed = data->precision == 2;
    const bool sliced = data->precision == 3;
    const int band = data->diag_thick > 0 ? data->diag_thick : 1;
    if (mixed && grad)
        return xg_fail(XG_ERR_UNSUPPORTED, "the gradient is computed with precision 0 or 3, not 2");
    if (xg_bivariate(kernel) && (mixed || grad))
        return xg_fail(XG_ERR_UNSUPPORTED, "bivariate kernels: precision 0 or 3 without a gradient");
    if (mixed && (!f->mx || f->mx->band != band)) {
        rc = xg_field_set_mixed(f, band, f->mx ? f->mx->passes : 3);
        if (rc) return rc;
    }
    if (sliced && !f->sl) {
        rc = xg_field_set_sliced(f);
        if (rc) return rc;
    }
    double res[3], times[3] = {0, 0, 0};
    data->det = 0;
    data->dotp = 0;
    double t_gen = 0, t_fact = 0;
    if (data->recovery_file && data->recovery_file[0] &&
        xg_recover(data->recovery_file, data->iter_count, np, loglik)) {
        rc = XG_OK;
    } else {
        rc = mixed             ? xg_field_loglik_mixed(f, theta, res, times)
             : sliced && grad  ? xg_field_loglik_grad_sliced(f, theta, res, grad, times)
             : sliced          ? xg_field_loglik_sliced(f, theta, res, times)
             : grad            ? xg_field_loglik_grad(f, theta, res, grad, times)
                               : xg_field_loglik(f, theta, res, times);
        if (rc == XG_OK) {
            *loglik = res[0];
            data->det = 0.5 * res[1];
            data->dotp = res[2];
            t_gen = times[0];
            t_fact = times[1];
        }
    }
    if (rc != XG_OK) {
        *loglik = -INFINITY;
        if (grad)
            for (int i = 0; i < np; ++i) grad[i] = NAN;
    }
    /* per-iterate record, MLE_dexact.c:441-488 */
    if (!xg_quiet()) {
        fprintf(stderr, " %3d- Model Parameters (", data->iter_count + 1);
        for (int i = 0; i < np; ++i) fprintf(stderr, "%.8f%s", theta[i], i < np - 1 ? "," : "");
        fprintf(stderr, ")----> LogLi: %.18f\n", *loglik);
        fprintf(stderr, " ---- Facto Time: %6.2f\n", t_fact);
        fprintf(stderr, " ---- Matrix Generation Time: %6.2f\n", t_gen);
        fprintf(stderr, " ---- Total Time: %6.2f\n", t_gen + t_fact);
    }
    if (data->log == 1 && data->pFileLog) {
        fprintf(data->pFileLog, " %3d- Model Parameters (", data->iter_count + 1);
        for (int i = 0; i < np; ++i) fprintf(data->pFileLog, "%.8f, ", theta[i]);
        fprintf(data->pFileLog, ")----> LogLi: %.18f\n", *loglik);
    }
    if (data->checkpoint_file && data->checkpoint_file[0])
        xg_checkpoint(data->checkpoint_file, data->iter_count, theta, np, *loglik);
    if (results.estimated_theta)
        for (int i = 0; i < np; ++i) results.estimated_theta[i] = theta[i];
    data->iter_count++;
    const double n = f->N;
    data->avg_exec_time_per_iter += t_fact;
    if (t_fact > 0) data->avg_flops_per_iter += (n * n * n / 3.0 + n * n) / 1e9 / t_fact;
    data->avg_generation_per_iter += t_gen;
    data->avg_cholesky_per_iter += t_fact;
    data->final_loglik = *loglik;
    data->variance = theta[0];
    results.final_loglik = *loglik;
    return rc;
}

extern "C" double EXAGEOSTAT_dmle_Tile(unsigned n, const double *theta, double *grad, void *vdata)
{
    (void)n;
    double ll = -INFINITY;
    int rc = exageostat_b200_loglik((MLE_data *)vdata, theta, &ll, grad);
    if (rc && rc != XG_ERR_NOT_SPD) fprintf(stderr, "EXAGEOSTAT_dmle_Tile: %s\n", exageostat_last_error());
    return ll;
}

extern "C" double MORSE_dmle_Tile(unsigned n, const double *theta, double *grad, void *data)
{
    return EXAGEOSTAT_dmle_Tile(n, theta, grad, data);
}

/* EXAGEOSTAT_sdmle_Tile (MLE_sdexact.c:172-357): the banded mixed-precision
 * objective; data->diag_thick is the band width in tiles */
extern "C" double EXAGEOSTAT_sdmle_Tile(unsigned n, const double *theta, double *grad, void *vdata)
{
    MLE_data *data = (MLE_data *)vdata;
    const int saved = data->precision;
    data->precision = 2;
    const double ll = EXAGEOSTAT_dmle_Tile(n, theta, grad, vdata);
    data->precision = saved;
    return ll;
}

extern "C" double MLE_alg(unsigned n, const double *theta, double *grad, void *vdata)
{
    MLE_data *data = (MLE_data *)vdata;
    if (!xg_is_exact(data)) {
        fprintf(stderr, "MLE_alg: computation \"%s\" is not provided by this library\n", data->computation);
        return 0;
    }
    if (data->precision == 0 || data->precision == 2 || data->precision == 3)
        return EXAGEOSTAT_dmle_Tile(n, theta, grad, vdata);
    fprintf(stderr, "MLE_alg: precision %d is not provided by this library\n", data->precision);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* prediction                                                                */
/* ------------------------------------------------------------------------- */

extern "C" void EXAGEOSTAT_dmle_Predict_Allocate(MLE_data *data, int nZmiss, int nZobs, int dts, int p_grid,
                                                 int q_grid, int mse_flag)
{
    (void)p_grid;
    (void)q_grid;
    if (nZmiss <= 0) {
        fprintf(stderr, " Number of missing values should be positive value\n");
        return;
    }
    if (data->descC22) prediction_finalize(data);
    int kernel = 0, np = 0;
    if (xg_kernel_of(data, &kernel, &np) == XG_OK && xg_bivariate(kernel)) {
        /* the bivariate matrices have two rows per location (MLE_dexact.c:640-653) */
        nZobs *= 2;
        nZmiss *= 2;
    }
    XgPredict *q = nullptr;
    if (xg_predict_create(&q, nZmiss, nZobs, dts > 0 ? dts : g_xg.dts)) {
        fprintf(stderr, "EXAGEOSTAT_dmle_Predict_Allocate: %s\n", exageostat_last_error());
        return;
    }
    q->mse_flag = mse_flag;
    data->descC22 = q;
    data->descC12 = q;
    data->descZobs = q;
    data->descZmiss = q;
    data->descZactual = q;
    data->descmse = &data->mserror;
}

extern "C" void prediction_init(MLE_data *data, int nZmiss, int nZobs, int ts, int p_grid, int q_grid, int mse_flag)
{
    if (data->precision == 0 || data->precision == 2 || data->precision == 3)
        EXAGEOSTAT_dmle_Predict_Allocate(data, nZmiss, nZobs, ts, p_grid, q_grid, mse_flag);
}

extern "C" double EXAGEOSTAT_dmle_Predict_Tile(MLE_data *data, double *theta, int nZmiss, int nZobs, double *Zobs,
                                               double *Zactual, double *Zmiss, int n)
{
    (void)n;
    data->mserror = 0;
    if (nZmiss <= 0) {
        fprintf(stderr, " Number of missing values should be positive value\n");
        return -1;
    }
    int kernel = 0, np = 0;
    if (xg_kernel_of(data, &kernel, &np)) {
        fprintf(stderr, "EXAGEOSTAT_dmle_Predict_Tile: %s\n", exageostat_last_error());
        return -1;
    }
    XgPredict *q = (XgPredict *)data->descC22;
    if (!q || q->nmiss != nZmiss || q->nobs != nZobs) {
        if (q) prediction_finalize(data);
        /* nZmiss / nZobs count matrix rows here; the allocation takes locations */
        const int p = xg_bivariate(kernel) ? 2 : 1;
        EXAGEOSTAT_dmle_Predict_Allocate(data, nZmiss / p, nZobs / p, 0, 1, 1, Zactual != NULL);
        q = (XgPredict *)data->descC22;
        if (!q) return -1;
    }
    if (!xg_quiet()) {
        printf("estimated parameters:");
        for (int i = 0; i < np; ++i) printf("%.8f,", theta[i]);
        printf(")\n");
    }
    double mse = -1;
    const double t0 = 0;
    double parts[2] = {-1, -1};
    int rc = xg_predict_run(q, theta, kernel, xg_metric_of(data), data->lmiss.x, data->lmiss.y, data->lobs.x,
                            data->lobs.y, Zobs, Zactual, Zmiss, &mse, parts);
    (void)t0;
    if (rc) {
        fprintf(stderr, "EXAGEOSTAT_dmle_Predict_Tile: %s\n", exageostat_last_error());
        data->mserror = rc == XG_ERR_NOT_SPD ? -2 : -1;
        return data->mserror;
    }
    data->mserror = mse;
    results.mse_pred = mse;
    if (xg_bivariate(kernel)) { /* per-variable errors of the bivariate field (MLE_dexact.c:838-847, 859-860) */
        data->mserror1 = parts[0];
        data->mserror2 = parts[1];
        results.mse_pred1 = parts[0];
        results.mse_pred2 = parts[1];
    }
    return mse;
}

extern "C" double MORSE_dmle_Predict_Tile(MLE_data *data, double *theta, int nZmiss, int nZobs, double *Zobs,
                                          double *Zactual, double *Zmiss, int n)
{
    return EXAGEOSTAT_dmle_Predict_Tile(data, theta, nZmiss, nZobs, Zobs, Zactual, Zmiss, n);
}

extern "C" void prediction_finalize(MLE_data *data)
{
    XgPredict *q = (XgPredict *)data->descC22;
    if (q) xg_predict_destroy(q);
    data->descC22 = data->descC12 = data->descZobs = data->descZmiss = data->descZactual = NULL;
    data->descmse = NULL;
}

/* ------------------------------------------------------------------------- */
/* assessment: Fisher information, MLOE / MMOM                               */
/* ------------------------------------------------------------------------- */

/* MLE_dexact.c:1777-1934.  The reference generates Sigma and its derivatives
 * with univariate_matern_stationary whatever data->kernel_fun holds
 * (:1825, :1840-1842), so kernel 0 here too. */
extern "C" double *EXAGEOSTAT_Fisher_Tile(MLE_data *data, int N, double *initial_theta, int dts, int p_grid,
                                          int q_grid)
{
    (void)dts;
    (void)p_grid;
    (void)q_grid;
    XgField *f = xg_field_of(data);
    if (f && xg_bivariate(f->kernel)) {
        xg_fail(XG_ERR_UNSUPPORTED, "the Fisher matrix of a bivariate field");
        fprintf(stderr, "EXAGEOSTAT_Fisher_Tile: %s\n", exageostat_last_error());
        return NULL;
    }
    if (!f || f->N != N) {
        xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors for N = %d: call EXAGEOSTAT_dmle_Call first", N);
        fprintf(stderr, "EXAGEOSTAT_Fisher_Tile: %s\n", exageostat_last_error());
        return NULL;
    }
    double F[9], inv[9], t = 0.0;
    int rc = xg_field_fisher(f, initial_theta, 0, F, &t);
    if (!rc) rc = xg_small_spd_inverse(3, F, inv);
    if (rc) {
        fprintf(stderr, "EXAGEOSTAT_Fisher_Tile: %s\n", exageostat_last_error());
        return NULL;
    }
    if (!xg_quiet()) {
        printf("Fisher matrix\n");
        for (int i = 0; i < 3; ++i) printf("%12.6e %12.6e %12.6e\n", F[i * 3], F[i * 3 + 1], F[i * 3 + 2]);
        printf("Fisher matrix (inverse)\n");
        for (int i = 0; i < 3; ++i) printf("%12.6e %12.6e %12.6e\n", inv[i * 3], inv[i * 3 + 1], inv[i * 3 + 2]);
        fprintf(stderr, " ---- Time to calculate Fisher matrix: %6.4f seconds\n", t);
    }
    results.fisher_00 = inv[0];
    results.fisher_11 = inv[4];
    results.fisher_22 = inv[8];
    results.fisher_time = t;
    double *r = (double *)calloc(10, sizeof(double));
    if (!r) return NULL;
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) r[i + 3 * j] = inv[i * 3 + j];
    return r;
}

extern "C" int exageostat_b200_fisher(MLE_data *data, const double *theta, double *fisher, double *fisher_inv)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    int kernel = 0, np = 0;
    int rc = xg_kernel_of(data, &kernel, &np);
    if (rc) return rc;
    double F[16], inv[16], t = 0.0;
    rc = xg_field_fisher(f, theta, kernel, F, &t);
    if (rc) return rc;
    if (fisher) memcpy(fisher, F, np * np * sizeof(double));
    if (fisher_inv) {
        rc = xg_small_spd_inverse(np, F, inv);
        if (rc) return rc;
        memcpy(fisher_inv, inv, np * np * sizeof(double));
    }
    results.fisher_time = t;
    return XG_OK;
}

/* MLE_dexact.c:1002-1107: the descriptor handles all point at one workspace;
 * the reference exits on an unknown kernel_fun (:1055-1059), this prints the error. */
extern "C" void EXAGEOSTAT_dmle_mloe_mmom_Allocate(MLE_data *data, int nZmiss, int nZobs, int dts, int p_grid,
                                                   int q_grid)
{
    (void)p_grid;
    (void)q_grid;
    if (nZmiss <= 0) {
        fprintf(stderr, " Number of missing values should be positive value\n");
        return;
    }
    int kernel = 0, np = 0;
    if (xg_kernel_of(data, &kernel, &np) ||
        (xg_bivariate(kernel) && xg_fail(XG_ERR_UNSUPPORTED, "MLOE / MMOM with a bivariate kernel"))) {
        fprintf(stderr, "EXAGEOSTAT_dmle_mloe_mmom_Allocate: %s\n", exageostat_last_error());
        return;
    }
    if (data->desck_t) mloe_mmom_finalize(data);
    XgAssess *q = nullptr;
    if (xg_assess_create(&q, nZmiss, nZobs, dts > 0 ? dts : g_xg.dts)) {
        fprintf(stderr, "EXAGEOSTAT_dmle_mloe_mmom_Allocate: %s\n", exageostat_last_error());
        return;
    }
    data->mloe = 0;
    data->mmom = 0;
    data->desck_t = data->desck_a = data->desck_atmp = data->desck_ttmp = q;
    data->descK_t = data->descK_a = q;
    data->descexpr1 = data->descexpr2 = data->descexpr3 = data->descexpr4 = q;
    data->descmloe = &data->mloe;
    data->descmmom = &data->mmom;
}

extern "C" void mloe_mmom_init(MLE_data *data, int nZmiss, int nZobs, int ts, int p_grid, int q_grid)
{
    EXAGEOSTAT_dmle_mloe_mmom_Allocate(data, nZmiss, nZobs, ts, p_grid, q_grid);
}

extern "C" void mloe_mmom_finalize(MLE_data *data)
{
    XgAssess *q = (XgAssess *)data->desck_t;
    if (q) xg_assess_destroy(q);
    data->desck_t = data->desck_a = data->desck_atmp = data->desck_ttmp = NULL;
    data->descK_t = data->descK_a = NULL;
    data->descexpr1 = data->descexpr2 = data->descexpr3 = data->descexpr4 = NULL;
    data->descmloe = data->descmmom = NULL;
}

extern "C" void MLOE_MMOM_Finalize(MLE_data *data) { mloe_mmom_finalize(data); }

/* flop count the reference reports (MLE_dexact.c:1265-1359, 1395): two
 * factorisations and, per missing point, four vector TRSMs and four
 * vector-vector products */
static double xg_mloe_mmom_flops(int nmiss, int nobs)
{
    const double n = nobs;
    return 2.0 * (n * n * n / 3.0 + n * n / 2.0 + n / 6.0) + (double)nmiss * (4.0 * n * n + 4.0 * 2.0 * n);
}

static void xg_mloe_mmom(MLE_data *data, double *truth_theta, double *estimated_theta, int nZmiss, int nZobs,
                         const char *mode)
{
    int kernel = 0, np = 0;
    if (xg_kernel_of(data, &kernel, &np) ||
        (xg_bivariate(kernel) && xg_fail(XG_ERR_UNSUPPORTED, "MLOE / MMOM with a bivariate kernel"))) {
        fprintf(stderr, "EXAGEOSTAT_dmle_mloe_mmom_Tile: %s\n", exageostat_last_error());
        data->mloe = data->mmom = NAN;
        return;
    }
    if (!data->lmiss.x || !data->lmiss.y || !data->lobs.x || !data->lobs.y) {
        xg_fail(XG_ERR_BAD_ARGUMENT, "data->lobs / data->lmiss hold no locations (pick_random_points sets them)");
        fprintf(stderr, "EXAGEOSTAT_dmle_mloe_mmom_Tile: %s\n", exageostat_last_error());
        data->mloe = data->mmom = NAN;
        return;
    }
    XgAssess *q = (XgAssess *)data->desck_t;
    if (!q || q->nmiss != nZmiss || q->nobs != nZobs) {
        EXAGEOSTAT_dmle_mloe_mmom_Allocate(data, nZmiss, nZobs, 0, 1, 1);
        q = (XgAssess *)data->desck_t;
        if (!q) return;
    }
    double mloe = 0, mmom = 0, times[4] = {0, 0, 0, 0};
    int rc = xg_assess_run(q, truth_theta, estimated_theta, kernel, xg_metric_of(data), data->lmiss.x, data->lmiss.y,
                           data->lobs.x, data->lobs.y, &mloe, &mmom, NULL, times);
    if (rc) {
        fprintf(stderr, "EXAGEOSTAT_dmle_mloe_mmom_Tile: %s\n", exageostat_last_error());
        data->mloe = data->mmom = NAN;
        return;
    }
    data->mloe = mloe;
    data->mmom = mmom;
    results.mloe = mloe;
    results.mmom = mmom;
    results.mloe_exec = (char *)mode;
    results.total_mloe_mmom_time = times[3];
    results.matrix_gen_mloe_mmom_time = times[0];
    results.cho_fact_mloe_mmom_time = times[1];
    results.loop_mloe_mmom_time = times[2];
    results.total_mloe_mmom_flops = xg_mloe_mmom_flops(nZmiss, nZobs) / 1e9 / (times[1] + times[2]);
    if (!xg_quiet()) {
        printf("\nnZmiss = %d\n", nZmiss);
        printf(" ----(MLOE-MMOM) Gflop/s: %6.2f\n", results.total_mloe_mmom_flops);
        printf("\nMMLOE = %f", mloe);
        printf("\nMMOM = %f\n\n\n", mmom);
        fprintf(stderr, " ---- mloe_mmom Time: %6.2f seconds\n\n", times[3]);
    }
}

extern "C" void EXAGEOSTAT_dmle_mloe_mmom_Tile(MLE_data *data, double *truth_theta, double *estimated_theta,
                                               int nZmiss, int nZobs, int n)
{
    (void)n;
    xg_mloe_mmom(data, truth_theta, estimated_theta, nZmiss, nZobs, "sync");
}

extern "C" void EXAGEOSTAT_dmle_mloe_mmom_Tile_Async(MLE_data *data, double *truth_theta, double *estimated_theta,
                                                     int nZmiss, int nZobs, int n)
{
    (void)n;
    xg_mloe_mmom(data, truth_theta, estimated_theta, nZmiss, nZobs, "async");
}

extern "C" int exageostat_b200_fisher_host(int n, const double *x, const double *y, const double *theta, int kernel,
                                           int metric, int ts, double *fisher)
{
    if (kernel != 0 && kernel != 1) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    XgField *f = nullptr;
    int rc = xg_field_create(&f, n, ts, x, y, kernel, metric);
    if (rc) return rc;
    double t = 0.0;
    rc = xg_field_fisher(f, theta, kernel, fisher, &t);
    xg_field_destroy(f);
    return rc;
}

extern "C" int exageostat_b200_mloe_mmom_host(int nmiss, const double *xmiss, const double *ymiss, int nobs,
                                              const double *xobs, const double *yobs, const double *truth_theta,
                                              const double *estimated_theta, int kernel, int metric, int ts,
                                              double *mloe, double *mmom, double *terms, double *times)
{
    if (kernel != 0 && kernel != 1) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    XgAssess *q = nullptr;
    int rc = xg_assess_create(&q, nmiss, nobs, ts);
    if (rc) return rc;
    rc = xg_assess_run(q, truth_theta, estimated_theta, kernel, metric, xmiss, ymiss, xobs, yobs, mloe, mmom, terms,
                       times);
    xg_assess_destroy(q);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* one-shot and diagnostic entry points                                      */
/* ------------------------------------------------------------------------- */

extern "C" int exageostat_b200_dmle_host(int n, const double *x, const double *y, const double *z,
                                         const double *theta, int kernel, int metric, int ts, double *out)
{
    if (kernel < 0 || kernel > 3) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    XgField *f = nullptr;
    int rc = xg_field_create(&f, n, ts, x, y, kernel, metric);
    if (rc) return rc;
    rc = xg_field_set_z(f, z);
    double res[3];
    if (!rc) rc = xg_field_loglik(f, theta, res, nullptr);
    if (!rc) memcpy(out, res, sizeof res);
    xg_field_destroy(f);
    return rc;
}

extern "C" int exageostat_b200_set_mixed(MLE_data *data, int band, int passes)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    data->diag_thick = band;
    return xg_field_set_mixed(f, band, passes);
}

extern "C" int exageostat_b200_dmle_host_mixed(int n, const double *x, const double *y, const double *z,
                                               const double *theta, int kernel, int metric, int ts, int band,
                                               int passes, double *out)
{
    if (kernel != 0 && kernel != 1) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    XgField *f = nullptr;
    int rc = xg_field_create(&f, n, ts > 0 ? ts : 512, x, y, kernel, metric);
    if (rc) return rc;
    rc = xg_field_set_z(f, z);
    if (!rc) rc = xg_field_set_mixed(f, band, passes);
    double res[3];
    if (!rc) rc = xg_field_loglik_mixed(f, theta, res, nullptr);
    if (!rc) memcpy(out, res, sizeof res);
    xg_field_destroy(f);
    return rc;
}

extern "C" int exageostat_b200_set_sliced(MLE_data *data)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    data->precision = 3;
    return xg_field_set_sliced(f);
}

extern "C" int exageostat_b200_dmle_host_sliced(int n, const double *x, const double *y, const double *z,
                                                const double *theta, int kernel, int metric, int ts, double *out)
{
    if (kernel < 0 || kernel > 3) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    XgField *f = nullptr;
    int rc = xg_field_create(&f, n, ts, x, y, kernel, metric);
    if (rc) return rc;
    rc = xg_field_set_z(f, z);
    if (!rc) rc = xg_field_set_sliced(f);
    double res[3];
    if (!rc) rc = xg_field_loglik_sliced(f, theta, res, nullptr);
    if (!rc) memcpy(out, res, sizeof res);
    xg_field_destroy(f);
    return rc;
}

extern "C" int exageostat_b200_sliced_factor_dense(int n, const double *x, const double *y, const double *theta,
                                                   int kernel, int metric, int ts, double *out)
{
    return xg_sliced_factor_dense(n, x, y, theta, kernel, metric, ts, out);
}

extern "C" int exageostat_b200_autotune(MLE_data *data, const double *theta, double tol, int *ts, int *band,
                                        double *report)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    if (!f->have_z) return xg_fail(XG_ERR_BAD_ARGUMENT, "no observations: call MLE_zvg or set z first");
    if (!data->l1.x || !data->l1.y) return xg_fail(XG_ERR_BAD_ARGUMENT, "data->l1 holds no locations");
    int kernel = 0, np = 0;
    int rc = xg_kernel_of(data, &kernel, &np);
    if (rc) return rc;
    rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    int ts_out = 0, band_out = 0;
    rc = xg_autotune_field(&f, data->l1.x, data->l1.y, theta, data->precision, tol > 0 ? tol : 1e-6, &ts_out,
                           &band_out, report);
    data->descC = data->descZ = data->descZcpy = f;
    if (rc) return rc;
    if (ts) *ts = ts_out;
    if (band) *band = band_out;
    if (data->precision == 2) data->diag_thick = band_out;
    return XG_OK;
}

extern "C" int exageostat_b200_mixed_factor_dense(int n, const double *x, const double *y, const double *theta,
                                                  int kernel, int metric, int ts, int band, int passes, double *out)
{
    return xg_mixed_factor_dense(n, x, y, theta, kernel, metric, ts, band, passes, out);
}

extern "C" int exageostat_b200_bessel_knu(int n, const double *nu, const double *x, double *out)
{
    return xg_bessel_knu_host(n, nu, x, out);
}

extern "C" int exageostat_b200_matern_pairs(int n, const double *x1, const double *y1, const double *x2,
                                            const double *y2, const double *theta, int kernel, int metric,
                                            double *out)
{
    return xg_matern_pairs_host(n, x1, y1, x2, y2, theta, kernel, metric, out);
}

extern "C" int exageostat_b200_covariance_dense(int n, const double *x, const double *y, const double *theta,
                                                int kernel, int metric, int ts, int factor, double *out)
{
    return xg_covariance_dense(n, x, y, theta, kernel, metric, ts, factor, out);
}

extern "C" int exageostat_b200_set_data(MLE_data *data, const double *x, const double *y, const double *z)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    return xg_field_set_data(f, x, y, z);
}

extern "C" int exageostat_b200_set_profiling(MLE_data *data, int on)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    return xg_field_set_profiling(f, on);
}

extern "C" int exageostat_b200_get_profile(MLE_data *data, double *out, int n)
{
    XgField *f = xg_field_of(data);
    if (!f) return xg_fail(XG_ERR_NOT_INITIALIZED, "no descriptors: call EXAGEOSTAT_dmle_Call first");
    double info[15] = {f->prof[0], f->prof[1], f->prof[2], f->prof[3], f->prof[4],  f->prof[5],
                       f->prof[6], f->prof[7], (double)f->C.ts, (double)f->C.nt, (double)f->N,
                       f->prof[8], f->prof[9], f->prof[10], f->prof[11]};
    for (int i = 0; i < n && i < 15; ++i) out[i] = info[i];
    return XG_OK;
}

extern "C" int exageostat_b200_abi_version(void) { return 1; }
extern "C" size_t exageostat_b200_sizeof_MLE_data(void) { return sizeof(MLE_data); }
extern "C" size_t exageostat_b200_sizeof_output(void) { return sizeof(output); }

extern "C" long exageostat_b200_offsetof_MLE_data(const char *field)
{
#define XG_OFF(name)                                                                                                   \
    if (strcmp(field, #name) == 0) return (long)offsetof(MLE_data, name)
    XG_OFF(variance);
    XG_OFF(computation);
    XG_OFF(iter_count);
    XG_OFF(l1);
    XG_OFF(lmiss);
    XG_OFF(lobs);
    XG_OFF(descC);
    XG_OFF(descZcpy);
    XG_OFF(descC22);
    XG_OFF(verbose);
    XG_OFF(log);
    XG_OFF(avg_exec_time_per_iter);
    XG_OFF(final_loglik);
    XG_OFF(det);
    XG_OFF(dotp);
    XG_OFF(sdotp);
    XG_OFF(mserror);
    XG_OFF(dm);
    XG_OFF(diag_thick);
    XG_OFF(pFileLog);
    XG_OFF(hicma_acc);
    XG_OFF(opt_tol);
    XG_OFF(kernel_fun);
    XG_OFF(precision);
    XG_OFF(expr1);
    XG_OFF(mloe_mmom);
    XG_OFF(recovery_file);
    XG_OFF(checkpoint_file);
    XG_OFF(seed);
#undef XG_OFF
    return -1;
}
