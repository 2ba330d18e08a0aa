/*
 * Host engine: device objects behind the MLE_data handles.
 */
#ifndef EXAGEOSTAT_B200_ENGINE_H
#define EXAGEOSTAT_B200_ENGINE_H

#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "xg_kernels.h"

struct XgContext {
    bool initialized = false;
    int device = 0;
    int sm_count = 0;
    int dts = 0;
    cudaStream_t stream = nullptr;    /* trailing updates, generation, solves */
    cudaStream_t stream_hi = nullptr; /* high priority: the lookahead panel (POTRF + TRSM) */
    std::mutex mu;
};

/* Streams and events of one factorisation.  With st_hi == nullptr the steps
 * run in order on st; otherwise panel k+1 (POTRF, TRSM on st_hi) overlaps the
 * trailing update of step k (st), ordered by the two events. */
struct XgFactorStreams {
    cudaStream_t st = nullptr;
    cudaStream_t st_hi = nullptr;
    cudaEvent_t ev_panel = nullptr, ev_upd = nullptr;
    cudaEvent_t *pev = nullptr; /* optional profiling events, 4 per step + 1 */
};
extern XgContext g_xg;

struct XgTileMatrix {
    int N = 0, ts = 0, nt = 0;
    long long ntiles = 0;
    double *d = nullptr;
    int2 *ij = nullptr; /* (i, j) of every packed tile */
    CUtensorMap map;    /* TMA view for the trailing-update kernel */
    double *dinv = nullptr; /* ts x 32: inverted 32 x 32 diagonal blocks of the current panel */
};

/* Banded mixed-precision workspace (mixed.cu): compact FP64 band tiles,
 * compact FP32 off-band tiles, double-buffered panel copies. */
struct XgMixed {
    int band = 1, passes = 3;
    XgTileArgs T;
    double *p64[2] = {nullptr, nullptr};
    float *phi[2] = {nullptr, nullptr}, *plo[2] = {nullptr, nullptr};
    XgMixedMaps maps[2];
};

/* FP64 tiles with INT8-sliced trailing updates (sliced.cu), left-looking:
 * the digit planes and row scales of every factored panel tile
 * (tile-packed, 4 bytes + 8 / ts bytes per element) and the lookahead events. */
struct XgSliced {
    long long plane_rows = 0; /* rows per digit plane (ntiles * ts) */
    int8_t *dig = nullptr;
    double *scale = nullptr;
    CUtensorMap map_a, map_b; /* A and B operand views (boxes of 128 rows x 64 bytes) */
    cudaEvent_t ev_a = nullptr, ev_p[2] = {nullptr, nullptr};
    /* gradient: digit planes of the inverse factor X = L^-T (slot layout of X) */
    int8_t *xdig = nullptr;
    double *xscale = nullptr;
    CUtensorMap xmap;
};

/* One dataset: locations, observations and the covariance / factor. */
struct XgField {
    int N = 0;
    int kernel = 0; /* 0 Matern, 1 Matern + nugget */
    int metric = 0; /* 0 Euclidean, 1 great circle */
    XgTileMatrix C;
    double *x = nullptr, *y = nullptr; /* padded to nt * ts */
    double *z = nullptr;               /* observations (zero padded); never modified by evaluations */
    double *v = nullptr;               /* solve work vector */
    double *e = nullptr;               /* N(0,1) draws for MLE_zvg */
    double *part = nullptr;            /* per-tile log-det / dot partials (2 nt) */
    double *out = nullptr;             /* device result record */
    int *status = nullptr, *info = nullptr;
    double *h_out = nullptr; /* pinned copy of out */
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    bool have_z = false;
    cudaEvent_t ev_panel = nullptr, ev_upd = nullptr; /* lookahead ordering */
    /* gradient workspace, allocated on the first gradient request */
    XgTileMatrix X;              /* X = L^-T (lower-tile slots, X_IK at slot (K, I)) */
    XgMixed *mx = nullptr;       /* mixed-precision workspace (precision 2) */
    XgSliced *sl = nullptr;      /* INT8-sliced workspace (precision 3) */
    double *gpart = nullptr;     /* per-CTA contraction partials */
    double *gout = nullptr;      /* 4 gradient sums */
    /* optional per-kernel-class timing (exageostat_b200_set_profiling) */
    bool profiling = false;
    cudaEvent_t *pev = nullptr; /* 8 per step around the factorisation kernels */
    /* gen, potrf, trsm(+panel prep), trailing seconds; trailing flops; launches; evals; total seconds;
     * mixed only: off-band (tcgen05) seconds, off-band flops, band (DMMA) seconds, band flops */
    double prof[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
};

struct XgPredict {
    int nmiss = 0, nobs = 0;
    int mse_flag = 1;
    XgTileMatrix C22;
    double *xm = nullptr, *ym = nullptr, *xo = nullptr, *yo = nullptr;
    double *v = nullptr, *zact = nullptr, *zmiss = nullptr, *part = nullptr, *out = nullptr;
    int *status = nullptr;
    cudaEvent_t ev_panel = nullptr, ev_upd = nullptr;
    int *info() { return status + 1; }
};

/* kernels whose rows and columns interleave two variables per location:
 * 2 bivariate parsimonious, 3 bivariate flexible Matern */
inline bool xg_bivariate(int kernel) { return kernel == 2 || kernel == 3; }

int xg_fail(int code, const char *fmt, ...);
int xg_context_start(int dts);
int xg_context_require();
int xg_choose_ts(int N, int dts);
int xg_tm_alloc(XgTileMatrix &M, int N, int ts);
int xg_encode_tiles(CUtensorMap *map, double *base, long long ntiles, int ts);
void xg_tm_free(XgTileMatrix &M);
XgMaternParams xg_params(const double *theta, int kernel);
int xg_check_theta(const double *theta, int kernel);
void xg_factor(XgTileMatrix &M, double *v, double *part, int *status, int *info, cudaStream_t st,
               cudaEvent_t *pev = nullptr);
void xg_factor_lookahead(XgTileMatrix &M, double *v, double *part, int *status, int *info, const XgFactorStreams &fs);
double xg_trailing_flops(int nt, int ts, int k);
int xg_field_set_data(XgField *f, const double *x, const double *y, const double *z);
int xg_field_set_profiling(XgField *f, int on);

int xg_field_create(XgField **out, int N, int ts, const double *x, const double *y, int kernel, int metric);
void xg_field_destroy(XgField *f);
int xg_field_set_z(XgField *f, const double *z);
int xg_field_loglik(XgField *f, const double *theta, double *res, double *times);
int xg_field_zvg(XgField *f, const double *theta, const double *nrand, double *times);
int xg_field_loglik_grad(XgField *f, const double *theta, double *res, double *grad, double *times);
int xg_field_set_mixed(XgField *f, int band, int passes);
int xg_field_loglik_mixed(XgField *f, const double *theta, double *res, double *times);
void xg_mixed_destroy(XgMixed *m);
int xg_mixed_factor_dense(int n, const double *x, const double *y, const double *theta, int kernel, int metric, int ts,
                          int band, int passes, double *out);
double xg_digamma(double x);
void xg_field_collect_profile_mixed(XgField *f);
int xg_field_get_z(XgField *f, double *z, int n);
int xg_autotune_field(XgField **pf, const double *x, const double *y, const double *theta, int precision, double tol,
                      int *ts_out, int *band_out, double *report);
int xg_field_set_sliced(XgField *f);
int xg_field_loglik_sliced(XgField *f, const double *theta, double *res, double *times);
int xg_field_loglik_grad_sliced(XgField *f, const double *theta, double *res, double *grad, double *times);
void xg_sliced_destroy(XgSliced *s);
int xg_sliced_factor_dense(int n, const double *x, const double *y, const double *theta, int kernel, int metric,
                           int ts, double *out);

int xg_predict_create(XgPredict **out, int nmiss, int nobs, int ts);
void xg_predict_destroy(XgPredict *q);
int xg_predict_run(XgPredict *q, const double *theta, int kernel, int metric, const double *xm, const double *ym,
                   const double *xo, const double *yo, const double *zobs, const double *zactual, double *zmiss,
                   double *mse, double *mse_parts);

/* MLOE / MMOM workspace (assess.cu): the two observed-set factors and five
 * R-layout right-hand-side stores (one row per missing point): k_a -> A,
 * k_t -> U, k_t -> T, W, V. */
struct XgAssess {
    int nmiss = 0, nobs = 0, ts = 0, nt = 0, mt = 0;
    XgTileMatrix Ca, Ct;
    double *R[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    CUtensorMap mR[5];
    double *xo = nullptr, *yo = nullptr, *xm = nullptr, *ym = nullptr;
    double *terms = nullptr, *part = nullptr;
    int *status = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t ev_panel = nullptr, ev_upd = nullptr;
};

int xg_field_fisher(XgField *f, const double *theta, int kernel, double *F, double *seconds);
int xg_small_spd_inverse(int n, const double *A, double *inv);
int xg_assess_create(XgAssess **out, int nmiss, int nobs, int ts);
void xg_assess_destroy(XgAssess *q);
int xg_assess_run(XgAssess *q, const double *truth, const double *est, int kernel, int metric, const double *xm,
                  const double *ym, const double *xo, const double *yo, double *mloe, double *mmom, double *terms,
                  double *times);

int xg_covariance_dense(int n, const double *x, const double *y, const double *theta, int kernel, int metric, int ts,
                        int factor, double *out);
int xg_matern_pairs_host(int n, const double *x1, const double *y1, const double *x2, const double *y2,
                         const double *theta, int kernel, int metric, double *out);
int xg_bessel_knu_host(int n, const double *nu, const double *x, double *out);

#endif
