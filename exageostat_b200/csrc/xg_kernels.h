/*
 * Internal interface between the host engine and the CUDA kernels.
 */
#ifndef EXAGEOSTAT_B200_KERNELS_H
#define EXAGEOSTAT_B200_KERNELS_H

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "xg_temme.h"

/* Tile sizes are multiples of 128 up to XG_MAX_TS: the panel TRSM stages
 * 32 x ts doubles in shared memory. */
#define XG_MAX_TS 512

/* A lower-tile matrix on the device (see dense_fp64.cu for the layout).
 * band == 0: every lower tile is FP64 in data, packed (xg_tile_index).
 * band  > 0: banded mixed precision -- data holds only the FP64 band tiles
 * (0 <= i - j < band, compact: slot j * band + (i - j)), data32 the FP32
 * off-band tiles (compact, xg_slot32). */
struct XgTileArgs {
    double *data;
    int ts; /* tile size */
    int nt; /* tiles per side */
    int band = 0;
    float *data32 = nullptr;
    long long tile_off = 0; /* first tile of this matrix inside a shared TMA tensor (batches) */
    /* band == 0 only: restricts the DMMA trailing update to the targets
     * 0 <= i - j < band_targets (the others go to the INT8-sliced kernel) */
    int band_targets = 0;
    /* optional: ts x 32 doubles receiving the inverses of the 32 x 32
     * diagonal blocks of the current panel's L_kk (written by
     * xg_launch_potrf_tiled); with it the panel TRSM applies them as DMMA
     * products instead of a serial substitution */
    double *dinv = nullptr;
};

__host__ __device__ inline long long xg_slot64(const XgTileArgs &T, int i, int j)
{
    if (T.band) return (long long)j * T.band + (i - j);
    return (long long)j * T.nt - (long long)j * (j - 1) / 2 + (i - j);
}

/* off-band tile (i, j), i - j >= band: column j holds nt - j - band tiles */
__host__ __device__ inline long long xg_slot32(int i, int j, int nt, int band)
{
    const long long M = nt - band;
    return (long long)j * M - (long long)j * (j - 1) / 2 + (i - j - band);
}

__host__ __device__ inline long long xg_num_offband_tiles(int nt, int band)
{
    const long long M = nt - band;
    return M > 0 ? M * (M + 1) / 2 : 0;
}

/* Matern parameters of one covariance evaluation.  con = sigma^2 /
 * (2^(nu-1) Gamma(nu)) is computed on the host exactly as core_zcmg.c:976-978;
 * half_integer = 0, 1, 2 selects the closed form for nu = 0.5, 1.5, 2.5
 * (exact match of nu), -1 the general Bessel path. */
struct XgMaternParams {
    double sigma2;
    double beta;
    double nu;
    double nugget; /* tau^2, added on the zero-distance branch only */
    double con;
    int half_integer;
    /* bivariate parsimonious Matern (kernel 2): rows and columns interleave
     * the two variables of each location (index 2 l + v); sigma2, nu, con
     * above are variable 0's, these variable 1's and the cross block's
     * (core_zcmg.c:1628-1651) */
    int bivariate;
    double sigma2b, nu2, con2, nu12, con12, cross0;
    /* scales of variable 1 and of the cross covariance (beta is variable 0's):
     * all three equal beta for the parsimonious kernel; the flexible kernel
     * (kernel 3, core_zcmg.c:1514-1580) has one per component */
    double beta2, beta12;
    /* Temme's order constants of nu (univariate kernels, general nu) */
    XgTemme tm;
};

/* One field of a batch of independent fields sharing one tile store. */
struct XgBField {
    long long tile_off; /* first packed tile of the field in the batch store */
    long long vec_off;  /* first entry of its vectors (x, y, z, v); a multiple of ts */
    long long part_off; /* first entry of its partial sums (2 nt) */
    long long sched_off; /* first of its scheduler counters (nt + 2 lower tiles) */
    int N, nt;
    int kernel, pad_;
    XgMaternParams p;   /* this evaluation's parameters */
};

/* Device-resident tile scheduler of a batch (xg_batch_sched_kernel).  The
 * task list holds every POTRF(k), TRSM(i, k) and update (i, j) <- step k of
 * every field in one topological order; persistent CTAs take tasks in list
 * order (one atomic counter), wait (bounded) on the task's dependency
 * counters, run it and publish its completion.  Per field, at sched_off:
 *   pdone[k]            POTRF(k) done
 *   tdone[tile (i, k)]  TRSM(i, k) done
 *   ucount[tile (i, j)] updates applied to tile (i, j) (final at min(i, j))
 * Dependencies: POTRF(k) <- ucount(k, k) = k; TRSM(i, k) <- pdone(k),
 * ucount(i, k) = k; update (i, j, k) <- tdone(i, k), tdone(j, k),
 * ucount(i, j) = k (the updates of a tile are applied in k order). */
#define XG_TASK_POTRF 0
#define XG_TASK_TRSM 1
#define XG_TASK_GEMM 2
struct XgSched {
    const int4 *tasks;         /* x = type | field << 2, y = i, z = j, w = k */
    long long ntasks;
    unsigned long long *next;  /* index of the next task to take */
    int *abort;                /* set after a wait that timed out: no CTA takes another task */
    int *cnt;                  /* the counters of every field */
    double *dinv;              /* per CTA, ts x 32: the inverted diagonal blocks of its TRSM task's L_kk */
};

/* The fields taking part in one batched launch and the CTA ranges they own. */
struct XgBStep {
    const int *fields;          /* nact field indices */
    const long long *blk_start; /* nact + 1 prefix sums of CTAs */
    int nact;
};

/* field owning CTA `bid` of a batched launch, and the CTA index within it */
__device__ inline int xg_batch_resolve(const XgBStep &S, long long bid, long long *local)
{
    int lo = 0, hi = S.nact - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (S.blk_start[mid] <= bid)
            lo = mid;
        else
            hi = mid - 1;
    }
    *local = bid - S.blk_start[lo];
    return S.fields[lo];
}

/* (i, j) of packed lower tile t of an nt x nt tile grid */
__host__ __device__ inline int2 xg_tile_decode(long long t, int nt)
{
    int j = 0;
    while (t >= nt - j) {
        t -= nt - j;
        ++j;
    }
    return make_int2(j + (int)t, j);
}

cudaError_t xg_kernels_configure();
size_t xg_potrf_smem_bytes(int ts);
size_t xg_trsm_smem_bytes(int ts);
size_t xg_gemm_smem_bytes();

void xg_launch_gen(const XgTileArgs &T, const int2 *tile_ij, long long ntiles, const double *xr, const double *yr,
                   const double *xc, const double *yc, int n_rows, int n_cols, const XgMaternParams &p, int metric,
                   int identity_pad, cudaStream_t st);
void xg_launch_potrf_diag(const XgTileArgs &T, int k, double *v, double *part_logdet, double *part_dot, int with_rhs,
                          int *status, int *info, cudaStream_t st);
void xg_launch_trsm_panel(const XgTileArgs &T, int k, double *v, int with_rhs, const int *status, cudaStream_t st,
                          int i1 = -1);
/* POTRF(k, k) with the fused log-det and solve, by 128 x 128 sub-blocks on
 * several CTAs (map: the TMA view of the tile store); fills T.dinv too */
void xg_launch_potrf_tiled(const CUtensorMap &map, const XgTileArgs &T, int k, double *v, double *part_logdet,
                           double *part_dot, int with_rhs, int *status, int *info, cudaStream_t st);
int xg_potrf_tiled_launches(int ts);
void xg_launch_syrk_gemm(const CUtensorMap &map, const XgTileArgs &T, int k, int *status, cudaStream_t st,
                         int part = 0);

/* mixed.cu: banded mixed precision */
struct XgMixedMaps {
    CUtensorMap p64;           /* FP64 panel copy, boxes 128 x 16 (DMMA band targets) */
    CUtensorMap ahi, bhi;      /* TF32 "hi" panel, boxes 128 x 32 and 256 x 32 (FP32) */
    CUtensorMap alo, blo;      /* TF32 "lo" panel */
};
cudaError_t xg_mixed_kernels_configure();
void xg_launch_gen_mixed(const XgTileArgs &T, const int2 *tile_ij, long long ntiles, const double *x, const double *y,
                         int n, const XgMaternParams &p, int metric, cudaStream_t st);
/* panel TRSM of column k by 128-column blocks (TMA-fed DMMA GEMMs and in-block
 * solves with the inverted 32 x 32 diagonal blocks in T.dinv); ts a multiple of 128 */
void xg_launch_trsm_gemm(const CUtensorMap &map, const XgTileArgs &T, int k, double *v, int with_rhs, int *status,
                         cudaStream_t st);
void xg_launch_trsm_panel32(const XgTileArgs &T, int k, double *v, int with_rhs, const int *status, cudaStream_t st);
void xg_launch_panel_prep(const XgTileArgs &T, int k, double *p64, float *phi, float *plo, int passes,
                          const int *status, cudaStream_t st);
void xg_launch_band_gemm(const CUtensorMap &p64map, const XgTileArgs &T, int k, int part, int *status,
                         cudaStream_t st);
void xg_launch_offband_gemm(const XgMixedMaps &maps, const XgTileArgs &T, int k, int part, int passes, int sm_count,
                            int *status, cudaStream_t st);
/* sliced.cu: FP64 tiles, trailing updates on INT8 tensor cores (four digit slices), left-looking.
 * One launch of xg_sliced_left_kernel computes, for each output tile, C (+)= sign sum_k A_k B_k^T
 * over panel chunks k, with A_k, B_k read from digit stores:
 *   XG_SL_FACTOR : column col of the Cholesky factor, chunks k0 <= k < k1: L(i,col) -= sum L(i,k) L(col,k)^T
 *   XG_SL_INVERSE: column col of X = L^-T (X(a,b) at slot (b,a)): X(a,col) -= sum_{a<=c<col} X(a,c) L(col,c)^T
 *   XG_SL_SYRK   : S = X X^T into the lower tiles: S(a,b) = sum_{c>=a} X(a,c) X(b,c)^T */
#define XG_SL_FACTOR 0
#define XG_SL_INVERSE 1
#define XG_SL_SYRK 2
struct XgSlTask {
    int mode;
    int col;       /* target column (factor, inverse) */
    int k0, k1;    /* chunk window */
    double sign;   /* -1: C -= sum; +1: C += sum */
    int overwrite; /* C = sign sum (C is not read) */
};
cudaError_t xg_sliced_kernels_configure();
void xg_launch_slice_panel(const XgTileArgs &T, int k, int row_mode, int8_t *dig, double *scale, long long plane,
                           const int *status, cudaStream_t st);
void xg_launch_sliced(const CUtensorMap &map_a, const CUtensorMap &map_b, const double *scale_a,
                      const double *scale_b, const XgTileArgs &T, const XgSlTask &S, int plane_rows, int max_ctas,
                      int *status, cudaStream_t st);

void xg_launch_finalize(const double *part_logdet, const double *part_dot, int nt, int N, double *out,
                        const int *status, const int *info, cudaStream_t st);

/* batched fields (one launch per tile step covering every active field) */
void xg_launch_batch_gen(const XgTileArgs &base, const XgBField *F, const XgBStep &S, long long blocks,
                         const double *x, const double *y, int metric, cudaStream_t st);
void xg_launch_batch_potrf(const XgTileArgs &base, const XgBField *F, const XgBStep &S, int k, double *v, double *part,
                           int *status, int *info, cudaStream_t st);
void xg_launch_batch_trsm(const XgTileArgs &base, const XgBField *F, const XgBStep &S, long long blocks, int k,
                          double *v, const int *status, cudaStream_t st);
void xg_launch_batch_gemm(const CUtensorMap &map, const XgTileArgs &base, const XgBField *F, const XgBStep &S,
                          long long blocks, int k, int *status, cudaStream_t st);
void xg_launch_batch_finalize(const XgBField *F, int nfields, const double *part, double *out, cudaStream_t st);
/* the whole batched factorisation (with the fused log-det and solve) in one
 * persistent launch of `ctas` CTAs driven by the task list of `sch` */
void xg_launch_batch_sched(const CUtensorMap &map, const XgTileArgs &base, const XgBField *F, const XgSched &sch,
                           int ctas, double *v, double *part, int *status, cudaStream_t st);

/* solve.cu */
void xg_launch_trmv_lower(const XgTileArgs &T, const double *e, double *z, const int *status, cudaStream_t st);
void xg_launch_trsv_lower_t_step(const XgTileArgs &T, int k, double *v, const int *status, cudaStream_t st);
void xg_launch_predict_cross(const double *xm, const double *ym, int nmiss, const double *xo, const double *yo,
                             int nobs, const double *alpha, const XgMaternParams &p, int metric, double *zmiss,
                             cudaStream_t st);
void xg_launch_mse(const double *zactual, const double *zmiss, int nmiss, double *out, cudaStream_t st);
void xg_launch_matern_pairs(const double *x1, const double *y1, const double *x2, const double *y2, int n,
                            const XgMaternParams &p, int metric, double *out, cudaStream_t st);

void xg_launch_bessel(const double *nu, const double *x, int n, double *out, cudaStream_t st);

/* gradient_fp64.cu */
cudaError_t xg_gradient_kernels_configure();
void xg_launch_inverse_factor(const CUtensorMap &mapX, const CUtensorMap &mapL, double *X, const double *L, int nt,
                              int ts, int *status, cudaStream_t st);
void xg_launch_inverse_syrk(const CUtensorMap &mapX, double *S, int nt, int ts, int *status, cudaStream_t st);
/* X = 0 with identity diagonal tiles; step K of X L^T = I: X(I, K) <- X(I, K) L_KK^-T for I <= K */
void xg_launch_identity_x(double *X, int nt, int ts, cudaStream_t st);
void xg_launch_xtrsm(double *X, const double *L, int nt, int ts, int K, int *status, cudaStream_t st);
void xg_launch_rhs_forward_solve(const CUtensorMap &mapR, double *R, int mt, const CUtensorMap &mapL, const double *L,
                                 int nt, int ts, int *status, cudaStream_t st);
void xg_launch_rhs_backward_solve(const CUtensorMap &mapR, double *R, int mt, const CUtensorMap &mapLT,
                                  const double *LT, int nt, int ts, int *status, cudaStream_t st);
void xg_launch_rhs_tri_product(const CUtensorMap &mapA, const CUtensorMap &mapB, double *C, int mt, int nt, int ts,
                               int *status, cudaStream_t st);
void xg_launch_dense_gemm_nt(const CUtensorMap &mapA, const CUtensorMap &mapB, double *C, int nt, int ts, int *status,
                             cudaStream_t st);
long long xg_grad_contract_blocks(long long ntiles, int ts);
void xg_launch_grad_contract(const double *S, const int2 *tile_ij, long long ntiles, int nt, int ts, const double *x,
                             const double *y, const double *alpha, int N, const XgMaternParams &mp, int kernel,
                             int metric, double dlogcon, double *part, double *out, cudaStream_t st);

/* assess.cu (Fisher information, MLOE / MMOM) */
void xg_launch_cross_gen_r(double *D, int mt, int nt, int ts, const double *xm, const double *ym, int nmiss,
                           const double *xo, const double *yo, int nobs, const XgMaternParams &p, int metric,
                           cudaStream_t st);
void xg_launch_tile_transpose(double *D, long long ntiles, int ts, cudaStream_t st);
void xg_launch_mloe_terms(const double *A, const double *U, const double *T, const double *V, int mt, int nt, int ts,
                          int nmiss, double sigma2_t, double sigma2_a, double *terms, cudaStream_t st);
void xg_launch_sym_full(const double *S, double *F, int nt, int ts, cudaStream_t st);
void xg_launch_dsigma_full(double *D, int nt, int ts, const double *x, const double *y, int N,
                           const XgMaternParams &p, double dlogcon, int metric, int which, cudaStream_t st);
void xg_launch_fisher_trace(const double *const g[4], int np, int nt, int ts, int N, double *part, int nctas,
                            cudaStream_t st);

#endif
