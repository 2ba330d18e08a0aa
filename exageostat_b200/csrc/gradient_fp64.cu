/*
 * Gradient of the exact Matern log-likelihood (FP64), on sm_100a.
 *
 *   d loglik / d theta_p = 1/2 alpha^T (dSigma/dtheta_p) alpha - 1/2 tr(Sigma^-1 dSigma/dtheta_p)
 *                        = sum_{R,C} W_RC (dSigma/dtheta_p)_RC,   W = (alpha alpha^T - Sigma^-1) / 2,
 * alpha = Sigma^-1 z.  The reference has no gradient (NLopt's derivative-free
 * BOBYQA ignores grad, examples/synthetic_dmle_test.c:140-142); its dSigma/dtheta
 * element kernels (core_dcmg_matern_dsigma_square / _dbeta / _dnu,
 * exageostat_exact/cpu_core/compute/core_zcmg.c:315-488) are the math spec.
 *
 * After the forward factorisation (Sigma = L L^T in the lower tiles):
 *   1. alpha = L^-T (L^-1 z) with the backward tile solve (solve.cu).
 *   2. X = L^-T, upper triangular, by the right-looking blocked solve
 *      X L^T = I: per tile column K, X_IK = B_IK L_KK^-T (I <= K, panel TRSM
 *      on row strips), then B_IK' -= X_IK L_K'K^T (K' > K) on the FP64 tensor
 *      cores.  X_IK is stored row-major at packed slot (K, I) of a second
 *      lower-tile buffer, so both GEMM operands stay K-major for TMA.
 *   3. Sigma^-1 lower = X X^T: S_IJ = sum_{K >= I} X_IK X_JK^T, a K-looped
 *      DMMA SYRK written over the factor.
 *   4. One fused pass over the lower tiles of S generates dSigma/dtheta_p on
 *      the fly (never stored) and contracts it with W.
 * Steps 2 and 3 are N^3/3 flops each (TRTRI- and LAUUM-class), so a gradient
 * costs about two extra factorisations.
 */
#include <math.h>
#include <stdint.h>

#include "kbessel.cuh"
#include "xg_common.cuh"
#include "xg_kernels.h"
#include "xg_matern.cuh"

/* ========================================================================== */
/* Generalised tile GEMM: C (+)= -/+ sum_q A_q B_q^T over 128 x 128 blocks    */
/* ========================================================================== */

#define XG_TG_BM 128
#define XG_TG_BK 16
#define XG_TG_STAGES 4
#define XG_TG_THREADS 256
#define XG_TG_STAGE_BYTES (2 * XG_TG_BM * XG_TG_BK * 8)

/* modes.  "R layout": an mt x nt grid of tiles whose tile (R, K) sits at
 * slot K * mt + R (right-hand sides stored transposed, one row per
 * right-hand side). */
#define XG_TG_XUPDATE 1 /* step K of X L^T = I: slot(K', I) of X -= X_slot(K, I) L_slot(K', K)^T */
#define XG_TG_SYRKX 2   /* S_IJ = sum_{K >= I} X_slot(K, I) X_slot(K, J)^T, written to C storage */
#define XG_TG_RFWD 3    /* step K of Y L^T = B (R layout): B(R, K') -= Y(R, K) L_slot(K', K)^T, K' > K */
#define XG_TG_RTRI 4    /* C(R, I) = sum_{K >= I} A(R, K) B_slot(K, I)^T (R layout, B lower-tile packed) */
#define XG_TG_DENSE 5   /* full nt x nt tiles (slot A nt + B): C(A, B) = sum_K A(A, K) B(B, K)^T */
#define XG_TG_RBWD 6    /* step K of Z L = B (R layout), B holding L's tiles transposed in place:
                           B(R, K') -= Z(R, K) B_slot(K, K')^T, K' < K */

struct XgTileGemmJob {
    int c_slot;  /* packed slot of the output tile */
    int a_slot0; /* slot of the first A operand tile */
    int b_slot0;
    int ntiles_k; /* number of K tiles summed */
    int k_step_a; /* slot stride between successive A tiles */
    int k_step_b;
    bool skip;
};

__device__ inline XgTileGemmJob xg_tg_decode(int mode, long long job, int nt, int K, int mt)
{
    XgTileGemmJob j;
    j.skip = false;
    if (mode == XG_TG_RFWD) {
        const int R = (int)(job % mt), Kp = K + 1 + (int)(job / mt);
        j.c_slot = Kp * mt + R;
        j.a_slot0 = K * mt + R;
        j.b_slot0 = (int)xg_tile_index(Kp, K, nt);
        j.ntiles_k = 1;
        j.k_step_a = j.k_step_b = 0;
    } else if (mode == XG_TG_RTRI) {
        const int R = (int)(job % mt), I = (int)(job / mt);
        j.c_slot = I * mt + R;
        j.a_slot0 = I * mt + R;
        j.k_step_a = mt;
        /* slot(K, I) for K = I.. nt-1 are consecutive in the packed column I */
        j.b_slot0 = (int)xg_tile_index(I, I, nt);
        j.k_step_b = 1;
        j.ntiles_k = nt - I;
    } else if (mode == XG_TG_RBWD) {
        const int R = (int)(job % mt), Kp = (int)(job / mt);
        j.c_slot = Kp * mt + R;
        j.a_slot0 = K * mt + R;
        j.b_slot0 = (int)xg_tile_index(K, Kp, nt);
        j.ntiles_k = 1;
        j.k_step_a = j.k_step_b = 0;
    } else if (mode == XG_TG_DENSE) {
        const int A = (int)(job / nt), B = (int)(job % nt);
        j.c_slot = A * nt + B;
        j.a_slot0 = A * nt;
        j.b_slot0 = B * nt;
        j.k_step_a = j.k_step_b = 1;
        j.ntiles_k = nt;
    } else if (mode == XG_TG_XUPDATE) {
        const int width = K + 1; /* I in [0, K] */
        const int I = (int)(job % width), Kp = K + 1 + (int)(job / width);
        j.c_slot = (int)xg_tile_index(Kp, I, nt);
        j.a_slot0 = (int)xg_tile_index(K, I, nt);
        j.b_slot0 = (int)xg_tile_index(Kp, K, nt);
        j.ntiles_k = 1;
        j.k_step_a = j.k_step_b = 0;
    } else {
        int I, J;
        xg_pair_decode(job, &I, &J); /* I >= J */
        j.c_slot = (int)xg_tile_index(I, J, nt);
        /* slot(K, I) for K = I.. nt-1 are consecutive in the packed column I */
        j.a_slot0 = (int)xg_tile_index(I, I, nt);
        j.b_slot0 = (int)xg_tile_index(I, J, nt);
        j.ntiles_k = nt - I;
        j.k_step_a = 1;
        j.k_step_b = 1;
    }
    return j;
}

__global__ void __launch_bounds__(XG_TG_THREADS, 1)
    xg_tile_gemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB,
                        double *__restrict__ Cbase, int nt, int ts, int mode, int K, int mt, int *status)
{
    extern __shared__ __align__(1024) unsigned char xg_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)xg_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + XG_TG_STAGES * XG_TG_STAGE_BYTES);
    uint64_t *empty = full + XG_TG_STAGES;
    const int bpt = ts / XG_TG_BM;
    const long long job = blockIdx.x / (bpt * bpt);
    const int blk = blockIdx.x % (bpt * bpt);
    const int bi = blk / bpt, bj = blk % bpt;
    const XgTileGemmJob J = xg_tg_decode(mode, job, nt, K, mt);
    /* S output is symmetric: skip the strictly upper 128-blocks of diagonal tiles */
    bool diag_upper = false;
    if (mode == XG_TG_SYRKX) {
        int I, Jc;
        xg_pair_decode(job, &I, &Jc);
        diag_upper = (I == Jc && bj > bi);
    }
    if (xg_cta_should_skip(status, diag_upper)) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < XG_TG_STAGES; ++s) {
            xg_mbar_init(&full[s], 1);
            xg_mbar_init(&empty[s], 8);
        }
        xg_fence_barrier_init();
    }
    __syncthreads();
    const int kper = ts / XG_TG_BK;
    const int KT = J.ntiles_k * kper;
    auto issue = [&](int q, int s) {
        const int kt = q / kper, kk = (q % kper) * XG_TG_BK;
        const int ya = (J.a_slot0 + kt * J.k_step_a) * ts + bi * XG_TG_BM;
        const int yb = (J.b_slot0 + kt * J.k_step_b) * ts + bj * XG_TG_BM;
        unsigned char *sa = smem + s * XG_TG_STAGE_BYTES;
        xg_mbar_arrive_expect_tx(&full[s], XG_TG_STAGE_BYTES);
        xg_tma_load_2d(sa, &mapA, kk, ya, &full[s]);
        xg_tma_load_2d(sa + XG_TG_BM * XG_TG_BK * 8, &mapB, kk, yb, &full[s]);
    };
    int issued = 0;
    if (tid == 0) {
        xg_prefetch_tensormap(&mapA);
        xg_prefetch_tensormap(&mapB);
        for (; issued < XG_TG_STAGES && issued < KT; ++issued) issue(issued, issued);
    }
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, tq = lane & 3;
    double *C = Cbase + (long long)J.c_slot * ts * ts + (long long)(bi * XG_TG_BM) * ts + bj * XG_TG_BM;
    double acc[4][4][4];
    const bool subtract = (mode == XG_TG_XUPDATE || mode == XG_TG_RFWD || mode == XG_TG_RBWD);
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                double cx = 0.0, cy = 0.0;
                if (subtract) {
                    const int r = wm * 64 + mi * 16 + g + 8 * h;
                    const int c = wn * 32 + ni * 8 + 2 * tq;
                    const double2 cv = *reinterpret_cast<const double2 *>(C + (long long)r * ts + c);
                    cx = -cv.x;
                    cy = -cv.y;
                }
                acc[mi][ni][2 * h] = cx;
                acc[mi][ni][2 * h + 1] = cy;
            }
    bool ok = true;
    for (int kb = 0; kb < KT; ++kb) {
        const int s = kb % XG_TG_STAGES;
        if (!xg_mbar_wait(&full[s], (kb / XG_TG_STAGES) & 1)) {
            ok = false;
            break;
        }
        const unsigned char *sa = smem + s * XG_TG_STAGE_BYTES;
        const unsigned char *sb = sa + XG_TG_BM * XG_TG_BK * 8;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int chunk = 2 * tq + half;
            double2 b[4];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int r = wn * 32 + ni * 8 + g;
                b[ni] = *(const double2 *)(sb + (r << 7) + ((chunk ^ (r & 7)) << 4));
            }
#pragma unroll
            for (int mi = 0; mi < 4; ++mi) {
                const int r = wm * 64 + mi * 16 + g;
                const double2 a0 = *(const double2 *)(sa + (r << 7) + ((chunk ^ (r & 7)) << 4));
                const double2 a1 = *(const double2 *)(sa + ((r + 8) << 7) + ((chunk ^ ((r + 8) & 7)) << 4));
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) {
                    xg_dmma_16x8x4(acc[mi][ni][0], acc[mi][ni][1], acc[mi][ni][2], acc[mi][ni][3], a0.x, a1.x,
                                   b[ni].x);
                    xg_dmma_16x8x4(acc[mi][ni][0], acc[mi][ni][1], acc[mi][ni][2], acc[mi][ni][3], a0.y, a1.y,
                                   b[ni].y);
                }
            }
        }
        __syncwarp();
        if (lane == 0) xg_mbar_arrive(&empty[s]);
        if (tid == 0 && issued < KT) {
            if (xg_mbar_wait(&empty[s], (kb / XG_TG_STAGES) & 1)) {
                issue(issued, s);
                ++issued;
            } else {
                ok = false;
            }
        }
        __syncwarp();
        if (!ok) break;
    }
    if (!ok) {
        atomicOr(status, XG_ST_TIMEOUT);
        if (tid == 0)
            for (int q = (issued > XG_TG_STAGES ? issued - XG_TG_STAGES : 0); q < issued; ++q)
                xg_mbar_wait(&full[q % XG_TG_STAGES], (q / XG_TG_STAGES) & 1);
        return;
    }
    const double sgn = subtract ? -1.0 : 1.0;
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = wm * 64 + mi * 16 + g + 8 * h;
                const int c = wn * 32 + ni * 8 + 2 * tq;
                *reinterpret_cast<double2 *>(C + (long long)r * ts + c) =
                    make_double2(sgn * acc[mi][ni][2 * h], sgn * acc[mi][ni][2 * h + 1]);
            }
}

/* ========================================================================== */
/* Right-side TRSM on the row of X tiles of step K: X_IK <- X_IK L_KK^-T      */
/* ========================================================================== */

#define XG_XT_THREADS 512
#define XG_XT_SR 32

/* mt == 0: the tiles X_IK, I <= K, at slot (K, I) (inverse factor);
 * mt  > 0: the tiles (R, K), R < mt, of an R-layout matrix (right-hand sides).
 * UPPER: the diagonal tile holds U = L_KK^T (a factor transposed in place)
 * and the solve is B <- B U^-T = B L_KK^-1, by 32-column blocks from the
 * right (backward substitution). */
template <bool UPPER>
__global__ void __launch_bounds__(XG_XT_THREADS) xg_xtrsm_kernel(double *__restrict__ X, const double *__restrict__ Lt,
                                                                 int nt, int ts, int K, int mt, const int *status)
{
    const int LDS = ts + 4;
    extern __shared__ __align__(16) double xg_smem_d[];
    double *S = xg_smem_d;             /* [SR][LDS] */
    double *LD = S + XG_XT_SR * LDS;   /* [32][33] */
    if (xg_cta_should_skip(status)) return;
    const int strips = ts / XG_XT_SR;
    const int I = blockIdx.x / strips, strip = blockIdx.x % strips; /* I in [0, K] */
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tq = lane & 3;
    const long long bslot = mt > 0 ? (long long)K * mt + I : xg_tile_index(K, I, nt);
    double *B = X + bslot * (long long)ts * ts + (long long)strip * XG_XT_SR * ts;
    const double *L = Lt + xg_tile_index(K, K, nt) * (long long)ts * ts;
    for (int idx = tid; idx < XG_XT_SR * ts; idx += blockDim.x) {
        const int r = idx / ts, c = idx - r * ts;
        S[r * LDS + c] = B[(long long)r * ts + c];
    }
    for (int blk = 0; blk < ts / 32; ++blk) {
        const int cb = UPPER ? ts - 32 * (blk + 1) : 32 * blk;
        for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
            const int r = idx >> 5, c = idx & 31;
            LD[r * 33 + c] = L[(long long)(cb + r) * ts + cb + c];
        }
        __syncthreads();
        if (warp == 0) {
            double row[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) row[j] = S[lane * LDS + cb + j];
            if (UPPER) {
#pragma unroll
                for (int j = 31; j >= 0; --j) {
                    double s = row[j];
#pragma unroll
                    for (int q = j + 1; q < 32; ++q) s -= row[q] * LD[j * 33 + q];
                    row[j] = s / LD[j * 33 + j];
                }
            } else {
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    double s = row[j];
#pragma unroll
                    for (int q = 0; q < j; ++q) s -= row[q] * LD[j * 33 + q];
                    row[j] = s / LD[j * 33 + j];
                }
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) S[lane * LDS + cb + j] = row[j];
        }
        __syncthreads();
        /* the solved block's contribution to the columns still to solve:
         * right of it (lower) or left of it (upper) */
        const int ngrp = UPPER ? cb / 32 : (ts - cb - 32) / 32;
        for (int grp = warp; grp < ngrp; grp += XG_XT_THREADS / 32) {
            const int c0 = UPPER ? grp * 32 : cb + 32 + grp * 32;
            double acc[2][4][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;
#pragma unroll
            for (int p0 = 0; p0 < 32; p0 += 4) {
                double a[2][2], b[4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    a[mi][0] = S[(mi * 16 + g) * LDS + cb + p0 + tq];
                    a[mi][1] = S[(mi * 16 + g + 8) * LDS + cb + p0 + tq];
                }
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) b[ni] = __ldg(L + (long long)(c0 + ni * 8 + g) * ts + cb + p0 + tq);
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
                        xg_dmma_16x8x4(acc[mi][ni][0], acc[mi][ni][1], acc[mi][ni][2], acc[mi][ni][3], a[mi][0],
                                       a[mi][1], b[ni]);
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        double *ps = S + (mi * 16 + g + 8 * h) * LDS + c0 + ni * 8 + 2 * tq;
                        ps[0] -= acc[mi][ni][2 * h];
                        ps[1] -= acc[mi][ni][2 * h + 1];
                    }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < XG_XT_SR * ts; idx += blockDim.x) {
        const int r = idx / ts, c = idx - r * ts;
        B[(long long)r * ts + c] = S[r * LDS + c];
    }
}

/* X starts as the identity on its diagonal tiles and zero elsewhere. */
__global__ void xg_identity_diag_kernel(double *X, int nt, int ts)
{
    const int K = blockIdx.y;
    double *T = X + xg_tile_index(K, K, nt) * (long long)ts * ts;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < ts; r += gridDim.x * blockDim.x) T[(long long)r * ts + r] = 1.0;
}

/* ========================================================================== */
/* Fused dSigma/dtheta generation and contraction with W                      */
/* ========================================================================== */

struct XgGradParams {
    double sigma2, beta, nu, nugget, con, dlogcon;
    int kernel; /* 0 Matern, 1 Matern + nugget */
    int metric;
};

#define XG_GC_ROWS 8
/* one CTA: XG_GC_ROWS rows of one lower tile of S; partial sums of the four
 * parameters' contractions go to part[4 * blockIdx.x + p] */
__global__ void __launch_bounds__(256) xg_grad_contract_kernel(const double *__restrict__ S,
                                                               const int2 *__restrict__ tile_ij, int nt, int ts,
                                                               const double *__restrict__ x,
                                                               const double *__restrict__ y,
                                                               const double *__restrict__ alpha, int N,
                                                               XgGradParams p, double *__restrict__ part)
{
    __shared__ double red[4][8];
    const int strips = ts / XG_GC_ROWS;
    const long long t = blockIdx.x / strips;
    const int strip = blockIdx.x % strips;
    const int2 ij = tile_ij[t];
    const double *tile = S + t * (long long)ts * ts;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int rr = 0; rr < XG_GC_ROWS; ++rr) {
        const int r = strip * XG_GC_ROWS + rr;
        const int R = ij.x * ts + r;
        if (R >= N) break;
        const double xr = x[R], yr = y[R], ar = alpha[R];
        for (int c = threadIdx.x; c < ts; c += blockDim.x) {
            const int Cc = ij.y * ts + c;
            if (Cc >= N || Cc > R) continue;
            const double w = (Cc == R ? 0.5 : 1.0) * (ar * alpha[Cc] - tile[(long long)r * ts + c]);
            const double d = xg_distance(xr, yr, x[Cc], y[Cc], p.metric);
            const double rd = d / p.beta;
            if (rd == 0.0) {
                acc[0] += w;                     /* dSigma/dsigma2 = 1 on the zero-distance branch */
                if (p.kernel == 1) acc[3] += w;  /* dSigma/dtau2 */
            } else {
                double m, ds, db, dn;
                xg_matern_grad(rd, p.nu, p.con, p.sigma2, p.beta, p.dlogcon, &m, &ds, &db, &dn);
                acc[0] += w * ds;
                acc[1] += w * db;
                acc[2] += w * dn;
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double v = acc[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
        part[4 * (long long)blockIdx.x + threadIdx.x] = v;
    }
}

/* deterministic final sum of the per-CTA partials */
__global__ void xg_grad_reduce_kernel(const double *part, long long nblocks, double *out)
{
    __shared__ double red[4][32];
    const int p = threadIdx.y; /* 4 x 32 threads */
    double v = 0.0;
    for (long long b = threadIdx.x; b < nblocks; b += 32) v += part[4 * b + p];
    red[p][threadIdx.x] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < 32; ++i) s += red[p][i];
        out[p] = s;
    }
}

/* ========================================================================== */
/* launchers                                                                  */
/* ========================================================================== */

size_t xg_tile_gemm_smem_bytes() { return (size_t)XG_TG_STAGES * XG_TG_STAGE_BYTES + 2 * XG_TG_STAGES * 8 + 1024; }
size_t xg_xtrsm_smem_bytes(int ts) { return ((size_t)XG_XT_SR * (ts + 4) + 32 * 33) * sizeof(double); }

cudaError_t xg_gradient_kernels_configure()
{
    cudaError_t e = cudaFuncSetAttribute(xg_tile_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)xg_tile_gemm_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_xtrsm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_xtrsm_smem_bytes(XG_MAX_TS));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(xg_xtrsm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)xg_xtrsm_smem_bytes(XG_MAX_TS));
}

/* X = L^-T into Xbuf (lower-tile layout, X_IK at slot (K, I)) */
void xg_launch_inverse_factor(const CUtensorMap &mapX, const CUtensorMap &mapL, double *X, const double *L, int nt,
                              int ts, int *status, cudaStream_t st)
{
    const size_t bytes = (size_t)xg_num_lower_tiles(nt) * ts * ts * sizeof(double);
    cudaMemsetAsync(X, 0, bytes, st);
    xg_identity_diag_kernel<<<dim3(1, nt), 256, 0, st>>>(X, nt, ts);
    const int bpt = ts / XG_TG_BM;
    for (int K = 0; K < nt; ++K) {
        xg_xtrsm_kernel<false><<<(K + 1) * (ts / XG_XT_SR), XG_XT_THREADS, xg_xtrsm_smem_bytes(ts), st>>>(X, L, nt, ts, K, 0,
                                                                                                 status);
        const long long jobs = (long long)(K + 1) * (nt - K - 1);
        if (jobs > 0)
            xg_tile_gemm_kernel<<<(unsigned)(jobs * bpt * bpt), XG_TG_THREADS, xg_tile_gemm_smem_bytes(), st>>>(
                mapX, mapL, X, nt, ts, XG_TG_XUPDATE, K, 0, status);
    }
}

/* S = X X^T (lower tiles) into Sbuf */
void xg_launch_identity_x(double *X, int nt, int ts, cudaStream_t st)
{
    cudaMemsetAsync(X, 0, (size_t)xg_num_lower_tiles(nt) * ts * ts * sizeof(double), st);
    xg_identity_diag_kernel<<<dim3(1, nt), 256, 0, st>>>(X, nt, ts);
}

void xg_launch_xtrsm(double *X, const double *L, int nt, int ts, int K, int *status, cudaStream_t st)
{
    xg_xtrsm_kernel<false><<<(K + 1) * (ts / XG_XT_SR), XG_XT_THREADS, xg_xtrsm_smem_bytes(ts), st>>>(X, L, nt, ts, K, 0,
                                                                                             status);
}

void xg_launch_inverse_syrk(const CUtensorMap &mapX, double *S, int nt, int ts, int *status, cudaStream_t st)
{
    const int bpt = ts / XG_TG_BM;
    const long long jobs = xg_num_lower_tiles(nt);
    xg_tile_gemm_kernel<<<(unsigned)(jobs * bpt * bpt), XG_TG_THREADS, xg_tile_gemm_smem_bytes(), st>>>(
        mapX, mapX, S, nt, ts, XG_TG_SYRKX, 0, 0, status);
}

long long xg_grad_contract_blocks(long long ntiles, int ts) { return ntiles * (ts / XG_GC_ROWS); }

void xg_launch_grad_contract(const double *S, const int2 *tile_ij, long long ntiles, int nt, int ts, const double *x,
                             const double *y, const double *alpha, int N, const XgMaternParams &mp, int kernel,
                             int metric, double dlogcon, double *part, double *out, cudaStream_t st)
{
    XgGradParams p;
    p.sigma2 = mp.sigma2;
    p.beta = mp.beta;
    p.nu = mp.nu;
    p.nugget = mp.nugget;
    p.con = mp.con;
    p.dlogcon = dlogcon;
    p.kernel = kernel;
    p.metric = metric;
    const long long blocks = xg_grad_contract_blocks(ntiles, ts);
    xg_grad_contract_kernel<<<(unsigned)blocks, 256, 0, st>>>(S, tile_ij, nt, ts, x, y, alpha, N, p, part);
    xg_grad_reduce_kernel<<<1, dim3(32, 4), 0, st>>>(part, blocks, out);
}

/* Y L^T = B for an R-layout right-hand side B (mt tile rows) and the lower
 * tile factor L, right-looking like the inverse factor: B is overwritten with
 * Y, the transpose of L^-1 B^T. */
void xg_launch_rhs_forward_solve(const CUtensorMap &mapR, double *R, int mt, const CUtensorMap &mapL, const double *L,
                                 int nt, int ts, int *status, cudaStream_t st)
{
    const int bpt = ts / XG_TG_BM;
    for (int K = 0; K < nt; ++K) {
        xg_xtrsm_kernel<false><<<mt * (ts / XG_XT_SR), XG_XT_THREADS, xg_xtrsm_smem_bytes(ts), st>>>(R, L, nt, ts, K, mt,
                                                                                            status);
        const long long jobs = (long long)mt * (nt - K - 1);
        if (jobs > 0)
            xg_tile_gemm_kernel<<<(unsigned)(jobs * bpt * bpt), XG_TG_THREADS, xg_tile_gemm_smem_bytes(), st>>>(
                mapR, mapL, R, nt, ts, XG_TG_RFWD, K, mt, status);
    }
}

/* Z L = B for an R-layout right-hand side B and a factor whose tiles were
 * transposed in place (LT: slot (i, j) holds L_ij^T), left-looking from the
 * last tile column: B is overwritten with Z, the transpose of L^-T B^T. */
void xg_launch_rhs_backward_solve(const CUtensorMap &mapR, double *R, int mt, const CUtensorMap &mapLT,
                                  const double *LT, int nt, int ts, int *status, cudaStream_t st)
{
    const int bpt = ts / XG_TG_BM;
    for (int K = nt - 1; K >= 0; --K) {
        xg_xtrsm_kernel<true><<<mt * (ts / XG_XT_SR), XG_XT_THREADS, xg_xtrsm_smem_bytes(ts), st>>>(R, LT, nt, ts, K,
                                                                                                 mt, status);
        const long long jobs = (long long)mt * K;
        if (jobs > 0)
            xg_tile_gemm_kernel<<<(unsigned)(jobs * bpt * bpt), XG_TG_THREADS, xg_tile_gemm_smem_bytes(), st>>>(
                mapR, mapLT, R, nt, ts, XG_TG_RBWD, K, mt, status);
    }
}

/* C(R, I) = sum_{K >= I} A(R, K) B_slot(K, I)^T: A and C R-layout (C != A),
 * B lower-tile packed.  With B = X (X_IK at slot (K, I)) this is C = A X^T;
 * with B holding the transposed tiles of a factor L, C = A L. */
void xg_launch_rhs_tri_product(const CUtensorMap &mapA, const CUtensorMap &mapB, double *C, int mt, int nt, int ts,
                               int *status, cudaStream_t st)
{
    const int bpt = ts / XG_TG_BM;
    const long long jobs = (long long)mt * nt;
    xg_tile_gemm_kernel<<<(unsigned)(jobs * bpt * bpt), XG_TG_THREADS, xg_tile_gemm_smem_bytes(), st>>>(
        mapA, mapB, C, nt, ts, XG_TG_RTRI, 0, mt, status);
}

/* C = A B^T on full nt x nt tile grids (tile (A, B) at slot A nt + B) */
void xg_launch_dense_gemm_nt(const CUtensorMap &mapA, const CUtensorMap &mapB, double *C, int nt, int ts, int *status,
                             cudaStream_t st)
{
    const int bpt = ts / XG_TG_BM;
    const long long jobs = (long long)nt * nt;
    xg_tile_gemm_kernel<<<(unsigned)(jobs * bpt * bpt), XG_TG_THREADS, xg_tile_gemm_smem_bytes(), st>>>(
        mapA, mapB, C, nt, ts, XG_TG_DENSE, 0, 0, status);
}
