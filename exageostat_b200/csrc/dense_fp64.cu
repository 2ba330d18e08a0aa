/*
 * FP64 kernels of the exact Matern log-likelihood path on sm_100a.
 *
 * Storage ("lower tile" layout): an N x N covariance is padded to
 * Np = nt * ts (the padding is the identity, so it adds log 1 = 0 to the
 * log-determinant and 0 to the quadratic form) and only the nt (nt + 1) / 2
 * lower tiles are kept, each ts x ts row-major, packed column by column
 * (xg_tile_index).  Row-major tiles make both operands of the trailing
 * update A_ij -= L_ik L_jk^T K-major, which is the layout TMA's 128-byte
 * swizzle and the DMMA fragments want.
 *
 * Reference steps these kernels replace (paths inside the reference tree):
 *   xg_gen_matern_kernel      core_dcmg / core_dcmg_nuggets
 *                             (exageostat_exact/cpu_core/compute/core_zcmg.c:963-994,
 *                              core_zcmg_nuggets.c:107-156), tile loop of
 *                             EXAGEOSTAT_MLE_dcmg_Tile_Async (runtime/starpu/codelets/codelet_zcmg.c:316-342)
 *   xg_potrf_diag_kernel      POTRF(k,k) of CHAMELEON_dpotrf_Tile (MLE_dexact.c:372) fused with
 *                             core_dmdet (cpu_core/compute/core_zmdet.c:50-59) and the diagonal block of
 *                             CHAMELEON_dtrsm_Tile on Z (MLE_dexact.c:391)
 *   xg_trsm_panel_kernel      TRSM(m,k) of dpotrf fused with the off-diagonal GEMV of the Z solve
 *   xg_syrk_gemm_kernel       SYRK/GEMM trailing updates of dpotrf (algorithm shown in-tree by
 *                             exageostat_exact/src/compute/psdportf.c:85-186 with an infinite band)
 *   xg_finalize_kernel        dot product (MLE_dexact.c:399) and the log-likelihood formula (:426)
 */
#include <math.h>
#include <stdint.h>

#include "kbessel.cuh"
#include "xg_common.cuh"
#include "xg_kernels.h"
#include "xg_matern.cuh"

/* ========================================================================== */
/* Matern tile generation                                                     */
/* ========================================================================== */

/* One CTA fills XG_GEN_ROWS rows of one tile; threads stride the columns so
 * the row-major stores and the column-location loads are coalesced. */
#define XG_GEN_ROWS 8
/* General-order univariate elements, grouped by K_nu branch: the lanes of a
 * warp would otherwise mix Temme's series, two trapezoid lengths and the
 * asymptotic series (unsorted locations) and run every branch they hold.
 * Each warp takes 32 columns x XG_GEN_ROWS rows at a time: every lane
 * computes r for its 8 elements and files them by branch in a per-warp
 * index list (ballots), the warp then evaluates the list branch by branch,
 * one element per lane, and stores its 8 x 32 block row by row (coalesced).
 * Each element is computed by the same function as the ungrouped path, so
 * the values are the same bit for bit. */
__device__ __forceinline__ void xg_gen_body_grouped(double *tile, int ts, int2 ij, int strip,
                                                    const double *__restrict__ xr, const double *__restrict__ yr,
                                                    const double *__restrict__ xc, const double *__restrict__ yc,
                                                    int n_rows, int n_cols, const XgMaternParams &p, int metric,
                                                    int identity_pad)
{
    __shared__ double s_val[8][32 * XG_GEN_ROWS];
    __shared__ unsigned short s_idx[8][32 * XG_GEN_ROWS];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (int)(blockDim.x >> 5);
    double *val = s_val[warp];
    unsigned short *idx = s_idx[warp];
    const unsigned lt = (1u << lane) - 1u;
    for (int g = warp; g * 32 < ts; g += nwarps) {
        const int c = g * 32 + lane;
        const int C = ij.y * ts + c;
        const bool col_ok = C < n_cols;
        const double x2 = col_ok ? xc[C] : 0.0, y2 = col_ok ? yc[C] : 0.0;
        int q_of[XG_GEN_ROWS];
#pragma unroll
        for (int rr = 0; rr < XG_GEN_ROWS; ++rr) {
            const int R = ij.x * ts + strip * XG_GEN_ROWS + rr;
            double v;
            int q = -1;
            if (R < n_rows && col_ok) {
                const double d = xg_distance(xr[R], yr[R], x2, y2, metric);
                const double r = d / p.beta;
                if (r == 0.0) {
                    v = p.sigma2 + p.nugget;
                } else {
                    q = xg_matern_branch(r, p.nu);
                    v = r;
                }
            } else {
                v = (identity_pad && R == C) ? 1.0 : 0.0;
            }
            val[rr * 32 + lane] = v; /* r for the listed elements, the value otherwise */
            q_of[rr] = q;
        }
        int start[5];
        start[0] = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int n = 0;
#pragma unroll
            for (int rr = 0; rr < XG_GEN_ROWS; ++rr) n += __popc(__ballot_sync(0xffffffffu, q_of[rr] == q));
            start[q + 1] = start[q] + n;
        }
        {
            int pos[4] = {start[0], start[1], start[2], start[3]};
#pragma unroll
            for (int rr = 0; rr < XG_GEN_ROWS; ++rr)
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const unsigned m = __ballot_sync(0xffffffffu, q_of[rr] == q);
                    if (q_of[rr] == q) idx[pos[q] + __popc(m & lt)] = (unsigned short)(rr * 32 + lane);
                    pos[q] += __popc(m);
                }
        }
        __syncwarp();
        for (int i = start[0] + lane; i < start[1]; i += 32) {
            const int e = idx[i];
            val[e] = xg_matern_small_c(val[e], p.con, p.tm);
        }
        for (int i = start[1] + lane; i < start[3]; i += 32) {
            const int e = idx[i];
            val[e] = xg_matern_trap(val[e], p.nu, p.con);
        }
        for (int i = start[3] + lane; i < start[4]; i += 32) {
            const int e = idx[i];
            val[e] = xg_matern_asym(val[e], p.nu, p.con);
        }
        __syncwarp();
#pragma unroll
        for (int rr = 0; rr < XG_GEN_ROWS; ++rr)
            tile[(long long)(strip * XG_GEN_ROWS + rr) * ts + c] = val[rr * 32 + lane];
        __syncwarp();
    }
}

__device__ __forceinline__ void xg_gen_body(const XgTileArgs &T, long long t, int2 ij, int strip,
                                            const double *__restrict__ xr, const double *__restrict__ yr,
                                            const double *__restrict__ xc, const double *__restrict__ yc, int n_rows,
                                            int n_cols, const XgMaternParams &p, int metric, int identity_pad)
{
    double *tile = T.data + t * (long long)T.ts * T.ts;
    if (!p.bivariate && p.half_integer < 0) {
        xg_gen_body_grouped(tile, T.ts, ij, strip, xr, yr, xc, yc, n_rows, n_cols, p, metric, identity_pad);
        return;
    }
    /* bivariate: matrix index 2 l + v -> location l, variable v */
    const int sh = p.bivariate ? 1 : 0;
    for (int rr = 0; rr < XG_GEN_ROWS; ++rr) {
        const int r = strip * XG_GEN_ROWS + rr;
        const int R = ij.x * T.ts + r;
        const bool row_ok = R < n_rows;
        const double x1 = row_ok ? xr[R >> sh] : 0.0, y1 = row_ok ? yr[R >> sh] : 0.0;
        for (int c = threadIdx.x; c < T.ts; c += blockDim.x) {
            const int C = ij.y * T.ts + c;
            double val;
            if (row_ok && C < n_cols) {
                const double d = xg_distance(x1, y1, xc[C >> sh], yc[C >> sh], metric);
                val = sh ? xg_matern_value_biv(d, p, R & 1, C & 1) : xg_matern_value(d, p);
            } else {
                val = (identity_pad && R == C) ? 1.0 : 0.0;
            }
            tile[(long long)r * T.ts + c] = val;
        }
    }
}

__global__ void __launch_bounds__(256) xg_gen_matern_kernel(XgTileArgs T, const int2 *__restrict__ tile_ij,
                                                            const double *__restrict__ xr, const double *__restrict__ yr,
                                                            const double *__restrict__ xc, const double *__restrict__ yc,
                                                            int n_rows, int n_cols, XgMaternParams p, int metric,
                                                            int identity_pad)
{
    const int strips = T.ts / XG_GEN_ROWS;
    const long long t = blockIdx.x / strips;
    xg_gen_body(T, t, tile_ij[t], (int)(blockIdx.x % strips), xr, yr, xc, yc, n_rows, n_cols, p, metric,
                identity_pad);
}

/* batched: every field's lower tiles, CTAs resolved through the step table */
__global__ void __launch_bounds__(256) xg_gen_matern_batch_kernel(XgTileArgs base, const XgBField *__restrict__ F,
                                                                  XgBStep S, const double *__restrict__ x,
                                                                  const double *__restrict__ y, int metric)
{
    long long local;
    const int f = xg_batch_resolve(S, blockIdx.x, &local);
    const XgBField &fd = F[f];
    XgTileArgs T = base;
    T.data = base.data + fd.tile_off * (long long)base.ts * base.ts;
    T.nt = fd.nt;
    const int strips = T.ts / XG_GEN_ROWS;
    const long long t = local / strips;
    const double *xf = x + fd.vec_off, *yf = y + fd.vec_off;
    xg_gen_body(T, t, xg_tile_decode(t, fd.nt), (int)(local % strips), xf, yf, xf, yf, fd.N, fd.N, fd.p, metric, 1);
}

/* ========================================================================== */
/* Loads of tile data.  COH = false: ordinary loads (the data was written by   */
/* an earlier launch).  COH = true: the bodies run inside the persistent       */
/* scheduler, where other CTAs of the same launch wrote the data: the loads go */
/* to L2 (ld.global.cg), never to a line this SM's L1 kept from an earlier     */
/* task.                                                                      */
/* ========================================================================== */

template <bool COH> __device__ __forceinline__ double xg_ldt(const double *p) { return COH ? __ldcg(p) : *p; }
template <bool COH> __device__ __forceinline__ double2 xg_ldt2(const double2 *p) { return COH ? __ldcg(p) : *p; }
template <bool COH> __device__ __forceinline__ double xg_ldro(const double *p) { return COH ? __ldcg(p) : __ldg(p); }

/* ========================================================================== */
/* POTRF of a diagonal tile, fused with log-det and the z block solve         */
/* ========================================================================== */

/* Panel of width NB (32, or 16 when ts = 1024) staged in shared memory with a
 * leading dimension NB + 4: row-per-thread access then costs one extra
 * wavefront but the DMMA fragment loads are conflict-free. */
#define XG_POTRF_THREADS 512

/* dst[r][c] = src[r][c] for r < rows, c < cols (leading dimensions ldd and
 * lds), by all threads of the CTA with U loads in flight per thread before
 * any store (the loads of a plain loop would wait one by one where the
 * compiler cannot tell dst and src apart). */
template <bool COH, int U = 8>
__device__ __forceinline__ void xg_stage_rows(double *dst, int ldd, const double *src, long long lds, int rows,
                                              int cols)
{
    const int total = rows * cols, step = (int)blockDim.x;
    for (int base = (int)threadIdx.x; base < total; base += U * step) {
        double t[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * step;
            if (idx < total) {
                const int r = idx / cols, c = idx - r * cols;
                t[u] = xg_ldt<COH>(src + (long long)r * lds + c);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int idx = base + u * step;
            if (idx < total) {
                const int r = idx / cols, c = idx - r * cols;
                dst[r * ldd + c] = t[u];
            }
        }
    }
}

/* Cholesky of the NB x NB block at P (leading dimension LDP, NB <= 32) by one
 * warp, lane r holding the part of row r still to be factored in registers:
 * at step j, w[t] is element (r, j + t), so the pivot column is always w[0]
 * and the loop over j stays rolled (one copy of the square root and the
 * division).  Per step the pivot is broadcast from lane j, the column is
 * scaled by the reciprocal of its square root (as LAPACK's dpotf2 scales by
 * ONE / AJJ) and stored, the lower trailing elements are updated with the
 * column's entries broadcast lane by lane, and the window shifts by one.
 * Writes L (zeros above the diagonal) back to P and 1 / L_jj to rdiag[j],
 * adds log L_rr to lane r's logdet; returns the first column (1-based) whose
 * pivot is not positive, or 0, the same value in every lane. */
template <int NB, int LDP>
__device__ __forceinline__ int xg_chol_warp(double *P, int lane, double &logdet_lane, double *rdiag)
{
    double w[NB];
    const bool act = lane < NB;
#pragma unroll
    for (int c = 0; c < NB; ++c) w[c] = act ? P[lane * LDP + c] : 0.0;
    int fail = 0;
#pragma unroll 1
    for (int j = 0; j < NB; ++j) {
        double d = __shfl_sync(0xffffffffu, w[0], j);
        if (!(d > 0.0)) {
            if (!fail) fail = j + 1;
            d = 1.0;
        }
        const double ljj = sqrt(d);
        const double rj = 1.0 / ljj;
        const double l = lane == j ? ljj : w[0] * rj; /* L(lane, j) for lane >= j */
        if (lane == j) rdiag[j] = rj;
        if (act && lane >= j) P[lane * LDP + j] = l;
#pragma unroll
        for (int t = 1; t < NB; ++t) {
            const double lcj = __shfl_sync(0xffffffffu, l, (j + t) & 31);
            if (t < NB - j && lane >= j + t) w[t] = fma(-l, lcj, w[t]);
        }
#pragma unroll
        for (int t = 0; t < NB - 1; ++t) w[t] = w[t + 1];
        w[NB - 1] = 0.0;
    }
    if (act) {
        for (int c = lane + 1; c < NB; ++c) P[lane * LDP + c] = 0.0;
        logdet_lane += log(P[lane * LDP + lane]);
    }
    return fail;
}

/* The same factorisation with the block left in shared memory (lane r
 * updates row r in place), for kernels launched with 512 threads whose
 * 128-register budget cannot hold a 32-double row: same results, same
 * return value. */
template <int NB, int LDP>
__device__ __forceinline__ int xg_chol_warp_smem(double *P, int lane, double &logdet_lane, double *rdiag)
{
    int fail = 0;
    for (int j = 0; j < NB; ++j) {
        double d = P[j * LDP + j];
        if (!(d > 0.0)) {
            if (!fail) fail = j + 1;
            d = 1.0;
        }
        const double ljj = sqrt(d);
        const double rj = 1.0 / ljj;
        __syncwarp();
        if (lane == j) {
            P[j * LDP + j] = ljj;
            logdet_lane += log(ljj);
            rdiag[j] = rj;
        } else if (lane > j && lane < NB) {
            P[lane * LDP + j] *= rj;
        }
        __syncwarp();
        if (lane > j && lane < NB) {
            const double lij = P[lane * LDP + j];
            for (int c = j + 1; c <= lane; ++c) P[lane * LDP + c] = fma(-lij, P[c * LDP + j], P[lane * LDP + c]);
        }
        __syncwarp();
    }
    if (lane < NB)
        for (int c = lane + 1; c < NB; ++c) P[lane * LDP + c] = 0.0;
    return fail;
}

/* Cholesky of the n x n block A (leading dimension lda; global memory or
 * shared memory) by NB-wide panels staged in P ([n][NB + 4], shared), fused
 * with the forward solve of vk (n entries, when with_rhs) using vs ([n],
 * shared).  A receives L with its strict upper triangle zeroed; a non-positive
 * pivot sets XG_ST_NOT_SPD and info = col0 + its 1-based column, and the call
 * returns false (CTA-uniformly).  *logdet_out = sum log L_ii, *dot_out = |vk|^2
 * after the solve (thread 0 / warp 0 write them). */
template <int NB, bool COH, bool REGCHOL = false>
__device__ __forceinline__ bool xg_potrf_block(double *A, int n, int lda, double *vk, int with_rhs, long long col0,
                                               int *status, int *info, double *logdet_out, double *dot_out,
                                               double *P, double *vs)
{
    constexpr int LDP = NB + 4;
    __shared__ int s_fail;
    __shared__ double s_logdet;
    __shared__ double s_rdiag[NB]; /* 1 / L_jj of the panel's diagonal block */
    const int ts = n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        s_fail = 0;
        s_logdet = 0.0;
    }
    if (with_rhs)
        for (int r = tid; r < ts; r += blockDim.x) vs[r] = xg_ldt<COH>(vk + r);
    double logdet_lane = 0.0;
    for (int c0 = 0; c0 < ts; c0 += NB) {
        const int rows = ts - c0;
        __syncthreads();
        xg_stage_rows<COH>(P, LDP, A + (long long)c0 * lda + c0, lda, rows, NB);
        __syncthreads();
        /* unblocked Cholesky of the NB x NB diagonal block (warp 0, in registers) */
        if (warp == 0) {
            const int f = REGCHOL ? xg_chol_warp<NB, LDP>(P, lane, logdet_lane, s_rdiag)
                                  : xg_chol_warp_smem<NB, LDP>(P, lane, logdet_lane, s_rdiag);
            if (f && lane == 0) s_fail = c0 + f;
        }
        __syncthreads();
        if (s_fail) {
            if (tid == 0) {
                atomicCAS(info, 0, (int)(col0 + s_fail));
                atomicOr(status, XG_ST_NOT_SPD);
            }
            return false;
        }
        /* rows below the diagonal block: X = B L_D^-T, one thread per row
         * (forward substitution, scaled by the reciprocals as dtrsm does) */
        for (int r = NB + tid; r < rows; r += blockDim.x) {
            double row[NB];
#pragma unroll
            for (int j = 0; j < NB; ++j) row[j] = P[r * LDP + j];
#pragma unroll
            for (int j = 0; j < NB; ++j) {
                double s = row[j];
#pragma unroll
                for (int q = 0; q < j; ++q) s -= row[q] * P[j * LDP + q];
                row[j] = s * s_rdiag[j];
            }
#pragma unroll
            for (int j = 0; j < NB; ++j) P[r * LDP + j] = row[j];
        }
        /* z block solve L_D w = vs[c0:c0+NB] (warp 0, forward substitution) */
        if (with_rhs && warp == 0) {
            double w = (lane < NB) ? vs[c0 + lane] : 0.0;
            for (int j = 0; j < NB; ++j) {
                if (lane == j) w = w / P[j * LDP + j];
                const double wj = __shfl_sync(0xffffffffu, w, j);
                if (lane > j && lane < NB) w -= P[lane * LDP + j] * wj;
            }
            if (lane < NB) vs[c0 + lane] = w;
        }
        __syncthreads();
        /* vs[below] -= P[below] . w ; write the panel back (upper of the
         * diagonal block zeroed, so the stored factor is exactly L) */
        if (with_rhs)
            for (int r = NB + tid; r < rows; r += blockDim.x) {
                double s = vs[c0 + r];
#pragma unroll
                for (int j = 0; j < NB; ++j) s -= P[r * LDP + j] * vs[c0 + j];
                vs[c0 + r] = s;
            }
        for (int idx = tid; idx < rows * NB; idx += blockDim.x) {
            const int rr = idx / NB, c = idx - rr * NB;
            A[(long long)(c0 + rr) * lda + c0 + c] = (rr < c) ? 0.0 : P[rr * LDP + c];
        }
        /* trailing update of the tile: A[t][t] -= Pb Pb^T on the lower part,
         * 32 x 32 output blocks per warp iteration, DMMA m16n8k4 */
        const int R = rows - NB;
        if (R > 0) {
            const int nbr = (R + 31) / 32;
            const int nblk = nbr * (nbr + 1) / 2;
            const int g = lane >> 2, tq = lane & 3;
            const double *Pb = P + NB * LDP;
            double *At = A + (long long)(c0 + NB) * lda + (c0 + NB);
            for (int blk = warp; blk < nblk; blk += (int)(blockDim.x >> 5)) {
                int bi = (int)((sqrtf(8.0f * blk + 1.0f) - 1.0f) * 0.5f);
                while ((bi + 1) * (bi + 2) / 2 <= blk) ++bi;
                while (bi * (bi + 1) / 2 > blk) --bi;
                const int bj = blk - bi * (bi + 1) / 2;
                const int r0 = bi * 32, cb0 = bj * 32;
                double acc[2][4][4];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                        for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;
#pragma unroll
                for (int p0 = 0; p0 < NB; p0 += 4) {
                    double a[2][2], b[4];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi) {
                        const int ra = r0 + mi * 16 + g;
                        a[mi][0] = (ra < R) ? Pb[ra * LDP + p0 + tq] : 0.0;
                        a[mi][1] = (ra + 8 < R) ? Pb[(ra + 8) * LDP + p0 + tq] : 0.0;
                    }
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni) {
                        const int cbn = cb0 + ni * 8 + g;
                        b[ni] = (cbn < R) ? Pb[cbn * LDP + p0 + tq] : 0.0;
                    }
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
                    for (int ni = 0; ni < 4; ++ni) {
                        const int cc = cb0 + ni * 8 + 2 * tq;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int rr = r0 + mi * 16 + g + 8 * h;
                            if (rr < R && cc < R) {
                                double2 *pc = reinterpret_cast<double2 *>(At + (long long)rr * lda + cc);
                                double2 cv = xg_ldt2<COH>(pc);
                                cv.x -= acc[mi][ni][2 * h];
                                cv.y -= acc[mi][ni][2 * h + 1];
                                *pc = cv;
                            }
                        }
                    }
            }
        }
    }
    /* zero the strict upper triangle outside the NB-wide diagonal blocks (the
     * panel write-back zeroed the part inside them), so the stored tile is
     * exactly L_kk and consumers may read it as a full tile */
    for (long long idx = tid; idx < (long long)ts * ts; idx += blockDim.x) {
        const int r = (int)(idx / ts), c = (int)(idx - (long long)r * ts);
        if (c >= (r / NB + 1) * NB) A[(long long)r * lda + c] = 0.0;
    }
    __syncthreads();
    /* deterministic reductions: log-det over lanes of warp 0, dot over vs */
    if (warp == 0) {
        double s = logdet_lane;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) s_logdet = s;
    }
    if (with_rhs)
        for (int rr = tid; rr < ts; rr += blockDim.x) vk[rr] = vs[rr];
    __syncthreads();
    if (tid == 0) *logdet_out = s_logdet;
    if (with_rhs && warp == 0) {
        double s = 0.0;
        for (int rr = lane; rr < ts; rr += 32) s += vs[rr] * vs[rr];
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) *dot_out = s;
    }
    return true;
}

template <int NB, bool COH = false, bool REGCHOL = false>
__device__ __forceinline__ void xg_potrf_body(const XgTileArgs &T, int k, double *__restrict__ v,
                                              double *__restrict__ part_logdet, double *__restrict__ part_dot,
                                              int with_rhs, int *status, int *info)
{
    extern __shared__ __align__(16) double xg_smem_d[];
    const int ts = T.ts;
    if (xg_cta_should_skip(status)) return;
    double *A = T.data + xg_slot64(T, k, k) * (long long)ts * ts;
    double *P = xg_smem_d;                     /* [ts][NB + 4] */
    double *vs = P + (size_t)ts * (NB + 4);    /* [ts] */
    xg_potrf_block<NB, COH, REGCHOL>(A, ts, ts, v + (long long)k * ts, with_rhs, (long long)k * ts, status, info,
                            part_logdet + k, part_dot + k, P, vs);
}

template <int NB>
__global__ void __launch_bounds__(XG_POTRF_THREADS) xg_potrf_diag_kernel(XgTileArgs T, int k, double *__restrict__ v,
                                                                         double *__restrict__ part_logdet,
                                                                         double *__restrict__ part_dot, int with_rhs,
                                                                         int *status, int *info)
{
    xg_potrf_body<NB>(T, k, v, part_logdet, part_dot, with_rhs, status, info);
}

/* batched: one CTA per field active at step k; info records the first
 * failing column of any field */
template <int NB>
__global__ void __launch_bounds__(XG_POTRF_THREADS) xg_potrf_diag_batch_kernel(XgTileArgs base,
                                                                               const XgBField *__restrict__ F,
                                                                               XgBStep S, int k, double *v,
                                                                               double *part, int *status, int *info)
{
    long long local;
    const int f = xg_batch_resolve(S, blockIdx.x, &local);
    const XgBField &fd = F[f];
    XgTileArgs T = base;
    T.data = base.data + fd.tile_off * (long long)base.ts * base.ts;
    T.nt = fd.nt;
    /* per-field status words: status[2 f] (flags), status[2 f + 1] (info) */
    xg_potrf_body<NB>(T, k, v + fd.vec_off, part + fd.part_off, part + fd.part_off + fd.nt, 1, status + 2 * f,
                      status + 2 * f + 1);
}

/* ========================================================================== */
/* Inverses of the 32 x 32 diagonal blocks of L_kk (for the panel TRSM)       */
/* ========================================================================== */

/* One warp inverts the 32 x 32 lower-triangular block LB (shared memory,
 * row stride 33): lane c forms column c by forward substitution,
 * z_i = (delta_ic - sum_{q<i} L_iq z_q) / L_ii, and stores D[i * 32 + c] = z_i.
 * The per-field and the batched paths share this arithmetic exactly. */
__device__ __forceinline__ void xg_lower32_inverse(const double *LB, int lane, double *D)
{
    double z[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        double s = (i == lane) ? 1.0 : 0.0;
#pragma unroll
        for (int q = 0; q < i; ++q) s -= LB[i * 33 + q] * z[q];
        z[i] = s / LB[i * 33 + i];
    }
#pragma unroll
    for (int i = 0; i < 32; ++i) D[i * 32 + lane] = z[i];
}


/* ========================================================================== */
/* Panel TRSM: L_ik = A_ik L_kk^-T, fused with v_i -= L_ik v_k                */
/* ========================================================================== */

#define XG_TRSM_THREADS 256 /* 255 registers a thread: a group's 32 L fragments are loaded before its DMMAs */
#define XG_TRSM_SR 32       /* rows of A_ik per CTA */

/* One 32-row strip B (leading dimension ld, w columns) <- B L^-T for the
 * lower-triangular w x w block L (same leading dimension), 32 columns at a
 * time: with dinv (the inverted 32 x 32 diagonal blocks of L, [(cb + r) * 32
 * + c]) each diagonal solve is a DMMA product -- warps 0-3 apply block b
 * while warps 4-7 fetch block b + 1 into the other buffer -- without it a
 * serial substitution; the rest of each step is a DMMA update in which each
 * warp takes 32-column groups and loads the group's 32 x 32 block of L
 * (32 fragments a thread) before its 64 DMMAs, so the L2 latency is paid
 * once per group.  With vk != nullptr also vi[0:32] -= B_new vk[0:w].
 * Called by every CTA thread after the status check. */
template <bool COH>
__device__ __forceinline__ void xg_trsm_core(double *B, const double *L, int ld, int w, const double *dinv,
                                             const double *vk, double *vi)
{
    const int LDS = w + 4;
    extern __shared__ __align__(16) double xg_smem_d[];
    double *S = xg_smem_d;              /* [SR][LDS] */
    double *LDb = S + XG_TRSM_SR * LDS; /* [2][32][33] */
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = (int)(blockDim.x >> 5);
    const int g = lane >> 2, tq = lane & 3;
    xg_stage_rows<COH>(S, LDS, B, ld, XG_TRSM_SR, w);
    if (dinv) xg_stage_rows<COH, 4>(LDb, 33, dinv, 32, 32, 32);
    for (int cb = 0, b = 0; cb < w; cb += 32, ++b) {
        double *LD = LDb + (b & 1) * (32 * 33);
        if (!dinv) {
            for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
                const int r = idx >> 5, c = idx & 31;
                LD[r * 33 + c] = xg_ldt<COH>(L + (long long)(cb + r) * ld + cb + c);
            }
        }
        __syncthreads();
        if (dinv) {
            /* S[:, cb:cb+32] <- S[:, cb:cb+32] D^T on DMMA: warp w < 4 computes
             * the 32 x 8 column block w (both 16-row halves); the results are
             * written after every warp has read its operands.  Warps 4.. fetch
             * the next block's inverse meanwhile. */
            double acc[2][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[mi][e] = 0.0;
            if (warp < 4) {
#pragma unroll
                for (int p0 = 0; p0 < 32; p0 += 4) {
                    const double b0 = LD[(warp * 8 + g) * 33 + p0 + tq];
#pragma unroll
                    for (int mi = 0; mi < 2; ++mi)
                        xg_dmma_16x8x4(acc[mi][0], acc[mi][1], acc[mi][2], acc[mi][3],
                                       S[(mi * 16 + g) * LDS + cb + p0 + tq], S[(mi * 16 + g + 8) * LDS + cb + p0 + tq],
                                       b0);
                }
            } else if (cb + 32 < w) {
                double *LN = LDb + ((b + 1) & 1) * (32 * 33);
                for (int idx = tid - 128; idx < 32 * 32; idx += (int)blockDim.x - 128) {
                    const int r = idx >> 5, c = idx & 31;
                    LN[r * 33 + c] = xg_ldt<COH>(dinv + (cb + 32 + r) * 32 + c);
                }
            }
            __syncthreads();
            if (warp < 4) {
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        double *ps = S + (mi * 16 + g + 8 * h) * LDS + cb + warp * 8 + 2 * tq;
                        ps[0] = acc[mi][2 * h];
                        ps[1] = acc[mi][2 * h + 1];
                    }
            }
        } else if (warp == 0) { /* lane = row of the strip */
            double row[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) row[j] = S[lane * LDS + cb + j];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                double s = row[j];
#pragma unroll
                for (int q = 0; q < j; ++q) s -= row[q] * LD[j * 33 + q];
                row[j] = s / LD[j * 33 + j];
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) S[lane * LDS + cb + j] = row[j];
        }
        __syncthreads();
        /* S[:, cb+32:] -= S[:, cb:cb+32] L[cb+32:, cb:cb+32]^T, 32-column groups */
        const int ncol = w - cb - 32;
        const int ngrp = ncol / 32;
        for (int grp = warp; grp < ngrp; grp += nwarps) {
            const int c0 = cb + 32 + grp * 32;
            double bl[8][4];
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni) bl[p][ni] = xg_ldro<COH>(L + (long long)(c0 + ni * 8 + g) * ld + cb + p * 4 + tq);
            double acc[2][4][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int e = 0; e < 4; ++e) acc[mi][ni][e] = 0.0;
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                double a[2][2];
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    a[mi][0] = S[(mi * 16 + g) * LDS + cb + p * 4 + tq];
                    a[mi][1] = S[(mi * 16 + g + 8) * LDS + cb + p * 4 + tq];
                }
#pragma unroll
                for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
                        xg_dmma_16x8x4(acc[mi][ni][0], acc[mi][ni][1], acc[mi][ni][2], acc[mi][ni][3], a[mi][0],
                                       a[mi][1], bl[p][ni]);
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
    }
    __syncthreads();
    for (int idx = tid; idx < XG_TRSM_SR * w; idx += blockDim.x) {
        const int r = idx / w, c = idx - r * w;
        B[(long long)r * ld + c] = S[r * LDS + c];
    }
    if (vk) {
        for (int r = warp; r < XG_TRSM_SR; r += nwarps) {
            double s = 0.0;
            for (int c = lane; c < w; c += 32) s += S[r * LDS + c] * xg_ldt<COH>(vk + c);
            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (lane == 0) vi[r] = xg_ldt<COH>(vi + r) - s;
        }
    }
}

template <bool COH = false>
__device__ __forceinline__ void xg_trsm_body(const XgTileArgs &T, int k, double *__restrict__ v, int with_rhs,
                                             const int *status, long long bid)
{
    const int ts = T.ts;
    if (xg_cta_should_skip(status)) return;
    const int strips = ts / XG_TRSM_SR;
    const int i = k + 1 + (int)(bid / strips);
    const int strip = (int)(bid % strips);
    double *B = T.data + xg_slot64(T, i, k) * (long long)ts * ts + (long long)strip * XG_TRSM_SR * ts;
    const double *L = T.data + xg_slot64(T, k, k) * (long long)ts * ts;
    xg_trsm_core<COH>(B, L, ts, ts, T.dinv, with_rhs ? v + (long long)k * ts : nullptr,
                      with_rhs ? v + (long long)i * ts + strip * XG_TRSM_SR : nullptr);
}

__global__ void __launch_bounds__(XG_TRSM_THREADS, 1) xg_trsm_panel_kernel(XgTileArgs T, int k, double *__restrict__ v,
                                                                        int with_rhs, const int *status)
{
    xg_trsm_body(T, k, v, with_rhs, status, blockIdx.x);
}

__global__ void __launch_bounds__(XG_TRSM_THREADS, 1) xg_trsm_panel_batch_kernel(XgTileArgs base,
                                                                              const XgBField *__restrict__ F,
                                                                              XgBStep S, int k, double *v,
                                                                              const int *status)
{
    long long local;
    const int f = xg_batch_resolve(S, blockIdx.x, &local);
    const XgBField &fd = F[f];
    XgTileArgs T = base;
    T.data = base.data + fd.tile_off * (long long)base.ts * base.ts;
    T.nt = fd.nt;
    xg_trsm_body(T, k, v + fd.vec_off, 1, status + 2 * f, local);
}

/* ========================================================================== */
/* Trailing update A_ij -= L_ik L_jk^T on FP64 tensor cores (DMMA), TMA fed   */
/* ========================================================================== */

/* 128 x 128 output block per CTA, K streamed in 16-wide slabs through a
 * 4-stage TMA ring (128-byte swizzle).  Eight warps compute (2 x 4 warps of
 * 64 x 32); thread 0 also issues the TMA loads, refilling a stage once all
 * eight warps have released it.  (A separate producer warp would make 9 warps,
 * which caps a 1-CTA kernel at 168 registers; 8 warps may use 255.) */
#define XG_G_BM 128
#define XG_G_BK 16
#define XG_G_STAGES 4
#define XG_G_THREADS 256
#define XG_G_STAGE_BYTES (2 * XG_G_BM * XG_G_BK * 8)

/* Updates the tiles (i, j), j0 <= j <= i < nt, with panel column k.  With
 * single_col the launch covers column j0 only (the lookahead split: the next
 * panel's column first, the rest of the trailing matrix in a second launch). */
/* One 128 x 128 block C -= A B^T on DMMA: A and B are 128-row boxes of the
 * TMA tensor `map` starting at rows rowA and rowB, K runs over KT 16-wide
 * slabs from column kx0 (a multiple of 16), C has leading dimension ldc.
 * Called by every CTA thread; the caller has done the status check. */
template <bool COH>
__device__ __forceinline__ void xg_gemm_core(const CUtensorMap &map, int rowA, int rowB, int kx0, int KT,
                                             double *C, int ldc, int *status)
{
    extern __shared__ __align__(1024) unsigned char xg_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)xg_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + XG_G_STAGES * XG_G_STAGE_BYTES);
    uint64_t *empty = full + XG_G_STAGES;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < XG_G_STAGES; ++s) {
            xg_mbar_init(&full[s], 1);
            xg_mbar_init(&empty[s], 8);
        }
        xg_fence_barrier_init();
    }
    __syncthreads();
    int issued = 0;
    __shared__ int s_gfail;
    if (COH) {
        /* each thread orders its earlier generic shared-memory writes (an
         * earlier task used this memory) before the TMA writes into it */
        xg_fence_proxy_async();
        if (tid == 0) s_gfail = 0;
        __syncthreads();
    }
    if (tid == 0) {
        /* the operand tiles may have been written by other CTAs of this launch
         * through ordinary stores: order them before the async-proxy reads */
        if (COH) asm volatile("fence.proxy.async.global;" ::: "memory");
        xg_prefetch_tensormap(&map);
        for (; issued < XG_G_STAGES && issued < KT; ++issued) {
            unsigned char *sa = smem + issued * XG_G_STAGE_BYTES;
            xg_mbar_arrive_expect_tx(&full[issued], XG_G_STAGE_BYTES);
            xg_tma_load_2d(sa, &map, kx0 + issued * XG_G_BK, rowA, &full[issued]);
            xg_tma_load_2d(sa + XG_G_BM * XG_G_BK * 8, &map, kx0 + issued * XG_G_BK, rowB, &full[issued]);
        }
    }
    const int wm = warp >> 2, wn = warp & 3;
    const int g = lane >> 2, tq = lane & 3;
    /* accumulators start at -C (loaded while the TMA ring fills), the main
     * loop adds L_ik L_jk^T and the epilogue stores -acc = C - L_ik L_jk^T */
    double acc[4][4][4];
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = wm * 64 + mi * 16 + g + 8 * h;
                const int c = wn * 32 + ni * 8 + 2 * tq;
                const double2 cv = xg_ldt2<COH>(reinterpret_cast<const double2 *>(C + (long long)r * ldc + c));
                acc[mi][ni][2 * h] = -cv.x;
                acc[mi][ni][2 * h + 1] = -cv.y;
            }
    bool ok = true;
    for (int kb = 0; kb < KT; ++kb) {
        const int s = kb % XG_G_STAGES;
        if (COH && __shfl_sync(0xffffffffu, *(volatile int *)&s_gfail, 0)) { /* warp-uniform */
            ok = false;
            break;
        }
        const bool landed = xg_mbar_wait(&full[s], (kb / XG_G_STAGES) & 1);
        if (COH ? !__all_sync(0xffffffffu, landed) : !landed) {
            ok = false;
            if (COH) s_gfail = 1;
            break;
        }
        const unsigned char *sa = smem + s * XG_G_STAGE_BYTES;
        const unsigned char *sb = sa + XG_G_BM * XG_G_BK * 8;
        /* k permutation inside the 16-wide slab: at MMA step ks, lane slot t
         * holds k = 4 t + ks.  A thread's four k values of a row are then
         * contiguous (two 16-byte chunks), read with conflict-free LDS.128
         * under the 128-byte swizzle. */
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int chunk = 2 * tq + half; /* k = 4 tq + 2 half + {0, 1} */
            double2 b[4];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni) {
                const int r = wn * 32 + ni * 8 + g;
                b[ni] = *(const double2 *)(sb + (r << 7) + ((chunk ^ (r & 7)) << 4));
            }
            /* one m-tile's A fragments at a time keeps the kernel within the
             * 168 registers a 288-thread CTA may use */
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
        /* refill this stage with slab kb + STAGES once every warp released it */
        if (tid == 0 && issued < KT) {
            if (xg_mbar_wait(&empty[s], (kb / XG_G_STAGES) & 1)) {
                unsigned char *sa = smem + s * XG_G_STAGE_BYTES;
                xg_mbar_arrive_expect_tx(&full[s], XG_G_STAGE_BYTES);
                xg_tma_load_2d(sa, &map, kx0 + issued * XG_G_BK, rowA, &full[s]);
                xg_tma_load_2d(sa + XG_G_BM * XG_G_BK * 8, &map, kx0 + issued * XG_G_BK, rowB, &full[s]);
                ++issued;
            } else {
                ok = false;
                if (COH) s_gfail = 1;
            }
        }
        __syncwarp();
        if (COH) ok = ok && !__shfl_sync(0xffffffffu, *(volatile int *)&s_gfail, 0);
        if (!ok) break;
    }
    if (COH) {
        /* a failed wait anywhere makes every warp leave together */
        __syncthreads();
        ok = s_gfail == 0;
    }
    if (!ok) {
        atomicOr(status, XG_ST_TIMEOUT);
        /* every copy thread 0 issued lands before the CTA may exit */
        if (tid == 0)
            for (int q = (issued > XG_G_STAGES ? issued - XG_G_STAGES : 0); q < issued; ++q)
                xg_mbar_wait(&full[q % XG_G_STAGES], (q / XG_G_STAGES) & 1);
        return;
    }
#pragma unroll
    for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = wm * 64 + mi * 16 + g + 8 * h;
                const int c = wn * 32 + ni * 8 + 2 * tq;
                *reinterpret_cast<double2 *>(C + (long long)r * ldc + c) =
                    make_double2(-acc[mi][ni][2 * h], -acc[mi][ni][2 * h + 1]);
            }
}

template <bool COH = false>
__device__ __forceinline__ void xg_gemm_body(const CUtensorMap &map, const XgTileArgs &T, int k, int j0,
                                             int single_col, int *status, long long bid)
{
    const int ts = T.ts;
    const int bpt = ts / XG_G_BM; /* blocks per tile side */
    const long long pair = bid / (bpt * bpt);
    const int blk = (int)(bid % (bpt * bpt));
    const int bi = blk / bpt, bj = blk % bpt;
    int i, j;
    const int nb = T.band ? T.band : T.band_targets;
    if (nb) {
        /* band targets (i, j), 0 <= i - j < nb, j from j0 */
        j = j0 + (int)(pair / nb);
        i = j + (int)(pair % nb);
        if (single_col && j != j0) i = T.nt; /* outside the launch */
    } else {
        int ii, jj;
        if (single_col) {
            ii = (int)pair;
            jj = 0;
        } else {
            xg_pair_decode(pair, &ii, &jj);
        }
        i = j0 + ii;
        j = j0 + jj;
    }
    if (xg_cta_should_skip(status, (i == j && bj > bi) || i >= T.nt)) return;
    /* operands: packed tiles (i, k), (j, k), or rows of the FP64 panel copy in mixed mode */
    const int rowA = T.band ? i * ts + bi * XG_G_BM
                            : (int)((T.tile_off + xg_tile_index(i, k, T.nt)) * ts + bi * XG_G_BM);
    const int rowB = T.band ? j * ts + bj * XG_G_BM
                            : (int)((T.tile_off + xg_tile_index(j, k, T.nt)) * ts + bj * XG_G_BM);
    double *C = T.data + xg_slot64(T, i, j) * (long long)ts * ts + (long long)(bi * XG_G_BM) * ts + bj * XG_G_BM;
    xg_gemm_core<COH>(map, rowA, rowB, 0, ts / XG_G_BK, C, ts, status);
}

__global__ void __launch_bounds__(XG_G_THREADS, 1) xg_syrk_gemm_kernel(const __grid_constant__ CUtensorMap map,
                                                                       XgTileArgs T, int k, int j0, int single_col,
                                                                       int *status)
{
    xg_gemm_body(map, T, k, j0, single_col, status, blockIdx.x);
}

/* batched: the trailing update of step k of every field with nt > k + 1 */
__global__ void __launch_bounds__(XG_G_THREADS, 1) xg_syrk_gemm_batch_kernel(const __grid_constant__ CUtensorMap map,
                                                                             XgTileArgs base,
                                                                             const XgBField *__restrict__ F,
                                                                             XgBStep S, int k, int *status)
{
    long long local;
    const int f = xg_batch_resolve(S, blockIdx.x, &local);
    const XgBField &fd = F[f];
    XgTileArgs T = base;
    T.data = base.data + fd.tile_off * (long long)base.ts * base.ts;
    T.nt = fd.nt;
    T.tile_off = fd.tile_off;
    xg_gemm_body(map, T, k, k + 1, 0, status + 2 * f, local);
}

/* ========================================================================== */
/* Panel TRSM by 128-column blocks: TMA-fed DMMA GEMMs + in-block solves      */
/* ========================================================================== */

/* L_ik = A_ik L_kk^-T for one 128-row block of A_ik per CTA, by the 128-column
 * blocks c of L_kk in order:
 *   T_c = A_c - sum_{q < c} X_q L_cq^T       (xg_gemm_core: K = 128 c, TMA-fed DMMA)
 *   X_c = T_c L_cc^-T                         (xg_block_trsm128: 4 steps of 32
 *                                              columns, each a DMMA product with the
 *                                              inverted 32 x 32 diagonal block and a
 *                                              DMMA update of the columns to its right)
 * so three quarters of the flops run at the trailing update's rate instead of
 * in 32-row strips.  The X_q read by the GEMM of step c are this CTA's own
 * stores of the steps before (ordered before the TMA reads by the proxy
 * fences of xg_gemm_core's coherent mode).  The rounding is that of the
 * strip TRSM up to the order of the sums: the solves use the same 32 x 32
 * inverses.  Fused: v_i -= L_ik v_k for the block's rows. */
#define XG_TB 128                                           /* rows of A_ik per CTA, columns per block */
#define XG_TB_S_BYTES ((size_t)XG_TB * XG_TB * sizeof(double)) /* the block, swizzled: fits the GEMM ring */

/* element (r, c) of the 128 x 128 staged block: each group of four rows is
 * shifted by a different multiple of four columns, so a DMMA fragment read
 * (rows g, columns tq of a 4-aligned column group) hits 32 distinct banks */
__device__ __forceinline__ int xg_tb_idx(int r, int c) { return r * XG_TB + (c ^ ((r & 3) << 2)); }

/* X = S L^-T in place for the staged 128 x 128 block S (xg_tb_idx layout),
 * L the 128 x 128 lower block (global, leading dimension ld), dinv its four
 * inverted 32 x 32 diagonal blocks ([(32 b + r) * 32 + c]); LDb: 2 x 32 x 33
 * doubles of shared memory.  256 threads. */
template <bool COH>
__device__ __forceinline__ void xg_block_trsm128(double *S, double *LDb, const double *L, int ld, const double *dinv)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tq = lane & 3;
    xg_stage_rows<COH, 4>(LDb, 33, dinv, 32, 32, 32);
    for (int cb = 0; cb < XG_TB / 32; ++cb) {
        const double *LD = LDb + (cb & 1) * (32 * 33);
        /* the next block's inverse, loaded now and stored after the barrier */
        double nd[4];
        const bool more = cb + 1 < XG_TB / 32;
        if (more)
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int idx = tid + u * 256;
                nd[u] = xg_ldt<COH>(dinv + (long long)(cb + 1) * 32 * 32 + idx);
            }
        __syncthreads(); /* S and LD[cb & 1] are complete */
        /* S[:, 32 cb : 32 cb + 32] <- that block D^T: warp w, rows 16 w .. + 15 */
        double acc[4][4];
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[ni][e] = 0.0;
        const int r0 = 16 * warp;
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            const int c = 32 * cb + 4 * p + tq;
            const double a0 = S[xg_tb_idx(r0 + g, c)], a1 = S[xg_tb_idx(r0 + g + 8, c)];
#pragma unroll
            for (int ni = 0; ni < 4; ++ni)
                xg_dmma_16x8x4(acc[ni][0], acc[ni][1], acc[ni][2], acc[ni][3], a0, a1, LD[(ni * 8 + g) * 33 + 4 * p + tq]);
        }
        __syncthreads(); /* every read of the block's columns is done */
#pragma unroll
        for (int ni = 0; ni < 4; ++ni)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + g + 8 * h, c = 32 * cb + ni * 8 + 2 * tq;
                *reinterpret_cast<double2 *>(&S[xg_tb_idx(r, c)]) = make_double2(acc[ni][2 * h], acc[ni][2 * h + 1]);
            }
        if (more) {
            double *LN = LDb + ((cb + 1) & 1) * (32 * 33);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int idx = tid + u * 256;
                LN[(idx >> 5) * 33 + (idx & 31)] = nd[u];
            }
        }
        __syncthreads();
        /* columns to the right: S[:, c0 : c0 + 32] -= S[:, 32 cb : +32] L[c0 : c0 + 32, 32 cb : +32]^T,
         * items = (32-row tile, 32-column group), the group's L fragments loaded first */
        const int ngrp = XG_TB / 32 - 1 - cb;
        for (int item = warp; item < 4 * ngrp; item += 8) {
            const int rt = item & 3, c0 = 32 * (cb + 1 + (item >> 2));
            double bl[8][4];
#pragma unroll
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
                    bl[p][ni] = xg_ldro<COH>(L + (long long)(c0 + ni * 8 + g) * ld + 32 * cb + 4 * p + tq);
            double ac[2][4][4];
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int e = 0; e < 4; ++e) ac[mi][ni][e] = 0.0;
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const int c = 32 * cb + 4 * p + tq;
#pragma unroll
                for (int mi = 0; mi < 2; ++mi) {
                    const int r = 32 * rt + 16 * mi + g;
                    const double a0 = S[xg_tb_idx(r, c)], a1 = S[xg_tb_idx(r + 8, c)];
#pragma unroll
                    for (int ni = 0; ni < 4; ++ni)
                        xg_dmma_16x8x4(ac[mi][ni][0], ac[mi][ni][1], ac[mi][ni][2], ac[mi][ni][3], a0, a1, bl[p][ni]);
                }
            }
#pragma unroll
            for (int mi = 0; mi < 2; ++mi)
#pragma unroll
                for (int ni = 0; ni < 4; ++ni)
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int r = 32 * rt + 16 * mi + g + 8 * h, c = c0 + ni * 8 + 2 * tq;
                        double2 *ps = reinterpret_cast<double2 *>(&S[xg_tb_idx(r, c)]);
                        double2 v = *ps;
                        v.x -= ac[mi][ni][2 * h];
                        v.y -= ac[mi][ni][2 * h + 1];
                        *ps = v;
                    }
        }
    }
    __syncthreads();
}

/* The TRSM of the 128-row block rb of panel tile (i, k); called by all 256
 * threads of a CTA after its status check.  Returns false (CTA-uniformly)
 * when a GEMM wait timed out.  Under the device scheduler (COH) the tiles and
 * inverses were written by other CTAs of the launch. */
template <bool COH>
__device__ __forceinline__ bool xg_trsm_gemm_body(const CUtensorMap &map, const XgTileArgs &T, int k, int i, int rb,
                                                  double *v, int with_rhs, int *status)
{
    extern __shared__ __align__(1024) unsigned char xg_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)xg_smem_raw + 1023) & ~(uintptr_t)1023);
    double *S = (double *)smem; /* aliases the GEMM ring, used between the GEMMs */
    double *LDb = (double *)(smem + XG_G_STAGES * XG_G_STAGE_BYTES + 1024);
    double *vacc = LDb + 2 * 32 * 33;
    __shared__ int s_stop;
    const int ts = T.ts, nb = ts / XG_TB, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const long long slot_i = T.tile_off + xg_tile_index(i, k, T.nt), slot_k = T.tile_off + xg_tile_index(k, k, T.nt);
    double *B = T.data + xg_slot64(T, i, k) * (long long)ts * ts + (long long)(rb * XG_TB) * ts;
    const double *Lkk = T.data + xg_slot64(T, k, k) * (long long)ts * ts;
    const double *vk = v + (long long)k * ts;
    if (with_rhs)
        for (int r = tid; r < XG_TB; r += blockDim.x) vacc[r] = 0.0;
    for (int c = 0; c < nb; ++c) {
        double *Bc = B + c * XG_TB;
        if (c > 0) {
            xg_gemm_core<true>(map, (int)(slot_i * ts + rb * XG_TB), (int)(slot_k * ts + c * XG_TB), 0,
                               c * XG_TB / XG_G_BK, Bc, ts, status);
            __syncthreads();
            if (tid == 0) s_stop = *(volatile int *)status != 0;
            __syncthreads();
            if (s_stop) return false;
        }
        /* stage T_c (this CTA's own stores, or the tile as the updates left it) */
        {
            constexpr int U = 8;
            for (int base = tid; base < XG_TB * XG_TB / 2; base += U * 256) {
                double2 t[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int idx = base + u * 256, r = idx >> 6, c2 = idx & 63;
                    t[u] = __ldcg(reinterpret_cast<const double2 *>(Bc + (long long)r * ts) + c2);
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int idx = base + u * 256, r = idx >> 6, c2 = idx & 63;
                    *reinterpret_cast<double2 *>(&S[xg_tb_idx(r, 2 * c2)]) = t[u];
                }
            }
        }
        xg_block_trsm128<COH>(S, LDb, Lkk + (long long)(c * XG_TB) * ts + c * XG_TB, ts,
                              T.dinv + (long long)(c * XG_TB) * 32);
        /* X_c back to the tile; v_i -= X_c v_k[c block] (row sums per warp) */
        for (int idx = tid; idx < XG_TB * XG_TB / 2; idx += 256) {
            const int r = idx >> 6, c2 = idx & 63;
            *(reinterpret_cast<double2 *>(Bc + (long long)r * ts) + c2) =
                *reinterpret_cast<const double2 *>(&S[xg_tb_idx(r, 2 * c2)]);
        }
        if (with_rhs) {
            for (int r = warp; r < XG_TB; r += 8) {
                double sum = 0.0;
                for (int cc = lane; cc < XG_TB; cc += 32) sum += S[xg_tb_idx(r, cc)] * __ldcg(vk + c * XG_TB + cc);
                for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
                if (lane == 0) vacc[r] += sum;
            }
        }
        __syncthreads(); /* S is read by everyone before the next GEMM's TMA writes the ring */
    }
    if (with_rhs) {
        double *vi = v + (long long)i * ts + rb * XG_TB;
        for (int r = tid; r < XG_TB; r += blockDim.x) vi[r] = xg_ldt<COH>(vi + r) - vacc[r];
    }
    return true;
}

__global__ void __launch_bounds__(XG_G_THREADS, 1)
    xg_trsm_gemm_kernel(const __grid_constant__ CUtensorMap map, XgTileArgs T, int k, double *v, int with_rhs,
                        int *status)
{
    if (xg_cta_should_skip(status)) return;
    const int nb = T.ts / XG_TB;
    xg_trsm_gemm_body<false>(map, T, k, k + 1 + (int)blockIdx.x / nb, (int)blockIdx.x % nb, v, with_rhs, status);
}

static size_t xg_trsm_gemm_smem_bytes()
{
    return 1024 + XG_G_STAGES * XG_G_STAGE_BYTES + 1024 + (2 * 32 * 33 + XG_TB) * sizeof(double);
}

/* ========================================================================== */
/* POTRF of a diagonal tile by 128 x 128 sub-blocks on several CTAs           */
/* ========================================================================== */

/* The one-CTA POTRF streams the whole ts x ts tile through one SM and updates
 * it in global memory once per 32-wide panel (1.5 ms at ts = 512).  Here the
 * tile is factored as a 4 x 4 (ts / 128 per side) grid of sub-blocks, right
 * looking, with three launches per sub-step s:
 *   xg_potrf_sub_kernel      L_ss = chol(A_ss) in shared memory (one CTA), the
 *                            forward solve of v's segment, log-det, and the
 *                            inverses of its four 32 x 32 diagonal blocks;
 *   xg_potrf_sub_trsm_kernel A_is <- A_is L_ss^-T for the sub-blocks below
 *                            (32-row strips, DMMA with the inverted blocks),
 *                            v_i -= L_is v_s;
 *   xg_potrf_sub_gemm_kernel A_ij -= L_is L_js^T for s < j <= i (TMA-fed DMMA,
 *                            one 128 x 128 block per CTA, K = 128).
 * The inverted diagonal blocks of the whole L_kk land in T.dinv on the way, so
 * the panel TRSM that follows needs no separate inversion. */
#define XG_SUB 128
#define XG_SUB_LDS (XG_SUB + 4)
#define XG_POTRF_SUB_THREADS 512
#define XG_POTRF_SUB_SMEM ((size_t)(XG_SUB * XG_SUB_LDS + XG_SUB * 36 + XG_SUB + 4 * 32 * 33) * sizeof(double))

__global__ void __launch_bounds__(XG_POTRF_SUB_THREADS) xg_potrf_sub_kernel(XgTileArgs T, int k, int s, double *v,
                                                                        double *part_logdet, double *part_dot,
                                                                        int with_rhs, int *status, int *info)
{
    extern __shared__ __align__(16) double xg_smem_d[];
    double *SD = xg_smem_d;                /* [128][132] the sub-block */
    double *P = SD + XG_SUB * XG_SUB_LDS;  /* [128][36] panel */
    double *vs = P + XG_SUB * 36;          /* [128] */
    double *LB = vs + XG_SUB;              /* [4][32 * 33] */
    __shared__ double s_ld, s_dot;
    if (xg_cta_should_skip(status)) return;
    const int ts = T.ts, r0 = s * XG_SUB;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double *A = T.data + xg_slot64(T, k, k) * (long long)ts * ts;
    double *vk = with_rhs ? v + (long long)k * ts : nullptr;
    xg_stage_rows<false>(SD, XG_SUB_LDS, A + (long long)r0 * ts + r0, ts, XG_SUB, XG_SUB);
    __syncthreads();
    if (!xg_potrf_block<32, false, true>(SD, XG_SUB, XG_SUB_LDS, vk ? vk + r0 : nullptr, with_rhs, (long long)k * ts + r0,
                                   status, info, &s_ld, &s_dot, P, vs))
        return;
    __syncthreads();
    if (T.dinv && warp < XG_SUB / 32) {
        double *lb = LB + warp * (32 * 33);
        for (int r = 0; r < 32; ++r) lb[r * 33 + lane] = SD[(warp * 32 + r) * XG_SUB_LDS + warp * 32 + lane];
        __syncwarp();
        xg_lower32_inverse(lb, lane, T.dinv + (long long)(r0 + 32 * warp) * 32);
    }
    /* L_ss (zeros above its diagonal) back to the tile, and zeros to its right */
    for (int idx = tid; idx < XG_SUB * XG_SUB; idx += blockDim.x) {
        const int r = idx / XG_SUB, c = idx - r * XG_SUB;
        A[(long long)(r0 + r) * ts + r0 + c] = SD[r * XG_SUB_LDS + c];
    }
    const int right = ts - r0 - XG_SUB;
    for (int idx = tid; idx < XG_SUB * right; idx += blockDim.x) {
        const int r = idx / right, c = idx - r * right;
        A[(long long)(r0 + r) * ts + r0 + XG_SUB + c] = 0.0;
    }
    __syncthreads();
    if (tid == 0) part_logdet[k] = (s == 0 ? 0.0 : part_logdet[k]) + s_ld;
    if (with_rhs && r0 + XG_SUB == ts && warp == 0) {
        /* |v_k|^2 over the whole tile, its segments all solved by now */
        double sum = 0.0;
        for (int rr = lane; rr < ts; rr += 32) {
            const double x = vk[rr];
            sum += x * x;
        }
        for (int off = 16; off > 0; off >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, off);
        if (lane == 0) part_dot[k] = sum;
    }
}

__global__ void __launch_bounds__(XG_TRSM_THREADS, 1) xg_potrf_sub_trsm_kernel(XgTileArgs T, int k, int s, double *v,
                                                                            int with_rhs, const int *status)
{
    if (xg_cta_should_skip(status)) return;
    const int ts = T.ts, r0 = s * XG_SUB;
    const int row = r0 + XG_SUB + (int)blockIdx.x * XG_TRSM_SR;
    double *A = T.data + xg_slot64(T, k, k) * (long long)ts * ts;
    double *vk = with_rhs ? v + (long long)k * ts : nullptr;
    xg_trsm_core<false>(A + (long long)row * ts + r0, A + (long long)r0 * ts + r0, ts, XG_SUB,
                        T.dinv ? T.dinv + (long long)r0 * 32 : nullptr, vk ? vk + r0 : nullptr,
                        vk ? vk + row : nullptr);
}

__global__ void __launch_bounds__(XG_G_THREADS, 1) xg_potrf_sub_gemm_kernel(const __grid_constant__ CUtensorMap map,
                                                                            XgTileArgs T, int k, int s, int *status)
{
    int ii, jj;
    xg_pair_decode(blockIdx.x, &ii, &jj);
    const int i = s + 1 + ii, j = s + 1 + jj;
    if (xg_cta_should_skip(status)) return;
    const int ts = T.ts;
    const long long slot = T.tile_off + xg_tile_index(k, k, T.nt);
    double *C = T.data + xg_slot64(T, k, k) * (long long)ts * ts + (long long)(i * XG_SUB) * ts + j * XG_SUB;
    xg_gemm_core<false>(map, (int)(slot * ts + i * XG_SUB), (int)(slot * ts + j * XG_SUB), s * XG_SUB,
                        XG_SUB / XG_G_BK, C, ts, status);
}

/* ========================================================================== */
/* Batched factorisation in one persistent launch (device tile scheduler)     */
/* ========================================================================== */

__device__ __forceinline__ int xg_ld_acquire(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void xg_add_release(int *p, int v)
{
    asm volatile("red.release.gpu.global.add.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

/* thread 0: waits until *p >= target; false when the wall-time limit passes
 * or another CTA aborted the launch */
__device__ __forceinline__ bool xg_sched_wait(const int *p, int target, const int *abort, uint64_t t0)
{
    while (xg_ld_acquire(p) < target) {
        if (*(volatile const int *)abort) return false;
        if (xg_globaltimer_ns() - t0 > 2000000000ull) return false;
        __nanosleep(256);
    }
    return true;
}

/* Persistent CTAs (one per SM, 256 threads) run the task list of XgSched:
 * thread 0 takes the next task, waits for its dependency counters, the CTA
 * runs the task body (the POTRF, TRSM and DMMA update bodies of the per-step
 * kernels, with L2-coherent loads), and thread 0 publishes it (release).
 * Tasks are taken in a topological order, so every task waited on was taken
 * earlier by a CTA that is running: the launch cannot deadlock.  A wait that
 * times out sets the field's XG_ST_TIMEOUT bit and the abort flag; a field
 * whose pivot fails skips its remaining bodies (status word) but still
 * publishes them, so no other field waits on it. */
template <int NB>
__global__ void __launch_bounds__(XG_G_THREADS, 1)
    xg_batch_sched_kernel(const __grid_constant__ CUtensorMap map, XgTileArgs base, const XgBField *__restrict__ F,
                          XgSched sch, double *v, double *part, int *status)
{
    __shared__ int4 s_task;
    __shared__ int s_go;
    const int tid = threadIdx.x;
    const int ts = base.ts;
    for (;;) {
        __syncthreads(); /* the previous task is finished by every thread */
        if (tid == 0) {
            int4 t = make_int4(-1, 0, 0, 0);
            if (!*(volatile int *)sch.abort) {
                const unsigned long long q = atomicAdd(sch.next, 1ULL);
                if (q < (unsigned long long)sch.ntasks) t = sch.tasks[q];
            }
            s_task = t;
        }
        __syncthreads();
        const int4 tk = s_task;
        if (tk.x < 0) break;
        const int type = tk.x & 3, f = tk.x >> 2, i = tk.y, j = tk.z, k = tk.w;
        const XgBField &fd = F[f];
        XgTileArgs T = base;
        T.data = base.data + fd.tile_off * (long long)ts * ts;
        T.nt = fd.nt;
        T.tile_off = fd.tile_off;
        int *stf = status + 2 * f;
        int *pdone = sch.cnt + fd.sched_off;
        int *tdone = pdone + fd.nt;
        int *ucnt = tdone + xg_num_lower_tiles(fd.nt);
        if (tid == 0) {
            const uint64_t t0 = xg_globaltimer_ns();
            bool ok;
            if (type == XG_TASK_POTRF)
                ok = xg_sched_wait(ucnt + xg_tile_index(k, k, fd.nt), k, sch.abort, t0);
            else if (type == XG_TASK_TRSM)
                ok = xg_sched_wait(pdone + k, 1, sch.abort, t0) &&
                     xg_sched_wait(ucnt + xg_tile_index(i, k, fd.nt), k, sch.abort, t0);
            else
                ok = xg_sched_wait(tdone + xg_tile_index(i, k, fd.nt), 1, sch.abort, t0) &&
                     xg_sched_wait(tdone + xg_tile_index(j, k, fd.nt), 1, sch.abort, t0) &&
                     xg_sched_wait(ucnt + xg_tile_index(i, j, fd.nt), k, sch.abort, t0);
            if (!ok) {
                atomicOr(stf, XG_ST_TIMEOUT);
                atomicExch(sch.abort, 1);
            }
            s_go = ok ? 1 : 0;
        }
        __syncthreads();
        if (s_go) {
            if (type == XG_TASK_POTRF) {
                xg_potrf_body<NB, true, true>(T, k, v + fd.vec_off, part + fd.part_off, part + fd.part_off + fd.nt, 1, stf,
                                        stf + 1);
            } else if (type == XG_TASK_TRSM) {
                /* the inverted diagonal blocks of L_kk into this CTA's scratch
                 * (warp w: blocks w, w + 8, ...), then the tile's row strips;
                 * done even for a field that has failed (its strips then skip),
                 * so every thread takes the same path */
                {
                    extern __shared__ __align__(16) double xg_smem_d[];
                    const int warp = tid >> 5, lane = tid & 31;
                    double *LB = xg_smem_d + warp * (32 * 33);
                    double *D = sch.dinv + (long long)blockIdx.x * ts * 32;
                    const double *Lkk = T.data + xg_tile_index(k, k, fd.nt) * (long long)ts * ts;
                    for (int bb = warp; bb < ts / 32; bb += XG_G_THREADS / 32) {
                        const double *Lb = Lkk + (long long)(bb * 32) * ts + bb * 32;
                        for (int r = 0; r < 32; ++r) LB[r * 33 + lane] = __ldcg(Lb + (long long)r * ts + lane);
                        __syncwarp();
                        xg_lower32_inverse(LB, lane, D + (long long)(bb * 32) * 32);
                        __syncwarp();
                    }
                    T.dinv = D;
                }
                __syncthreads();
                /* the tile's 128-row blocks one after the other (xg_trsm_gemm_body;
                 * a field that has failed skips them uniformly) */
                if (!xg_cta_should_skip(stf))
                    for (int rb = 0; rb < ts / XG_TB; ++rb)
                        if (!xg_trsm_gemm_body<true>(map, T, k, i, rb, v + fd.vec_off, 1, stf)) break;
            } else {
                const int bpt = ts / XG_G_BM;
                for (int b = 0; b < bpt * bpt; ++b)
                    xg_gemm_body<true>(map, T, k, j, 1, stf, (long long)(i - j) * bpt * bpt + b);
            }
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            if (type == XG_TASK_POTRF)
                xg_add_release(pdone + k, 1);
            else if (type == XG_TASK_TRSM)
                xg_add_release(tdone + xg_tile_index(i, k, fd.nt), 1);
            else
                xg_add_release(ucnt + xg_tile_index(i, j, fd.nt), 1);
        }
    }
}

static size_t xg_sched_smem_bytes(int ts)
{
    size_t b = xg_trsm_gemm_smem_bytes();
    b = b > xg_gemm_smem_bytes() ? b : xg_gemm_smem_bytes();
    b = b > xg_potrf_smem_bytes(ts) ? b : xg_potrf_smem_bytes(ts);
    b = b > xg_trsm_smem_bytes(ts) ? b : xg_trsm_smem_bytes(ts);
    return b;
}

void xg_launch_batch_sched(const CUtensorMap &map, const XgTileArgs &base, const XgBField *F, const XgSched &sch,
                           int ctas, double *v, double *part, int *status, cudaStream_t st)
{
    if (sch.ntasks <= 0 || ctas <= 0) return;
    xg_batch_sched_kernel<32><<<ctas, XG_G_THREADS, xg_sched_smem_bytes(base.ts), st>>>(map, base, F, sch, v, part,
                                                                                          status);
}

/* ========================================================================== */
/* Log-likelihood assembly                                                    */
/* ========================================================================== */

/* loglik = -0.5 dotp - 0.5 logdet - (N / 2.0) log(2 pi)  (MLE_dexact.c:426),
 * with logdet = 2 sum log L_ii (MLE_dexact.c:384) summed in tile order. */
__global__ void xg_finalize_kernel(const double *part_logdet, const double *part_dot, int nt, int N, double *out,
                                   const int *status, const int *info)
{
    if (threadIdx.x != 0) return;
    double det = 0.0, dot = 0.0;
    for (int k = 0; k < nt; ++k) {
        det += part_logdet[k];
        dot += part_dot[k];
    }
    const double logdet = 2.0 * det;
    out[0] = -0.5 * dot - 0.5 * logdet - (double)(N / 2.0) * log(2.0 * 3.141592653589793);
    out[1] = logdet;
    out[2] = dot;
    out[3] = (double)(*status);
    out[4] = (double)(*info);
}

/* batched: one thread per field */
__global__ void xg_finalize_batch_kernel(const XgBField *__restrict__ F, int nfields, const double *part,
                                         double *out)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfields) return;
    const XgBField &fd = F[f];
    double det = 0.0, dot = 0.0;
    for (int k = 0; k < fd.nt; ++k) {
        det += part[fd.part_off + k];
        dot += part[fd.part_off + fd.nt + k];
    }
    const double logdet = 2.0 * det;
    out[2 * f] = -0.5 * dot - 0.5 * logdet - (double)(fd.N / 2.0) * log(2.0 * 3.141592653589793);
    out[2 * f + 1] = logdet;
}

/* ========================================================================== */
/* Host launchers                                                             */
/* ========================================================================== */

static int xg_potrf_nb(int ts) { return ts > 512 ? 16 : 32; }

size_t xg_potrf_smem_bytes(int ts) { return ((size_t)ts * (xg_potrf_nb(ts) + 4) + ts) * sizeof(double); }
size_t xg_trsm_smem_bytes(int ts) { return ((size_t)XG_TRSM_SR * (ts + 4) + 2 * 32 * 33) * sizeof(double); }
size_t xg_gemm_smem_bytes() { return (size_t)XG_G_STAGES * XG_G_STAGE_BYTES + 2 * XG_G_STAGES * 8 + 1024; }

cudaError_t xg_kernels_configure()
{
    cudaError_t e;
    e = cudaFuncSetAttribute(xg_potrf_diag_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_potrf_smem_bytes(512));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_trsm_smem_bytes(XG_MAX_TS));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_syrk_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_gemm_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_potrf_diag_batch_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_potrf_smem_bytes(512));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_trsm_panel_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_trsm_smem_bytes(XG_MAX_TS));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_syrk_gemm_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_gemm_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_batch_sched_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_sched_smem_bytes(XG_MAX_TS));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_potrf_sub_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XG_POTRF_SUB_SMEM);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_potrf_sub_trsm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_trsm_smem_bytes(XG_SUB));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_potrf_sub_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_gemm_smem_bytes());
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(xg_trsm_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)xg_trsm_gemm_smem_bytes());
    return e;
}

void xg_launch_gen(const XgTileArgs &T, const int2 *tile_ij, long long ntiles, const double *xr, const double *yr,
                   const double *xc, const double *yc, int n_rows, int n_cols, const XgMaternParams &p, int metric,
                   int identity_pad, cudaStream_t st)
{
    const long long blocks = ntiles * (T.ts / XG_GEN_ROWS);
    xg_gen_matern_kernel<<<(unsigned)blocks, 256, 0, st>>>(T, tile_ij, xr, yr, xc, yc, n_rows, n_cols, p, metric,
                                                            identity_pad);
}

void xg_launch_potrf_diag(const XgTileArgs &T, int k, double *v, double *part_logdet, double *part_dot, int with_rhs,
                          int *status, int *info, cudaStream_t st)
{
    const size_t smem = xg_potrf_smem_bytes(T.ts);
    if (xg_potrf_nb(T.ts) == 16)
        xg_potrf_diag_kernel<16><<<1, XG_POTRF_THREADS, smem, st>>>(T, k, v, part_logdet, part_dot, with_rhs, status,
                                                                     info);
    else
        xg_potrf_diag_kernel<32><<<1, XG_POTRF_THREADS, smem, st>>>(T, k, v, part_logdet, part_dot, with_rhs, status,
                                                                     info);
}

void xg_launch_potrf_tiled(const CUtensorMap &map, const XgTileArgs &T, int k, double *v, double *part_logdet,
                           double *part_dot, int with_rhs, int *status, int *info, cudaStream_t st)
{
    const int nb = T.ts / XG_SUB;
    for (int s = 0; s < nb; ++s) {
        xg_potrf_sub_kernel<<<1, XG_POTRF_SUB_THREADS, XG_POTRF_SUB_SMEM, st>>>(T, k, s, v, part_logdet, part_dot,
                                                                           with_rhs, status, info);
        const int m = nb - s - 1;
        if (m > 0) {
            xg_potrf_sub_trsm_kernel<<<m * (XG_SUB / XG_TRSM_SR), XG_TRSM_THREADS, xg_trsm_smem_bytes(XG_SUB), st>>>(
                T, k, s, v, with_rhs, status);
            xg_potrf_sub_gemm_kernel<<<m * (m + 1) / 2, XG_G_THREADS, xg_gemm_smem_bytes(), st>>>(map, T, k, s,
                                                                                                 status);
        }
    }
}

int xg_potrf_tiled_launches(int ts) { return 3 * (ts / XG_SUB) - 2; }


void xg_launch_trsm_panel(const XgTileArgs &T, int k, double *v, int with_rhs, const int *status, cudaStream_t st,
                          int i1)
{
    /* tiles i = k+1 .. i1-1 (i1 < 0: to the last tile) */
    const int last = (i1 < 0 || i1 > T.nt) ? T.nt : i1;
    const int n = last - k - 1;
    if (n <= 0) return;
    xg_trsm_panel_kernel<<<n * (T.ts / XG_TRSM_SR), XG_TRSM_THREADS, xg_trsm_smem_bytes(T.ts), st>>>(T, k, v, with_rhs,
                                                                                                   status);
}

void xg_launch_trsm_gemm(const CUtensorMap &map, const XgTileArgs &T, int k, double *v, int with_rhs, int *status,
                         cudaStream_t st)
{
    const int n = T.nt - k - 1;
    if (n <= 0) return;
    xg_trsm_gemm_kernel<<<n * (T.ts / XG_TB), XG_G_THREADS, xg_trsm_gemm_smem_bytes(), st>>>(map, T, k, v, with_rhs,
                                                                                          status);
}

void xg_launch_syrk_gemm(const CUtensorMap &map, const XgTileArgs &T, int k, int *status, cudaStream_t st, int part)
{
    /* part: 0 = every trailing column, 1 = column k+1 only, 2 = columns >= k+2 */
    const int j0 = (part == 2) ? k + 2 : k + 1;
    const long long n = T.nt - j0;
    if (n <= 0) return;
    const int bpt = T.ts / XG_G_BM;
    const long long pairs = (part == 1) ? n : n * (n + 1) / 2;
    const long long blocks = pairs * bpt * bpt;
    xg_syrk_gemm_kernel<<<(unsigned)blocks, XG_G_THREADS, xg_gemm_smem_bytes(), st>>>(map, T, k, j0, part == 1,
                                                                                       status);
}

/* band targets of the trailing update in mixed mode: part 1 = column k+1,
 * part 2 = columns >= k+2, part 0 = all */
void xg_launch_band_gemm(const CUtensorMap &p64map, const XgTileArgs &T, int k, int part, int *status,
                         cudaStream_t st)
{
    const int j0 = (part == 2) ? k + 2 : k + 1;
    const long long ncol = (part == 1) ? 1 : T.nt - j0;
    if (j0 >= T.nt || ncol <= 0) return;
    const int bpt = T.ts / XG_G_BM;
    const long long blocks = ncol * (T.band ? T.band : T.band_targets) * bpt * bpt;
    xg_syrk_gemm_kernel<<<(unsigned)blocks, XG_G_THREADS, xg_gemm_smem_bytes(), st>>>(p64map, T, k, j0, part == 1,
                                                                                       status);
}

void xg_launch_batch_gen(const XgTileArgs &base, const XgBField *F, const XgBStep &S, long long blocks,
                         const double *x, const double *y, int metric, cudaStream_t st)
{
    if (blocks > 0) xg_gen_matern_batch_kernel<<<(unsigned)blocks, 256, 0, st>>>(base, F, S, x, y, metric);
}

void xg_launch_batch_potrf(const XgTileArgs &base, const XgBField *F, const XgBStep &S, int k, double *v, double *part,
                           int *status, int *info, cudaStream_t st)
{
    if (S.nact <= 0) return;
    xg_potrf_diag_batch_kernel<32><<<S.nact, XG_POTRF_THREADS, xg_potrf_smem_bytes(base.ts), st>>>(
        base, F, S, k, v, part, status, info);
}

void xg_launch_batch_trsm(const XgTileArgs &base, const XgBField *F, const XgBStep &S, long long blocks, int k,
                          double *v, const int *status, cudaStream_t st)
{
    if (blocks > 0)
        xg_trsm_panel_batch_kernel<<<(unsigned)blocks, XG_TRSM_THREADS, xg_trsm_smem_bytes(base.ts), st>>>(
            base, F, S, k, v, status);
}

void xg_launch_batch_gemm(const CUtensorMap &map, const XgTileArgs &base, const XgBField *F, const XgBStep &S,
                          long long blocks, int k, int *status, cudaStream_t st)
{
    if (blocks > 0)
        xg_syrk_gemm_batch_kernel<<<(unsigned)blocks, XG_G_THREADS, xg_gemm_smem_bytes(), st>>>(map, base, F, S, k,
                                                                                               status);
}

void xg_launch_batch_finalize(const XgBField *F, int nfields, const double *part, double *out, cudaStream_t st)
{
    xg_finalize_batch_kernel<<<(nfields + 127) / 128, 128, 0, st>>>(F, nfields, part, out);
}

void xg_launch_finalize(const double *part_logdet, const double *part_dot, int nt, int N, double *out,
                        const int *status, const int *info, cudaStream_t st)
{
    xg_finalize_kernel<<<1, 32, 0, st>>>(part_logdet, part_dot, nt, N, out, status, info);
}
