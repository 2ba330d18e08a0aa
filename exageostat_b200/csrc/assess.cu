/*
 * Assessment of a fitted model, on sm_100a: the Fisher information matrix and
 * the MLOE / MMOM criteria.
 *
 * Fisher (EXAGEOSTAT_Fisher_Tile, exageostat_exact/src/compute/MLE_dexact.c:1777-1934):
 *   F_jk = 1/2 tr(Sigma^-1 dSigma_j Sigma^-1 dSigma_k), then F^-1.
 *   The reference forms Sigma^-1 dSigma_j by two N x N triangular solves per
 *   (j, k) pair and multiplies the pairs (30 N^3 flops for three parameters).
 *   Here S = Sigma^-1 comes from the gradient's inverse factor and SYRK
 *   (2/3 N^3), each G_j = S dSigma_j is one DMMA GEMM on full tiles (2 N^3),
 *   and all traces tr(G_j G_k) come from one pass over the G_j
 *   (xg_fisher_trace_kernel).  dSigma_j is generated on the fly into full
 *   tiles from the element derivatives (core_dcmg_matern_dsigma_square /
 *   _dbeta / _dnu, exageostat_exact/cpu_core/compute/core_zcmg.c:315-488;
 *   the nu derivative of K_nu is exact instead of the reference's 1e-9
 *   forward difference, core_zcmg.c:228-235).  The nugget parameter has
 *   dSigma = I, so its G is S itself.
 *
 * MLOE / MMOM (EXAGEOSTAT_dmle_mloe_mmom_Tile, MLE_dexact.c:1109-1434, with
 * the per-point accumulation of CORE_dmloe_mmom_starpu,
 * exageostat_exact/runtime/starpu/codelets/codelet_zmloe_mmom.c:22-60):
 *   the reference loops over the missing points, each with four
 *   triangular solves and a triangular multiply of one vector against the
 *   full factors.  Here all missing points are right-hand sides of the same
 *   tile solves (an "R layout" matrix: one row per missing point, tile (R, K)
 *   at slot K mt + R), so the work runs on the FP64 tensor cores:
 *     A = L_a^-1 k_a,  U = L_a^-1 k_t,  T = L_t^-1 k_t      (forward solves)
 *     W = L_a^-T A = K_a^-1 k_a        (backward solve on L_a's tiles transposed in place)
 *     V = L_t^T W                      (triangular product with L_t's tiles transposed in place)
 *   and per missing point (one reduction kernel)
 *     expr1 = U.A,  expr2 = sigma_t^2 - 2 expr1 + V.V,
 *     expr3 = sigma_t^2 - T.T,  expr4 = sigma_a^2 - A.A,
 *     loe = expr2 / expr3 - 1,  mom = expr4 / expr2 - 1   (-1 on a zero denominator).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../include/exageostat_b200.h"
#include "kbessel.cuh"
#include "xg_common.cuh"
#include "xg_engine.h"
#include "xg_kernels.h"
#include "xg_matern.cuh"

#define XG_AS_ROWS 8

/* ------------------------------------------------------------------------- */
/* MLOE / MMOM kernels                                                       */
/* ------------------------------------------------------------------------- */

/* Cross-covariance k(obs o, miss m) in R layout: row m, column o of tile
 * (m / ts, o / ts) at slot (o / ts) mt + m / ts; zero outside nmiss x nobs.
 * One CTA: XG_AS_ROWS rows of one tile. */
__global__ void __launch_bounds__(256) xg_cross_gen_r_kernel(double *__restrict__ D, int mt, int ts,
                                                             const double *__restrict__ xm,
                                                             const double *__restrict__ ym, int nmiss,
                                                             const double *__restrict__ xo,
                                                             const double *__restrict__ yo, int nobs,
                                                             XgMaternParams p, int metric)
{
    const int strips = ts / XG_AS_ROWS;
    const long long slot = blockIdx.x / strips;
    const int strip = blockIdx.x % strips;
    const int K = (int)(slot / mt), R = (int)(slot % mt);
    double *tile = D + slot * (long long)ts * ts;
    for (int rr = 0; rr < XG_AS_ROWS; ++rr) {
        const int r = strip * XG_AS_ROWS + rr;
        const int m = R * ts + r;
        const bool mok = m < nmiss;
        const double x2 = mok ? xm[m] : 0.0, y2 = mok ? ym[m] : 0.0;
        for (int c = threadIdx.x; c < ts; c += blockDim.x) {
            const int o = K * ts + c;
            double v = 0.0;
            if (mok && o < nobs) v = xg_matern_value(xg_distance(xo[o], yo[o], x2, y2, metric), p);
            tile[(long long)r * ts + c] = v;
        }
    }
}

void xg_launch_cross_gen_r(double *D, int mt, int nt, int ts, const double *xm, const double *ym, int nmiss,
                           const double *xo, const double *yo, int nobs, const XgMaternParams &p, int metric,
                           cudaStream_t st)
{
    const long long blocks = (long long)mt * nt * (ts / XG_AS_ROWS);
    xg_cross_gen_r_kernel<<<(unsigned)blocks, 256, 0, st>>>(D, mt, ts, xm, ym, nmiss, xo, yo, nobs, p, metric);
}

/* Every tile of a packed store transposed in place: one CTA swaps the 32 x 32
 * blocks (a, b) and (b, a), a >= b, of one tile. */
__global__ void __launch_bounds__(256) xg_tile_transpose_kernel(double *__restrict__ D, int ts, int npairs)
{
    __shared__ double s1[32][33], s2[32][33];
    const long long t = blockIdx.x / npairs;
    int a, b;
    xg_pair_decode(blockIdx.x % npairs, &a, &b);
    double *tile = D + t * (long long)ts * ts;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int i = ty; i < 32; i += 8) {
        s1[i][tx] = tile[(long long)(a * 32 + i) * ts + b * 32 + tx];
        s2[i][tx] = tile[(long long)(b * 32 + i) * ts + a * 32 + tx];
    }
    __syncthreads();
    for (int i = ty; i < 32; i += 8) {
        tile[(long long)(a * 32 + i) * ts + b * 32 + tx] = s2[tx][i];
        tile[(long long)(b * 32 + i) * ts + a * 32 + tx] = s1[tx][i];
    }
}

void xg_launch_tile_transpose(double *D, long long ntiles, int ts, cudaStream_t st)
{
    const int nb = ts / 32, npairs = nb * (nb + 1) / 2;
    xg_tile_transpose_kernel<<<(unsigned)(ntiles * npairs), 256, 0, st>>>(D, ts, npairs);
}

/* One CTA per missing point m: the four row sums over its R-layout row in A,
 * U, T, V, combined into terms[6 m ..] = expr1, expr2, expr3, expr4, loe, mom. */
__global__ void __launch_bounds__(256) xg_mloe_terms_kernel(const double *__restrict__ A, const double *__restrict__ U,
                                                            const double *__restrict__ T, const double *__restrict__ V,
                                                            int mt, int nt, int ts, double sigma2_t, double sigma2_a,
                                                            double *__restrict__ terms)
{
    __shared__ double red[4][8];
    const int m = blockIdx.x;
    const int R = m / ts, r = m % ts;
    double s[4] = {0.0, 0.0, 0.0, 0.0}; /* A.A, U.A, T.T, V.V */
    for (int K = 0; K < nt; ++K) {
        const long long off = (((long long)K * mt + R) * ts + r) * ts;
        for (int c = threadIdx.x; c < ts; c += blockDim.x) {
            const double a = A[off + c], u = U[off + c], t = T[off + c], v = V[off + c];
            s[0] += a * a;
            s[1] += u * a;
            s[2] += t * t;
            s[3] += v * v;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double v = s[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double tot[4];
        for (int q = 0; q < 4; ++q) {
            double v = 0.0;
            for (int w = 0; w < 8; ++w) v += red[q][w];
            tot[q] = v;
        }
        /* MLE_dexact.c:1371-1375: expr1 <- alpha_t - 2 expr1, expr2 <- expr1 + expr2,
         * expr3 <- alpha_t - expr3, expr4 <- alpha_a - expr4 */
        const double e1 = tot[1];
        const double e2 = (sigma2_t - 2.0 * e1) + tot[3];
        const double e3 = sigma2_t - tot[2];
        const double e4 = sigma2_a - tot[0];
        double *o = terms + 6 * (long long)m;
        o[0] = e1;
        o[1] = e2;
        o[2] = e3;
        o[3] = e4;
        o[4] = e3 == 0.0 ? -1.0 : e2 / e3 - 1.0; /* codelet_zmloe_mmom.c:48-53 */
        o[5] = e2 == 0.0 ? -1.0 : e4 / e2 - 1.0; /* :55-60 */
    }
}

void xg_launch_mloe_terms(const double *A, const double *U, const double *T, const double *V, int mt, int nt, int ts,
                          int nmiss, double sigma2_t, double sigma2_a, double *terms, cudaStream_t st)
{
    xg_mloe_terms_kernel<<<nmiss, 256, 0, st>>>(A, U, T, V, mt, nt, ts, sigma2_t, sigma2_a, terms);
}

/* ------------------------------------------------------------------------- */
/* Fisher kernels                                                            */
/* ------------------------------------------------------------------------- */

/* Full tiles (slot A nt + B) of the symmetric S from its lower-tile store, by
 * 32 x 32 blocks: a block on or below the diagonal is copied, one above it is
 * the transpose of its mirror.  Only the diagonal 128-blocks of S's diagonal
 * tiles and the blocks below them are read (what the inverse SYRK writes). */
__global__ void __launch_bounds__(256) xg_sym_full_kernel(const double *__restrict__ S, double *__restrict__ F,
                                                          int nt, int ts)
{
    __shared__ double s[32][33];
    const int nb = ts / 32;
    const long long nbg = (long long)nt * nb;
    const int gb = (int)(blockIdx.x % nbg), ga = (int)(blockIdx.x / nbg);
    const int A = ga / nb, a = ga % nb, B = gb / nb, b = gb % nb;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double *dst = F + ((long long)A * nt + B) * ts * ts;
    if (ga >= gb) {
        const double *src = S + xg_tile_index(A, B, nt) * ts * ts;
        for (int i = ty; i < 32; i += 8)
            dst[(long long)(a * 32 + i) * ts + b * 32 + tx] = src[(long long)(a * 32 + i) * ts + b * 32 + tx];
    } else {
        const double *src = S + xg_tile_index(B, A, nt) * ts * ts;
        for (int i = ty; i < 32; i += 8) s[i][tx] = src[(long long)(b * 32 + i) * ts + a * 32 + tx];
        __syncthreads();
        for (int i = ty; i < 32; i += 8) dst[(long long)(a * 32 + i) * ts + b * 32 + tx] = s[tx][i];
    }
}

void xg_launch_sym_full(const double *S, double *F, int nt, int ts, cudaStream_t st)
{
    const long long nbg = (long long)nt * (ts / 32);
    xg_sym_full_kernel<<<(unsigned)(nbg * nbg), 256, 0, st>>>(S, F, nt, ts);
}

/* dSigma/dtheta_which (0 sigma^2, 1 beta, 2 nu) into full tiles, zero outside
 * N x N; at zero distance 1 for sigma^2 and 0 for beta and nu
 * (core_zcmg.c:331-332, 394-395, 471-472). */
__global__ void __launch_bounds__(256) xg_dsigma_full_kernel(double *__restrict__ D, int nt, int ts,
                                                             const double *__restrict__ x,
                                                             const double *__restrict__ y, int N, XgMaternParams p,
                                                             double dlogcon, int metric, int which)
{
    const int strips = ts / XG_AS_ROWS;
    const long long slot = blockIdx.x / strips;
    const int strip = blockIdx.x % strips;
    const int A = (int)(slot / nt), B = (int)(slot % nt);
    double *tile = D + slot * (long long)ts * ts;
    for (int rr = 0; rr < XG_AS_ROWS; ++rr) {
        const int r = strip * XG_AS_ROWS + rr;
        const int ga = A * ts + r;
        const bool rok = ga < N;
        const double x1 = rok ? x[ga] : 0.0, y1 = rok ? y[ga] : 0.0;
        for (int c = threadIdx.x; c < ts; c += blockDim.x) {
            const int gb = B * ts + c;
            double v = 0.0;
            if (rok && gb < N) {
                const double rd = xg_distance(x1, y1, x[gb], y[gb], metric) / p.beta;
                if (rd == 0.0) {
                    v = which == 0 ? 1.0 : 0.0;
                } else {
                    double m, ds, db, dn;
                    xg_matern_grad(rd, p.nu, p.con, p.sigma2, p.beta, dlogcon, &m, &ds, &db, &dn);
                    v = which == 0 ? ds : (which == 1 ? db : dn);
                }
            }
            tile[(long long)r * ts + c] = v;
        }
    }
}

void xg_launch_dsigma_full(double *D, int nt, int ts, const double *x, const double *y, int N,
                           const XgMaternParams &p, double dlogcon, int metric, int which, cudaStream_t st)
{
    const long long blocks = (long long)nt * nt * (ts / XG_AS_ROWS);
    xg_dsigma_full_kernel<<<(unsigned)blocks, 256, 0, st>>>(D, nt, ts, x, y, N, p, dlogcon, metric, which);
}

struct XgFisherG {
    const double *g[4];
};

/* part[10 blockIdx.x + q] for the pairs q = (j, k), j <= k < 4, in row order
 * (pairs with k >= np stay zero):
 * sum over a, b < N of G_j[a, b] G_k[b, a].  A CTA walks pairs of 32-blocks
 * (ga <= gb): the (gb, ga) blocks of every G are staged transposed in shared
 * memory, the (ga, gb) blocks are read in rows. */
__global__ void __launch_bounds__(256) xg_fisher_trace_kernel(XgFisherG G, int np, int nt, int ts, int N,
                                                              long long npairs, double *__restrict__ part)
{
    __shared__ double Q[4][32][33];
    __shared__ double red[10][8];
    const int nb = ts / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    double acc[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) acc[q] = 0.0;
    for (long long pid = blockIdx.x; pid < npairs; pid += gridDim.x) {
        int gi, gj;
        xg_pair_decode(pid, &gi, &gj);
        const int ga = gj, gb = gi; /* ga <= gb */
        const long long offQ =
            (((long long)(gb / nb) * nt + ga / nb) * ts + (gb % nb) * 32) * ts + (ga % nb) * 32;
        const long long offP =
            (((long long)(ga / nb) * nt + gb / nb) * ts + (ga % nb) * 32) * ts + (gb % nb) * 32;
        __syncthreads();
#pragma unroll
        for (int m = 0; m < 4; ++m)
            if (m < np)
                for (int i = ty; i < 32; i += 8) Q[m][i][tx] = G.g[m][offQ + (long long)i * ts + tx];
        __syncthreads();
        for (int i = ty; i < 32; i += 8) {
            if (ga * 32 + i >= N || gb * 32 + tx >= N) continue;
            double P[4];
#pragma unroll
            for (int m = 0; m < 4; ++m) P[m] = m < np ? G.g[m][offP + (long long)i * ts + tx] : 0.0;
            int q = 0;
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int k = j; k < 4; ++k, ++q)
                    if (k < np) {
                        double t = P[j] * Q[k][tx][i];
                        if (ga != gb) t += P[k] * Q[j][tx][i];
                        acc[q] += t;
                    }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 10; ++q) {
        double v = acc[q];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 10) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += red[threadIdx.x][w];
        part[10 * (long long)blockIdx.x + threadIdx.x] = v;
    }
}

void xg_launch_fisher_trace(const double *const g[4], int np, int nt, int ts, int N, double *part, int nctas,
                            cudaStream_t st)
{
    XgFisherG G;
    for (int m = 0; m < 4; ++m) G.g[m] = m < np ? g[m] : nullptr;
    const long long nbg = (long long)nt * (ts / 32);
    const long long npairs = nbg * (nbg + 1) / 2;
    xg_fisher_trace_kernel<<<nctas, 256, 0, st>>>(G, np, nt, ts, N, npairs, part);
}

/* ------------------------------------------------------------------------- */
/* host: Fisher information                                                  */
/* ------------------------------------------------------------------------- */

#define XG_ACU(call)                                                                                                   \
    do {                                                                                                               \
        cudaError_t _e = (call);                                                                                       \
        if (_e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));                   \
    } while (0)

static int xg_status_error(const int sv[2], const char *what)
{
    if (sv[0] & XG_ST_NOT_SPD) return xg_fail(XG_ERR_NOT_SPD, "%s is not positive definite (pivot %d)", what, sv[1]);
    if (sv[0] & XG_ST_TIMEOUT) return xg_fail(XG_ERR_TIMEOUT, "a device pipeline wait timed out");
    return xg_fail(XG_ERR_CUDA, "device status word 0x%x", sv[0]);
}

/* n x n SPD inverse as EXAGEOSTAT_Fisher_Tile does it (MLE_dexact.c:1893-1916):
 * A = L L^T, then X = L^-T (L^-1 I).  A and inv row-major (A symmetric). */
int xg_small_spd_inverse(int n, const double *A, double *inv)
{
    double L[16] = {0};
    for (int j = 0; j < n; ++j) {
        double d = A[j * n + j];
        for (int k = 0; k < j; ++k) d -= L[j * n + k] * L[j * n + k];
        if (!(d > 0.0)) return xg_fail(XG_ERR_NOT_SPD, "the Fisher matrix is not positive definite");
        L[j * n + j] = sqrt(d);
        for (int i = j + 1; i < n; ++i) {
            double s = A[i * n + j];
            for (int k = 0; k < j; ++k) s -= L[i * n + k] * L[j * n + k];
            L[i * n + j] = s / L[j * n + j];
        }
    }
    for (int c = 0; c < n; ++c) {
        double y[4];
        for (int i = 0; i < n; ++i) { /* L y = e_c */
            double s = i == c ? 1.0 : 0.0;
            for (int k = 0; k < i; ++k) s -= L[i * n + k] * y[k];
            y[i] = s / L[i * n + i];
        }
        for (int i = n - 1; i >= 0; --i) { /* L^T x = y */
            double s = y[i];
            for (int k = i + 1; k < n; ++k) s -= L[k * n + i] * inv[k * n + c];
            inv[i * n + c] = s / L[i * n + i];
        }
    }
    return XG_OK;
}

/* Fisher information of the field's locations at theta: kernel 0 gives the
 * 3 x 3 matrix of (sigma^2, beta, nu), kernel 1 the 4 x 4 one with tau^2.
 * F row-major; seconds = device time of the whole computation.  The field's
 * covariance store is overwritten (the next evaluation regenerates it). */
int xg_field_fisher(XgField *f, const double *theta, int kernel, double *F, double *seconds)
{
    if (xg_bivariate(kernel) || xg_bivariate(f->kernel))
        return xg_fail(XG_ERR_UNSUPPORTED, "the Fisher matrix of a bivariate field");
    int rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    const int nt = f->C.nt, ts = f->C.ts, N = f->N;
    const int np = kernel == 1 ? 4 : 3;
    if (!f->X.d) {
        rc = xg_tm_alloc(f->X, N, ts);
        if (rc) return rc;
    }
    const size_t full = (size_t)nt * nt * ts * ts;
    const int nctas = g_xg.sm_count * 8;
    double *Sf = nullptr, *D = nullptr, *G = nullptr, *part = nullptr;
    if (cudaMalloc(&Sf, full * sizeof(double)) != cudaSuccess || cudaMalloc(&D, full * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&G, 3 * full * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&part, 10 * (size_t)nctas * sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(Sf);
        cudaFree(D);
        cudaFree(G);
        cudaFree(part);
        return xg_fail(XG_ERR_NO_MEMORY, "Fisher workspace: %.2f GB", 5.0 * full * sizeof(double) / 1e9);
    }
    std::vector<double> hp(10 * (size_t)nctas);
    int sv[2] = {0, 0};
    CUtensorMap mS, mD;
    rc = xg_encode_tiles(&mS, Sf, (long long)nt * nt, ts);
    if (!rc) rc = xg_encode_tiles(&mD, D, (long long)nt * nt, ts);
    if (!rc) {
        cudaStream_t st = g_xg.stream;
        XgTileArgs T{f->C.d, ts, nt};
        const XgMaternParams p = xg_params(theta, kernel);
        const double dlogcon = -(log(2.0) + xg_digamma(theta[2]));
        cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st);
        cudaEventRecord(f->ev[0], st);
        /* Sigma (MLE_dexact.c:1824-1825), its factor (:1830) and S = Sigma^-1 */
        xg_launch_gen(T, f->C.ij, f->C.ntiles, f->x, f->y, f->x, f->y, N, N, p, f->metric, 1, st);
        XgFactorStreams fs;
        fs.st = st;
        fs.st_hi = g_xg.stream_hi;
        fs.ev_panel = f->ev_panel;
        fs.ev_upd = f->ev_upd;
        xg_factor_lookahead(f->C, nullptr, f->part, f->status, f->info, fs);
        xg_launch_inverse_factor(f->X.map, f->C.map, f->X.d, f->C.d, nt, ts, f->status, st);
        xg_launch_inverse_syrk(f->X.map, f->C.d, nt, ts, f->status, st);
        xg_launch_sym_full(f->C.d, Sf, nt, ts, st);
        /* G_j = S dSigma_j (dSigma_j symmetric: S dSigma_j^T) */
        for (int j = 0; j < 3; ++j) {
            xg_launch_dsigma_full(D, nt, ts, f->x, f->y, N, p, dlogcon, f->metric, j, st);
            xg_launch_dense_gemm_nt(mS, mD, G + j * full, nt, ts, f->status, st);
        }
        const double *g[4] = {G, G + full, G + 2 * full, Sf};
        xg_launch_fisher_trace(g, np, nt, ts, N, part, nctas, st);
        cudaEventRecord(f->ev[3], st);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(sv, f->status, sizeof sv, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = xg_fail(XG_ERR_CUDA, "Fisher: %s", cudaGetErrorString(e));
        if (!rc && seconds) {
            float ms = 0;
            cudaEventElapsedTime(&ms, f->ev[0], f->ev[3]);
            *seconds = ms * 1e-3;
        }
    }
    cudaFree(Sf);
    cudaFree(D);
    cudaFree(G);
    cudaFree(part);
    if (rc) return rc;
    if (sv[0]) return xg_status_error(sv, "the covariance");
    int q = 0;
    for (int j = 0; j < 4; ++j)
        for (int k = j; k < 4; ++k, ++q) {
            if (k >= np) continue;
            double s = 0.0;
            for (int b = 0; b < nctas; ++b) s += hp[10 * (size_t)b + q];
            F[j * np + k] = F[k * np + j] = 0.5 * s;
        }
    return XG_OK;
}

/* ------------------------------------------------------------------------- */
/* host: MLOE / MMOM                                                         */
/* ------------------------------------------------------------------------- */

void xg_assess_destroy(XgAssess *q)
{
    if (!q) return;
    xg_tm_free(q->Ca);
    xg_tm_free(q->Ct);
    for (int i = 0; i < 5; ++i) cudaFree(q->R[i]);
    cudaFree(q->xo);
    cudaFree(q->yo);
    cudaFree(q->xm);
    cudaFree(q->ym);
    cudaFree(q->terms);
    cudaFree(q->part);
    cudaFree(q->status);
    for (int i = 0; i < 4; ++i)
        if (q->ev[i]) cudaEventDestroy(q->ev[i]);
    if (q->ev_panel) cudaEventDestroy(q->ev_panel);
    if (q->ev_upd) cudaEventDestroy(q->ev_upd);
    delete q;
}

static int xg_assess_alloc(double **p, size_t n)
{
    cudaError_t e = cudaMalloc(p, n * sizeof(double));
    if (e != cudaSuccess) {
        *p = nullptr;
        return xg_fail(XG_ERR_NO_MEMORY, "cudaMalloc(%zu doubles): %s", n, cudaGetErrorString(e));
    }
    return cudaMemset(*p, 0, n * sizeof(double)) == cudaSuccess ? XG_OK : XG_ERR_CUDA;
}

int xg_assess_create(XgAssess **out, int nmiss, int nobs, int ts)
{
    *out = nullptr;
    int rc = xg_context_require();
    if (rc) return rc;
    if (nmiss <= 0 || nobs <= 0) return xg_fail(XG_ERR_BAD_ARGUMENT, "nZmiss = %d, nZobs = %d", nmiss, nobs);
    XgAssess *q = new XgAssess();
    q->nmiss = nmiss;
    q->nobs = nobs;
    q->ts = xg_choose_ts(nobs, ts);
    rc = xg_tm_alloc(q->Ca, nobs, q->ts);
    if (!rc) rc = xg_tm_alloc(q->Ct, nobs, q->ts);
    q->nt = q->Ca.nt;
    q->mt = (nmiss + q->ts - 1) / q->ts;
    const long long rtiles = (long long)q->mt * q->nt;
    for (int i = 0; i < 5 && !rc; ++i) {
        rc = xg_assess_alloc(&q->R[i], (size_t)rtiles * q->ts * q->ts);
        if (!rc) rc = xg_encode_tiles(&q->mR[i], q->R[i], rtiles, q->ts);
    }
    const size_t Np = (size_t)q->nt * q->ts;
    if (!rc) rc = xg_assess_alloc(&q->xo, Np);
    if (!rc) rc = xg_assess_alloc(&q->yo, Np);
    if (!rc) rc = xg_assess_alloc(&q->xm, nmiss);
    if (!rc) rc = xg_assess_alloc(&q->ym, nmiss);
    if (!rc) rc = xg_assess_alloc(&q->terms, 6 * (size_t)nmiss);
    if (!rc) rc = xg_assess_alloc(&q->part, 2 * (size_t)q->nt);
    if (!rc && cudaMalloc(&q->status, 2 * sizeof(int)) != cudaSuccess) rc = xg_fail(XG_ERR_NO_MEMORY, "status");
    for (int i = 0; i < 4 && !rc; ++i)
        if (cudaEventCreate(&q->ev[i]) != cudaSuccess) rc = xg_fail(XG_ERR_CUDA, "events");
    if (!rc && (cudaEventCreateWithFlags(&q->ev_panel, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&q->ev_upd, cudaEventDisableTiming) != cudaSuccess))
        rc = xg_fail(XG_ERR_CUDA, "lookahead events");
    if (rc) {
        xg_assess_destroy(q);
        return rc;
    }
    *out = q;
    return XG_OK;
}

/* mloe / mmom (means over the missing points), terms (6 per point, optional)
 * and times[4] = generation, the two factorisations, the solves and
 * reductions, total (seconds, CUDA events). */
int xg_assess_run(XgAssess *q, const double *truth, const double *est, int kernel, int metric, const double *xm,
                  const double *ym, const double *xo, const double *yo, double *mloe, double *mmom, double *terms,
                  double *times)
{
    int rc = xg_check_theta(truth, kernel);
    if (!rc) rc = xg_check_theta(est, kernel);
    if (rc) return rc;
    cudaStream_t st = g_xg.stream;
    const int nmiss = q->nmiss, nobs = q->nobs, nt = q->nt, mt = q->mt, ts = q->ts;
    const XgMaternParams pt = xg_params(truth, kernel), pa = xg_params(est, kernel);
    double *RA = q->R[0], *RU = q->R[1], *RT = q->R[2], *RW = q->R[3], *RV = q->R[4];
    const size_t rbytes = (size_t)mt * nt * ts * ts * sizeof(double);
    XG_ACU(cudaMemsetAsync(q->status, 0, 2 * sizeof(int), st));
    XG_ACU(cudaMemcpyAsync(q->xo, xo, nobs * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_ACU(cudaMemcpyAsync(q->yo, yo, nobs * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_ACU(cudaMemcpyAsync(q->xm, xm, nmiss * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_ACU(cudaMemcpyAsync(q->ym, ym, nmiss * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_ACU(cudaEventRecord(q->ev[0], st));
    /* K_a = Sigma(obs, obs; estimated), K_t (truth) (MLE_dexact.c:1239-1245),
     * k_a and k_t for every missing point at once (:1283-1286) */
    XgTileArgs Ta{q->Ca.d, ts, nt}, Tt{q->Ct.d, ts, nt};
    xg_launch_gen(Ta, q->Ca.ij, q->Ca.ntiles, q->xo, q->yo, q->xo, q->yo, nobs, nobs, pa, metric, 1, st);
    xg_launch_gen(Tt, q->Ct.ij, q->Ct.ntiles, q->xo, q->yo, q->xo, q->yo, nobs, nobs, pt, metric, 1, st);
    xg_launch_cross_gen_r(RA, mt, nt, ts, q->xm, q->ym, nmiss, q->xo, q->yo, nobs, pa, metric, st);
    xg_launch_cross_gen_r(RU, mt, nt, ts, q->xm, q->ym, nmiss, q->xo, q->yo, nobs, pt, metric, st);
    XG_ACU(cudaMemcpyAsync(RT, RU, rbytes, cudaMemcpyDeviceToDevice, st));
    XG_ACU(cudaEventRecord(q->ev[1], st));
    /* the two factorisations (:1252, :1261) */
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = q->ev_panel;
    fs.ev_upd = q->ev_upd;
    xg_factor_lookahead(q->Ca, nullptr, q->part, q->status, q->status + 1, fs);
    xg_factor_lookahead(q->Ct, nullptr, q->part, q->status, q->status + 1, fs);
    XG_ACU(cudaEventRecord(q->ev[2], st));
    /* the per-point solves (:1300-1364) for all points */
    xg_launch_rhs_forward_solve(q->mR[0], RA, mt, q->Ca.map, q->Ca.d, nt, ts, q->status, st); /* A = L_a^-1 k_a */
    xg_launch_rhs_forward_solve(q->mR[1], RU, mt, q->Ca.map, q->Ca.d, nt, ts, q->status, st); /* U = L_a^-1 k_t */
    xg_launch_rhs_forward_solve(q->mR[2], RT, mt, q->Ct.map, q->Ct.d, nt, ts, q->status, st); /* T = L_t^-1 k_t */
    /* W = L_a^-T A: the factor's tiles transposed in place, then the backward solve */
    XG_ACU(cudaMemcpyAsync(RW, RA, rbytes, cudaMemcpyDeviceToDevice, st));
    xg_launch_tile_transpose(q->Ca.d, q->Ca.ntiles, ts, st);
    xg_launch_rhs_backward_solve(q->mR[3], RW, mt, q->Ca.map, q->Ca.d, nt, ts, q->status, st);
    xg_launch_tile_transpose(q->Ct.d, q->Ct.ntiles, ts, st);
    xg_launch_rhs_tri_product(q->mR[3], q->Ct.map, RV, mt, nt, ts, q->status, st); /* V = L_t^T W */
    xg_launch_mloe_terms(RA, RU, RT, RV, mt, nt, ts, nmiss, truth[0], est[0], q->terms, st);
    XG_ACU(cudaEventRecord(q->ev[3], st));
    XG_ACU(cudaGetLastError());
    std::vector<double> h(6 * (size_t)nmiss);
    int sv[2];
    XG_ACU(cudaMemcpyAsync(h.data(), q->terms, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    XG_ACU(cudaMemcpyAsync(sv, q->status, sizeof sv, cudaMemcpyDeviceToHost, st));
    XG_ACU(cudaStreamSynchronize(st));
    if (sv[0]) return xg_status_error(sv, "K_a or K_t");
    double sl = 0.0, sm = 0.0;
    for (int m = 0; m < nmiss; ++m) {
        sl += h[6 * (size_t)m + 4];
        sm += h[6 * (size_t)m + 5];
    }
    *mloe = sl / nmiss;
    *mmom = sm / nmiss;
    if (terms) memcpy(terms, h.data(), h.size() * sizeof(double));
    if (times) {
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, q->ev[0], q->ev[1]);
        cudaEventElapsedTime(&b, q->ev[1], q->ev[2]);
        cudaEventElapsedTime(&c, q->ev[2], q->ev[3]);
        times[0] = a * 1e-3;
        times[1] = b * 1e-3;
        times[2] = c * 1e-3;
        times[3] = (a + b + c) * 1e-3;
    }
    return XG_OK;
}
