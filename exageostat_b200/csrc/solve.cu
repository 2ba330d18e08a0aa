/*
 * Memory-bound kernels on the lower-tile factor and the kriging kernels.
 *
 *   xg_trmv_lower_kernel      z = L e (CHAMELEON_dtrmm_Tile(Left, Lower, NoTrans, NonUnit),
 *                             exageostat_exact/src/compute/MLE_dexact.c:120)
 *   xg_trsv_lt_*              alpha = L^-T v, the backward half of CHAMELEON_dposv_Tile (MLE_dexact.c:812)
 *   xg_predict_cross_kernel   zmiss = Sigma(miss, obs) alpha with the cross-covariance generated on the
 *                             fly (dcmg of C12 + CHAMELEON_dgemm_Tile, MLE_dexact.c:803-820), never stored
 *   xg_mse_kernel             sum (zactual - zmiss)^2 / nmiss (CORE_dmse_starpu,
 *                             runtime/starpu/codelets/codelet_zmse.c:22-38; MLE_dexact.c:845)
 */
#include <math.h>

#include "kbessel.cuh"
#include "xg_common.cuh"
#include "xg_kernels.h"
#include "xg_matern.cuh"

/* ---- z = L e : 32 rows of tile-row i per CTA, 8 warps x 4 rows ---- */
__global__ void __launch_bounds__(256) xg_trmv_lower_kernel(XgTileArgs T, const double *__restrict__ e,
                                                            double *__restrict__ z, const int *status)
{
    if (*status != 0) return;
    const int ts = T.ts;
    const int strips = ts / 32;
    const int i = blockIdx.x / strips, strip = blockIdx.x % strips;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int j = 0; j <= i; ++j) {
        const double *tile = T.data + xg_tile_index(i, j, T.nt) * (long long)ts * ts;
        const double *ej = e + (long long)j * ts;
        for (int c = lane; c < ts; c += 32) {
            const double ec = ej[c];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int r = strip * 32 + warp * 4 + q;
                acc[q] += tile[(long long)r * ts + c] * ec;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double s = acc[q];
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) z[(long long)i * ts + strip * 32 + warp * 4 + q] = s;
    }
}

void xg_launch_trmv_lower(const XgTileArgs &T, const double *e, double *z, const int *status, cudaStream_t st)
{
    xg_trmv_lower_kernel<<<T.nt * (T.ts / 32), 256, 0, st>>>(T, e, z, status);
}

/* ---- alpha = L^-T v, right-looking over tile columns from the last ---- */

/* Diagonal tile k: solve L_kk^T a = v_k in place, 32-row blocks from the
 * bottom; within a block one lane per row, then the rows above are updated
 * by all threads. */
__global__ void __launch_bounds__(512) xg_trsv_lt_diag_kernel(XgTileArgs T, int k, double *__restrict__ v,
                                                              const int *status)
{
    if (xg_cta_should_skip(status)) return;
    const int ts = T.ts;
    extern __shared__ double vsh[];
    const double *L = T.data + xg_tile_index(k, k, T.nt) * (long long)ts * ts;
    double *vk = v + (long long)k * ts;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int r = tid; r < ts; r += blockDim.x) vsh[r] = vk[r];
    __syncthreads();
    for (int b0 = ts - 32; b0 >= 0; b0 -= 32) {
        if (warp == 0) {
            /* L_D^T a_D = w_D, L_D = L[b0:b0+32, b0:b0+32] lower: backward substitution */
            double w = vsh[b0 + lane];
            for (int j = 31; j >= 0; --j) {
                if (lane == j) w = w / L[(long long)(b0 + j) * ts + b0 + j];
                const double aj = __shfl_sync(0xffffffffu, w, j);
                if (lane < j) w -= L[(long long)(b0 + j) * ts + b0 + lane] * aj;
            }
            vsh[b0 + lane] = w;
        }
        __syncthreads();
        /* rows above: w[c] -= sum_{r in block} L[r][c] a[r], c < b0 */
        for (int c = tid; c < b0; c += blockDim.x) {
            double s = vsh[c];
#pragma unroll 8
            for (int r = 0; r < 32; ++r) s -= L[(long long)(b0 + r) * ts + c] * vsh[b0 + r];
            vsh[c] = s;
        }
        __syncthreads();
    }
    for (int r = tid; r < ts; r += blockDim.x) vk[r] = vsh[r];
}

/* Tiles i < k: v_i -= L_ki^T a_k; one CTA per (i, 256-column chunk). */
__global__ void __launch_bounds__(256) xg_trsv_lt_update_kernel(XgTileArgs T, int k, double *__restrict__ v,
                                                                const int *status)
{
    if (*status != 0) return;
    const int ts = T.ts;
    const int chunks = (ts + 255) / 256;
    const int i = blockIdx.x / chunks;
    const int c = (blockIdx.x % chunks) * 256 + threadIdx.x;
    if (c >= ts) return;
    const double *tile = T.data + xg_tile_index(k, i, T.nt) * (long long)ts * ts;
    const double *ak = v + (long long)k * ts;
    double s = 0.0;
    for (int r = 0; r < ts; ++r) s += tile[(long long)r * ts + c] * ak[r];
    v[(long long)i * ts + c] -= s;
}

void xg_launch_trsv_lower_t_step(const XgTileArgs &T, int k, double *v, const int *status, cudaStream_t st)
{
    xg_trsv_lt_diag_kernel<<<1, 512, T.ts * sizeof(double), st>>>(T, k, v, status);
    if (k > 0) xg_trsv_lt_update_kernel<<<k * ((T.ts + 255) / 256), 256, 0, st>>>(T, k, v, status);
}

/* ---- kriging: zmiss[m] = sum_o Sigma(miss_m, obs_o) alpha_o ---- */
__global__ void __launch_bounds__(256) xg_predict_cross_kernel(const double *__restrict__ xm,
                                                               const double *__restrict__ ym, int nmiss,
                                                               const double *__restrict__ xo,
                                                               const double *__restrict__ yo, int nobs,
                                                               const double *__restrict__ alpha, XgMaternParams p,
                                                               int metric, double *__restrict__ zmiss)
{
    __shared__ double red[8];
    const int m = blockIdx.x;
    double s = 0.0;
    if (p.bivariate) {
        /* rows and columns interleave the two variables: index 2 l + v */
        const double x1 = xm[m >> 1], y1 = ym[m >> 1];
        for (int o = threadIdx.x; o < nobs; o += blockDim.x)
            s += xg_matern_value_biv(xg_distance(x1, y1, xo[o >> 1], yo[o >> 1], metric), p, m & 1, o & 1) * alpha[o];
    } else {
        const double x1 = xm[m], y1 = ym[m];
        for (int o = threadIdx.x; o < nobs; o += blockDim.x)
            s += xg_matern_value(xg_distance(x1, y1, xo[o], yo[o], metric), p) * alpha[o];
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        zmiss[m] = t;
    }
}

void xg_launch_predict_cross(const double *xm, const double *ym, int nmiss, const double *xo, const double *yo,
                             int nobs, const double *alpha, const XgMaternParams &p, int metric, double *zmiss,
                             cudaStream_t st)
{
    if (nmiss <= 0) return;
    xg_predict_cross_kernel<<<nmiss, 256, 0, st>>>(xm, ym, nmiss, xo, yo, nobs, alpha, p, metric, zmiss);
}

__global__ void xg_mse_kernel(const double *__restrict__ za, const double *__restrict__ zm, int n, double *out)
{
    /* out[0] = the MSE; out[1], out[2] = the MSEs of the even and odd entries
     * (the two variables of a bivariate field, CORE_dmse_bivariate_starpu,
     * codelet_zmse_bivariate.c:22-51, averaged over n / 2 as MLE_dexact.c:845-847).
     * blockDim is even, so each thread sees entries of one parity only. */
    __shared__ double red[2][32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = za[i] - zm[i];
        s += d * d;
    }
    double se = (threadIdx.x & 1) ? 0.0 : s, so = (threadIdx.x & 1) ? s : 0.0;
    for (int off = 16; off > 0; off >>= 1) {
        se += __shfl_xor_sync(0xffffffffu, se, off);
        so += __shfl_xor_sync(0xffffffffu, so, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = se;
        red[1][threadIdx.x >> 5] = so;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double te = 0.0, to = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            te += red[0][w];
            to += red[1][w];
        }
        out[0] = (te + to) / n;
        const int half = n / 2;
        out[1] = half > 0 ? te / half : 0.0;
        out[2] = half > 0 ? to / half : 0.0;
    }
}

void xg_launch_mse(const double *zactual, const double *zmiss, int nmiss, double *out, cudaStream_t st)
{
    xg_mse_kernel<<<1, 1024, 0, st>>>(zactual, zmiss, nmiss, out);
}

/* ---- element-wise Matern of location pairs (diagnostics and tests) ---- */
__global__ void xg_matern_pairs_kernel(const double *x1, const double *y1, const double *x2, const double *y2, int n,
                                       XgMaternParams p, int metric, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = xg_matern_value(xg_distance(x1[i], y1[i], x2[i], y2[i], metric), p);
}

void xg_launch_matern_pairs(const double *x1, const double *y1, const double *x2, const double *y2, int n,
                            const XgMaternParams &p, int metric, double *out, cudaStream_t st)
{
    if (n <= 0) return;
    xg_matern_pairs_kernel<<<(n + 255) / 256, 256, 0, st>>>(x1, y1, x2, y2, n, p, metric, out);
}

__global__ void xg_bessel_kernel(const double *nu, const double *x, int n, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = xg_bessel_knu(nu[i], x[i]);
}

void xg_launch_bessel(const double *nu, const double *x, int n, double *out, cudaStream_t st)
{
    if (n <= 0) return;
    xg_bessel_kernel<<<(n + 255) / 256, 256, 0, st>>>(nu, x, n, out);
}
