/*
 * FP64-class trailing updates on the INT8 tensor cores (tcgen05 kind::i8).
 *
 * The banded mixed-precision scheme of the reference
 * (exageostat_exact/src/compute/psdportf.c:44-187) stores the off-band tiles
 * in FP32 and updates them with SGEMM; its error floor comes from FP32
 * storage and FP32 accumulation.  This file keeps every tile in FP64 and runs
 * the off-band trailing update A_ij -= L_ik L_jk^T as an error-free integer
 * product on sliced operands (the splitting of Ozaki, Ogita, Oishi & Rump,
 * Numer. Algorithms 59 (2012) 95-118, in the INT8 form of Ootomo, Ozaki &
 * Yokota, IJHPCA 38 (2024) 297-313):
 *
 *   every row r of a panel tile L_ik is scaled by s_r = max_c |L_ik[r][c]| / 127
 *   and written as four balanced digits in base 254,
 *       L_ik[r][c] = s_r (d0 + d1 / 254 + d2 / 254^2 + d3 / 254^3) + O(s_r 254^-3 / 2),
 *   |d_t| <= 127, so each digit plane is a signed 8-bit matrix;
 *
 *   the product of two rows is sum_{a, b} 254^-(a+b) D_a E_b^T.  The ten
 *   digit pairs with a + b <= 3 run on the tensor cores with exact S32
 *   accumulation into four "level" accumulators (a + b = 0..3), which the
 *   epilogue combines in FP64: U = s_r s_c sum_t 254^-t acc_t.
 *
 * The operands carry 8 + 3 x 7.99 ~ 32 significant bits relative to their row
 * maximum and the accumulation is exact, so the update error is that of a
 * ~32-bit fixed-point dot product -- far below FP32 storage, at the cost of 10
 * INT8 MMAs (= 2.5 TF32 passes) per FP64 product.  The S32 sums stay exact:
 * |level sum| <= 4 x 127^2 x ts < 2^31 for ts <= 16384.
 *
 * Kernels:
 *   xg_slice_panel_kernel : panel tiles (i, k), i > k -> four digit planes + row scales
 *   xg_sliced_gemm_kernel : persistent off-band update, 128 x 128 jobs, warp 0 TMA,
 *                           warp 1 MMA issue + TMEM (4 levels x 128 columns = all 512),
 *                           warps 2-9 epilogue (FP64 combine, C -= s_r s_c U)
 */
#include <stdint.h>

#include "xg_common.cuh"
#include "xg_kernels.h"
#include "xg_tcgen05.cuh"

#define XG_SL_BM 128
#define XG_SL_BN 128
#define XG_SL_BK 64 /* int8 per 64-byte swizzled row */
#define XG_SL_SLICES 4
#define XG_SL_LEVELS 4
#define XG_SL_THREADS 320
#define XG_SL_STAGES 3
#define XG_SL_BOX_BYTES (XG_SL_BM * XG_SL_BK)                           /* one digit plane, 128 rows */
#define XG_SL_STAGE_BYTES (2 * XG_SL_SLICES * XG_SL_BOX_BYTES)          /* A and B planes: 64 KB */
#define XG_SL_SMEM (XG_SL_STAGES * XG_SL_STAGE_BYTES + 1024 + 256)
#define XG_SL_RADIX 254.0
#define XG_SL_TOP 127.0

/* ========================================================================== */
/* panel slicing                                                              */
/* ========================================================================== */

/* One warp per panel row: rows of tiles k+1 .. nt-1 of column k.  Lane l owns
 * elements c * 128 + 4 l .. + 3 for every 128-column chunk c, so each load
 * instruction reads 1 KB of the row and each digit store writes 128 bytes. */
__global__ void __launch_bounds__(256) xg_slice_panel_kernel(XgTileArgs T, int k, int8_t *__restrict__ dig,
                                                             double *__restrict__ scale, long long plane,
                                                             const int *status)
{
    if (*(volatile const int *)status) return;
    const int ts = T.ts;
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    const long long nrows = (long long)(T.nt - k - 1) * ts;
    if (row >= nrows) return;
    const int i = k + 1 + (int)(row / ts), r = (int)(row % ts);
    const double *src = T.data + (xg_tile_index(i, k, T.nt) * ts + r) * (long long)ts;
    const int nch = ts / 128; /* <= 4 */
    double v[16];
    double m = 0.0;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (c < nch) {
            const double2 a = *reinterpret_cast<const double2 *>(src + c * 128 + 4 * lane);
            const double2 b = *reinterpret_cast<const double2 *>(src + c * 128 + 4 * lane + 2);
            v[4 * c] = a.x;
            v[4 * c + 1] = a.y;
            v[4 * c + 2] = b.x;
            v[4 * c + 3] = b.y;
            m = fmax(m, fmax(fmax(fabs(a.x), fabs(a.y)), fmax(fabs(b.x), fabs(b.y))));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const long long grow = (long long)i * ts + r; /* panel row index */
    const double c0 = m > 0.0 ? XG_SL_TOP / m : 0.0;
    if (lane == 0) scale[grow] = m / XG_SL_TOP;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (c < nch) {
            uint32_t w[XG_SL_SLICES] = {0u, 0u, 0u, 0u};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                double x = v[4 * c + e] * c0; /* |x| <= 127 */
#pragma unroll
                for (int t = 0; t < XG_SL_SLICES; ++t) {
                    double d = rint(x);
                    d = fmin(fmax(d, -XG_SL_TOP), XG_SL_TOP);
                    x = (x - d) * XG_SL_RADIX; /* remainder in [-1/2, 1/2] digit units, scaled to the next digit */
                    w[t] |= (uint32_t)(uint8_t)(int8_t)(int)d << (8 * e);
                }
            }
#pragma unroll
            for (int t = 0; t < XG_SL_SLICES; ++t)
                *reinterpret_cast<uint32_t *>(dig + t * plane + grow * ts + c * 128 + 4 * lane) = w[t];
        }
    }
}

/* ========================================================================== */
/* off-band trailing update: C64 -= s_r s_c sum_t 254^-t (sum_{a+b=t} D_a E_b^T) */
/* ========================================================================== */

struct XgSlJob {
    int i, j, bm, bn;
};

/* part 1: column k+1; part 2: columns >= k+2; part 0: columns >= k+1.  Targets
 * (i, j) with i - j >= band, each split into (ts / 128)^2 jobs of 128 x 128. */
__device__ inline XgSlJob xg_sl_decode(long long job, int ts, int band, int k, int part)
{
    const int bpt = ts / XG_SL_BM;
    const long long pair = job / (bpt * bpt);
    const int blk = (int)(job % (bpt * bpt));
    XgSlJob J;
    J.bm = blk / bpt;
    J.bn = blk % bpt;
    const int j0 = (part == 2) ? k + 2 : k + 1;
    if (part == 1) {
        J.j = j0;
        J.i = j0 + band + (int)pair;
    } else {
        int ii, jj;
        xg_pair_decode(pair, &ii, &jj);
        J.j = j0 + jj;
        J.i = j0 + band + ii;
    }
    return J;
}

/* digit pair p = 0..9 -> (a, b) with a + b <= 3, levels in order; the first
 * pair of each level (p = 0, 1, 3, 6) starts its accumulator */
__device__ __forceinline__ void xg_sl_pair(int p, int &a, int &b)
{
    /* (0,0) (0,1) (1,0) (0,2) (1,1) (2,0) (0,3) (1,2) (2,1) (3,0) */
    const int lv = p < 1 ? 0 : p < 3 ? 1 : p < 6 ? 2 : 3;
    const int first = lv * (lv + 1) / 2;
    a = p - first;
    b = lv - a;
}

__global__ void __launch_bounds__(XG_SL_THREADS, 1)
    xg_sliced_gemm_kernel(const __grid_constant__ CUtensorMap map, const double *__restrict__ scale,
                          XgTileArgs T, int band, int k, int part, long long njobs, int plane_rows, int *status)
{
    extern __shared__ __align__(1024) unsigned char xg_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)xg_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + XG_SL_STAGES * XG_SL_STAGE_BYTES);
    uint64_t *empty = full + XG_SL_STAGES;
    uint64_t *acc_full = empty + XG_SL_STAGES;
    uint64_t *acc_empty = acc_full + 1;
    uint64_t *drain = acc_empty + 1;
    uint32_t *tmem_slot = (uint32_t *)(drain + 1);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ts = T.ts;
    if (xg_cta_should_skip(status)) return;
    if (tid == 0) {
        for (int s = 0; s < XG_SL_STAGES; ++s) {
            xg_mbar_init(&full[s], 1);
            xg_mbar_init(&empty[s], 1);
        }
        xg_mbar_init(acc_full, 1);
        xg_mbar_init(acc_empty, 8);
        xg_mbar_init(drain, 1);
        xg_fence_barrier_init();
    }
    if (warp == 1) xg_tmem_alloc(tmem_slot, 512); /* four 128 x 128 S32 level accumulators */
    xg_tc_fence_before();
    __syncthreads();
    xg_tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int KT = ts / XG_SL_BK;
    bool ok = true;

    if (warp == 0) {
        /* ---- TMA producer: per stage the four A and four B digit boxes ---- */
        if (lane == 0) {
            xg_prefetch_tensormap(&map);
            long long it = 0;
            for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x) {
                const XgSlJob J = xg_sl_decode(job, ts, band, k, part);
                const int rowA = J.i * ts + J.bm * XG_SL_BM, rowB = J.j * ts + J.bn * XG_SL_BN;
                for (int kb = 0; kb < KT; ++kb, ++it) {
                    const int s = (int)(it % XG_SL_STAGES);
                    if (it >= XG_SL_STAGES &&
                        !xg_mbar_wait(&empty[s], (uint32_t)((it / XG_SL_STAGES) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    unsigned char *st = smem + s * XG_SL_STAGE_BYTES;
                    xg_mbar_arrive_expect_tx(&full[s], XG_SL_STAGE_BYTES);
#pragma unroll
                    for (int t = 0; t < XG_SL_SLICES; ++t) {
                        xg_tma_load_2d(st + t * XG_SL_BOX_BYTES, &map, kb * XG_SL_BK, t * plane_rows + rowA, &full[s]);
                        xg_tma_load_2d(st + (XG_SL_SLICES + t) * XG_SL_BOX_BYTES, &map, kb * XG_SL_BK,
                                       t * plane_rows + rowB, &full[s]);
                    }
                }
            }
            if (!ok) atomicOr(status, XG_ST_TIMEOUT);
            const long long first = it > XG_SL_STAGES ? it - XG_SL_STAGES : 0;
            for (long long q = first; q < it; ++q)
                xg_mbar_wait(&full[q % XG_SL_STAGES], (uint32_t)(q / XG_SL_STAGES) & 1);
        }
    } else if (warp == 1) {
        /* ---- MMA issuer ---- */
        if (lane == 0) {
            constexpr uint32_t idesc = xg_idesc_i8(XG_SL_BM, XG_SL_BN);
            const uint32_t sbase = xg_smem_u32(smem);
            long long it = 0;
            int jl = 0;
            for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x, ++jl) {
                if (jl >= 1 && !xg_mbar_wait(acc_empty, (uint32_t)(jl - 1) & 1)) {
                    ok = false;
                    break;
                }
                xg_tc_fence_after();
                for (int kb = 0; kb < KT; ++kb, ++it) {
                    const int s = (int)(it % XG_SL_STAGES);
                    if (!xg_mbar_wait(&full[s], (uint32_t)(it / XG_SL_STAGES) & 1)) {
                        ok = false;
                        break;
                    }
                    xg_tc_fence_after();
                    const uint32_t sa = sbase + s * XG_SL_STAGE_BYTES;
                    const uint32_t sb = sa + XG_SL_SLICES * XG_SL_BOX_BYTES;
#pragma unroll
                    for (int kk = 0; kk < XG_SL_BK / 32; ++kk) {
                        /* K = 32 int8 = 32 bytes per MMA inside the 64-byte swizzled row */
#pragma unroll
                        for (int p = 0; p < 10; ++p) {
                            int a, b;
                            xg_sl_pair(p, a, b);
                            const uint64_t ad = xg_umma_desc_sw64(sa + a * XG_SL_BOX_BYTES + kk * 32);
                            const uint64_t bd = xg_umma_desc_sw64(sb + b * XG_SL_BOX_BYTES + kk * 32);
                            const bool starts = (p == 0 || p == 1 || p == 3 || p == 6);
                            xg_umma_i8(tmem + (uint32_t)((a + b) * XG_SL_BN), ad, bd, idesc,
                                       (kb | kk) != 0 || !starts);
                        }
                    }
                    xg_umma_commit(&empty[s]);
                }
                if (!ok) break;
                xg_umma_commit(acc_full);
            }
            if (!ok) atomicOr(status, XG_ST_TIMEOUT);
            xg_umma_commit(drain);
            xg_mbar_wait(drain, 0);
        }
    } else {
        /* ---- epilogue: warps 2-9; TMEM lanes 32 (warp % 4) .. + 31, column half (warp - 2) / 4 ---- */
        const int q = warp & 3, h = (warp - 2) >> 2;
        const double inv = 1.0 / XG_SL_RADIX;
        int jl = 0;
        for (long long job = blockIdx.x; job < njobs; job += gridDim.x, ++jl) {
            if (!xg_mbar_wait(acc_full, (uint32_t)jl & 1)) {
                if (lane == 0) atomicOr(status, XG_ST_TIMEOUT);
                break;
            }
            xg_tc_fence_after();
            double res[64];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
#pragma unroll
                for (int t = XG_SL_LEVELS - 1; t >= 0; --t) {
                    uint32_t r[16];
                    xg_tmem_ld_32x32b_x16(tmem + ((uint32_t)(q * 32) << 16) +
                                              (uint32_t)(t * XG_SL_BN + h * 64 + c * 16),
                                          r);
                    xg_tmem_ld_wait();
#pragma unroll
                    for (int u = 0; u < 16; ++u) {
                        const double lv = (double)(int)r[u];
                        res[c * 16 + u] = (t == XG_SL_LEVELS - 1) ? lv : fma(res[c * 16 + u], inv, lv);
                    }
                }
            }
            /* the accumulators are free for the next job's MMAs */
            xg_tc_fence_before();
            __syncwarp();
            if (lane == 0) xg_mbar_arrive(acc_empty);
            const XgSlJob J = xg_sl_decode(job, ts, band, k, part);
            const int rl = J.bm * XG_SL_BM + q * 32 + lane;
            const double sr = scale[(long long)J.i * ts + rl];
            const double2 *sc = reinterpret_cast<const double2 *>(scale + (long long)J.j * ts + J.bn * XG_SL_BN + h * 64);
            double2 *C = reinterpret_cast<double2 *>(T.data + xg_tile_index(J.i, J.j, T.nt) * (long long)ts * ts +
                                                     (long long)rl * ts + J.bn * XG_SL_BN + h * 64);
            /* in groups of 8 column pairs: bounds how far the compiler hoists
             * the loads (registers hold the 64 results already) */
#pragma unroll
            for (int u0 = 0; u0 < 32; u0 += 8) {
#pragma unroll
                for (int u = u0; u < u0 + 8; ++u) {
                    const double2 s2 = sc[u];
                    double2 cv = C[u];
                    cv.x = fma(-sr * s2.x, res[2 * u], cv.x);
                    cv.y = fma(-sr * s2.y, res[2 * u + 1], cv.y);
                    C[u] = cv;
                }
                asm volatile("" ::: "memory");
            }
        }
    }
    xg_tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        xg_tc_fence_after();
        xg_tmem_dealloc(tmem, 512);
    }
}

/* ========================================================================== */
/* launchers                                                                  */
/* ========================================================================== */

cudaError_t xg_sliced_kernels_configure()
{
    return cudaFuncSetAttribute(xg_sliced_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, XG_SL_SMEM);
}

void xg_launch_slice_panel(const XgTileArgs &T, int k, int8_t *dig, double *scale, long long plane, const int *status,
                           cudaStream_t st)
{
    const long long rows = (long long)(T.nt - k - 1) * T.ts;
    if (rows <= 0) return;
    xg_slice_panel_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(T, k, dig, scale, plane, status);
}

void xg_launch_sliced_gemm(const CUtensorMap &map, const double *scale, const XgTileArgs &T, int band, int k,
                           int part, int plane_rows, int sm_count, int *status, cudaStream_t st)
{
    const int j0 = (part == 2) ? k + 2 : k + 1;
    const long long rows = (long long)T.nt - j0 - band; /* tiles in the first target column */
    if (rows <= 0) return;
    const long long pairs = (part == 1) ? rows : rows * (rows + 1) / 2;
    const long long bpt = T.ts / XG_SL_BM;
    const long long njobs = pairs * bpt * bpt;
    const unsigned grid = (unsigned)(njobs < sm_count ? njobs : sm_count);
    xg_sliced_gemm_kernel<<<grid, XG_SL_THREADS, XG_SL_SMEM, st>>>(map, scale, T, band, k, part, njobs, plane_rows,
                                                                   status);
}
