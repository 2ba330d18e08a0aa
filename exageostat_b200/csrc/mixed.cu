/*
 * Banded mixed-precision factorisation (precision = 2) on sm_100a.
 *
 * The reference's mixed scheme (exageostat_exact/src/compute/psdportf.c:44-187,
 * driven by EXAGEOSTAT_sdmle_Tile, MLE_sdexact.c:172-357) keeps tiles with
 * |m - n| < diag_thick in FP64 and does the rest in FP32 (SGEMM / STRSM),
 * with POTRF, log-det, the solve and the dot product in FP64.  Here:
 *
 *   band tiles (0 <= i - j < band)  FP64 storage; POTRF, TRSM and their
 *                                   trailing updates on FP64 DMMA
 *   off-band tiles                  FP32 storage; TRSM in FP64 arithmetic,
 *                                   rounded to FP32; trailing updates on the
 *                                   5th-generation tensor cores (tcgen05,
 *                                   kind::tf32, accumulators in TMEM) with
 *                                   one TF32 pass or three (hi/lo split:
 *                                   a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32-class
 *                                   products)
 *   log-det, z solve, quadratic form FP64, fused into POTRF / TRSM as in the
 *                                   FP64 path
 *
 * After the panel of step k is solved, xg_panel_prep_kernel writes it once
 * into three row-major panel buffers indexed by tile row i: an FP64 copy (the
 * DMMA operands of band targets) and the TF32 hi / lo parts (FP32 containers,
 * the tcgen05 operands).  The reference's mixed path has signature and type
 * defects (sdpotrf.c:292 vs psdportf.c:44; codelet_exageostat_sgemm.c:95), so
 * results are compared with the FP64 path, not with it.
 */
#include <math.h>
#include <stdint.h>

#include "kbessel.cuh"
#include "xg_common.cuh"
#include "xg_kernels.h"
#include "xg_matern.cuh"
#include "xg_tcgen05.cuh"

/* ========================================================================== */
/* generation into the band (FP64) / off-band (FP32) stores                   */
/* ========================================================================== */

#define XG_MG_ROWS 8
__global__ void __launch_bounds__(256) xg_gen_mixed_kernel(XgTileArgs T, const int2 *__restrict__ tile_ij,
                                                           const double *__restrict__ x, const double *__restrict__ y,
                                                           int n, XgMaternParams p, int metric)
{
    const int ts = T.ts;
    const int strips = ts / XG_MG_ROWS;
    const long long t = blockIdx.x / strips;
    const int strip = blockIdx.x % strips;
    const int2 ij = tile_ij[t];
    const bool band = ij.x - ij.y < T.band;
    double *t64 = band ? T.data + xg_slot64(T, ij.x, ij.y) * (long long)ts * ts : nullptr;
    float *t32 = band ? nullptr : T.data32 + xg_slot32(ij.x, ij.y, T.nt, T.band) * (long long)ts * ts;
    for (int rr = 0; rr < XG_MG_ROWS; ++rr) {
        const int r = strip * XG_MG_ROWS + rr;
        const int R = ij.x * ts + r;
        const bool row_ok = R < n;
        const double x1 = row_ok ? x[R] : 0.0, y1 = row_ok ? y[R] : 0.0;
        for (int c = threadIdx.x; c < ts; c += blockDim.x) {
            const int C = ij.y * ts + c;
            double val;
            if (row_ok && C < n)
                val = xg_matern_value(xg_distance(x1, y1, x[C], y[C], metric), p);
            else
                val = (R == C) ? 1.0 : 0.0;
            if (band)
                t64[(long long)r * ts + c] = val;
            else
                t32[(long long)r * ts + c] = (float)val;
        }
    }
}

/* ========================================================================== */
/* panel TRSM on FP32 off-band tiles: L_ik = A_ik L_kk^-T (FP64 arithmetic)   */
/* ========================================================================== */

#define XG_T32_THREADS 512
#define XG_T32_SR 32

__global__ void __launch_bounds__(XG_T32_THREADS) xg_trsm_panel32_kernel(XgTileArgs T, int k, int i0,
                                                                          double *__restrict__ v, int with_rhs,
                                                                          const int *status)
{
    const int ts = T.ts, LDS = ts + 4;
    extern __shared__ __align__(16) double xg_smem_d[];
    double *S = xg_smem_d;
    double *LD = S + XG_T32_SR * LDS;
    if (xg_cta_should_skip(status)) return;
    const int strips = ts / XG_T32_SR;
    const int i = i0 + blockIdx.x / strips;
    const int strip = blockIdx.x % strips;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tq = lane & 3;
    float *B = T.data32 + xg_slot32(i, k, T.nt, T.band) * (long long)ts * ts + (long long)strip * XG_T32_SR * ts;
    const double *L = T.data + xg_slot64(T, k, k) * (long long)ts * ts;
    for (int idx = tid; idx < XG_T32_SR * ts; idx += blockDim.x) {
        const int r = idx / ts, c = idx - r * ts;
        S[r * LDS + c] = (double)B[(long long)r * ts + c];
    }
    for (int cb = 0; cb < ts; cb += 32) {
        for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
            const int r = idx >> 5, c = idx & 31;
            LD[r * 33 + c] = L[(long long)(cb + r) * ts + cb + c];
        }
        __syncthreads();
        if (warp == 0) {
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
        const int ngrp = (ts - cb - 32) / 32;
        for (int grp = warp; grp < ngrp; grp += XG_T32_THREADS / 32) {
            const int c0 = cb + 32 + grp * 32;
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
    /* store rounded to FP32 and keep the rounded values for the z update, so
     * the solve uses exactly the stored factor */
    for (int idx = tid; idx < XG_T32_SR * ts; idx += blockDim.x) {
        const int r = idx / ts, c = idx - r * ts;
        const float f = (float)S[r * LDS + c];
        B[(long long)r * ts + c] = f;
        S[r * LDS + c] = (double)f;
    }
    __syncthreads();
    if (with_rhs) {
        const double *vk = v + (long long)k * ts;
        double *vi = v + (long long)i * ts + strip * XG_T32_SR;
        for (int r = warp; r < XG_T32_SR; r += XG_T32_THREADS / 32) {
            double s = 0.0;
            for (int c = lane; c < ts; c += 32) s += S[r * LDS + c] * vk[c];
            for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            if (lane == 0) vi[r] -= s;
        }
    }
}

/* ========================================================================== */
/* panel prep: L_ik (i > k) -> FP64 copy, TF32 hi and lo parts                */
/* ========================================================================== */

__global__ void __launch_bounds__(256) xg_panel_prep_kernel(XgTileArgs T, int k, double *__restrict__ p64,
                                                            float *__restrict__ phi, float *__restrict__ plo,
                                                            int passes, const int *status)
{
    if (*(volatile const int *)status) return;
    const int ts = T.ts;
    const int i = k + 1 + blockIdx.y;
    const long long per_tile = (long long)ts * ts;
    const bool band = i - k < T.band;
    const double *s64 = band ? T.data + xg_slot64(T, i, k) * per_tile : nullptr;
    const float *s32 = band ? nullptr : T.data32 + xg_slot32(i, k, T.nt, T.band) * per_tile;
    double *d64 = p64 + (long long)i * per_tile;
    float *dhi = phi + (long long)i * per_tile;
    float *dlo = plo + (long long)i * per_tile;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < per_tile;
         e += (long long)gridDim.x * blockDim.x) {
        const double vd = band ? s64[e] : (double)s32[e];
        d64[e] = vd;
        const float vf = (float)vd;
        const float hi = xg_to_tf32(vf); /* round once to TF32 (the MMA would truncate) */
        dhi[e] = hi;
        if (passes == 3) dlo[e] = vf - hi;
    }
}

/* ========================================================================== */
/* off-band trailing update on tcgen05: C32 -= A B^T (1 or 3 TF32 passes)     */
/* ========================================================================== */

#define XG_OB_BM 128
#define XG_OB_BN 256
#define XG_OB_BK 32 /* FP32 per 128-byte swizzled row */
#define XG_OB_THREADS 192
#define XG_OB_A_BYTES (XG_OB_BM * XG_OB_BK * 4)
#define XG_OB_B_BYTES (XG_OB_BN * XG_OB_BK * 4)

template <int PASSES>
struct XgObCfg {
    static constexpr int STAGES = PASSES == 3 ? 2 : 4;
    static constexpr int STAGE_BYTES = (XG_OB_A_BYTES + XG_OB_B_BYTES) * (PASSES == 3 ? 2 : 1);
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024 /* align */ + 256 /* barriers */;
};

struct XgObJob {
    int i, j, bm, bn;
};

/* part 1: column k+1; part 2: columns >= k+2; part 0: columns >= k+1 */
__device__ inline XgObJob xg_ob_decode(long long job, int nt, int ts, int band, int k, int part)
{
    const int bpm = ts / XG_OB_BM, bpn = ts / XG_OB_BN;
    const long long pair = job / (bpm * bpn);
    const int blk = (int)(job % (bpm * bpn));
    XgObJob J;
    J.bm = blk / bpn;
    J.bn = blk % bpn;
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

template <int PASSES>
__global__ void __launch_bounds__(XG_OB_THREADS, 1)
    xg_offband_gemm_kernel(const __grid_constant__ CUtensorMap m_ahi, const __grid_constant__ CUtensorMap m_bhi,
                           const __grid_constant__ CUtensorMap m_alo, const __grid_constant__ CUtensorMap m_blo,
                           float *__restrict__ T32, int nt, int ts, int band, int k, int part, long long njobs,
                           int *status)
{
    using Cfg = XgObCfg<PASSES>;
    constexpr int STAGES = Cfg::STAGES;
    extern __shared__ __align__(1024) unsigned char xg_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)xg_smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t *full = (uint64_t *)(smem + STAGES * Cfg::STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;
    uint64_t *acc_empty = acc_full + 2;
    uint64_t *drain = acc_empty + 2;
    uint32_t *tmem_slot = (uint32_t *)(drain + 1);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (xg_cta_should_skip(status)) return;
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            xg_mbar_init(&full[s], 1);
            xg_mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            xg_mbar_init(&acc_full[a], 1);
            xg_mbar_init(&acc_empty[a], 4);
        }
        xg_mbar_init(drain, 1);
        xg_fence_barrier_init();
    }
    if (warp == 1) xg_tmem_alloc(tmem_slot, 512); /* two 128 x 256 FP32 accumulators */
    xg_tc_fence_before();
    __syncthreads();
    xg_tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int KT = ts / XG_OB_BK;
    bool ok = true;

    if (warp == 0) {
        /* ---- TMA producer ---- */
        if (lane == 0) {
            xg_prefetch_tensormap(&m_ahi);
            xg_prefetch_tensormap(&m_bhi);
            long long it = 0;
            for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x) {
                const XgObJob J = xg_ob_decode(job, nt, ts, band, k, part);
                const int rowA = J.i * ts + J.bm * XG_OB_BM, rowB = J.j * ts + J.bn * XG_OB_BN;
                for (int kb = 0; kb < KT; ++kb, ++it) {
                    const int s = (int)(it % STAGES);
                    if (it >= STAGES && !xg_mbar_wait(&empty[s], (uint32_t)((it / STAGES) - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    unsigned char *st = smem + s * Cfg::STAGE_BYTES;
                    xg_mbar_arrive_expect_tx(&full[s], Cfg::STAGE_BYTES);
                    xg_tma_load_2d(st, &m_ahi, kb * XG_OB_BK, rowA, &full[s]);
                    xg_tma_load_2d(st + XG_OB_A_BYTES, &m_bhi, kb * XG_OB_BK, rowB, &full[s]);
                    if (PASSES == 3) {
                        xg_tma_load_2d(st + XG_OB_A_BYTES + XG_OB_B_BYTES, &m_alo, kb * XG_OB_BK, rowA, &full[s]);
                        xg_tma_load_2d(st + 2 * XG_OB_A_BYTES + XG_OB_B_BYTES, &m_blo, kb * XG_OB_BK, rowB,
                                       &full[s]);
                    }
                }
            }
            if (!ok) atomicOr(status, XG_ST_TIMEOUT);
            /* the copies in flight land before the CTA may exit */
            const long long first = it > STAGES ? it - STAGES : 0;
            for (long long q = first; q < it; ++q) xg_mbar_wait(&full[q % STAGES], (uint32_t)(q / STAGES) & 1);
        }
    } else if (warp == 1) {
        /* ---- MMA issuer ---- */
        if (lane == 0) {
            constexpr uint32_t idesc = xg_idesc_tf32(XG_OB_BM, XG_OB_BN);
            const uint32_t sbase = xg_smem_u32(smem);
            long long it = 0;
            int jl = 0;
            for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x, ++jl) {
                const int a = jl & 1;
                if (jl >= 2 && !xg_mbar_wait(&acc_empty[a], (uint32_t)((jl >> 1) - 1) & 1)) {
                    ok = false;
                    break;
                }
                xg_tc_fence_after();
                const uint32_t dt = tmem + (uint32_t)(a * XG_OB_BN);
                for (int kb = 0; kb < KT; ++kb, ++it) {
                    const int s = (int)(it % STAGES);
                    if (!xg_mbar_wait(&full[s], (uint32_t)(it / STAGES) & 1)) {
                        ok = false;
                        break;
                    }
                    xg_tc_fence_after();
                    const uint32_t sa = sbase + s * Cfg::STAGE_BYTES;
                    const uint32_t sb = sa + XG_OB_A_BYTES;
                    const uint32_t sal = sa + XG_OB_A_BYTES + XG_OB_B_BYTES;
                    const uint32_t sbl = sal + XG_OB_A_BYTES;
#pragma unroll
                    for (int kk = 0; kk < XG_OB_BK / 8; ++kk) {
                        /* K = 8 TF32 = 32 bytes per MMA: advance the start address inside the swizzled row */
                        const uint64_t ahi = xg_umma_desc_sw128(sa + kk * 32);
                        const uint64_t bhi = xg_umma_desc_sw128(sb + kk * 32);
                        xg_umma_tf32(dt, ahi, bhi, idesc, (kb | kk) != 0);
                        if (PASSES == 3) {
                            xg_umma_tf32(dt, ahi, xg_umma_desc_sw128(sbl + kk * 32), idesc, 1);
                            xg_umma_tf32(dt, xg_umma_desc_sw128(sal + kk * 32), bhi, idesc, 1);
                        }
                    }
                    xg_umma_commit(&empty[s]); /* frees the stage when these MMAs are done */
                }
                if (!ok) break;
                xg_umma_commit(&acc_full[a]);
            }
            if (!ok) atomicOr(status, XG_ST_TIMEOUT);
            /* every MMA issued here completes before TMEM is released */
            xg_umma_commit(drain);
            xg_mbar_wait(drain, 0);
        }
    } else {
        /* ---- epilogue: warps 2-5, TMEM lanes 32 (warp % 4) .. +31 ---- */
        const int lg = warp & 3;
        /* brings the next job's C row (256 FP32 of one row per thread) into L2
         * while this job's accumulator is drained */
        auto prefetch_c = [&](long long jb) {
            if (jb >= njobs) return;
            const XgObJob J = xg_ob_decode(jb, nt, ts, band, k, part);
            const float *p = T32 + xg_slot32(J.i, J.j, nt, band) * (long long)ts * ts +
                             (long long)(J.bm * XG_OB_BM + lg * 32 + lane) * ts + J.bn * XG_OB_BN;
#pragma unroll
            for (int l = 0; l < 8; ++l) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + 32 * l));
        };
        prefetch_c(blockIdx.x);
        int jl = 0;
        for (long long job = blockIdx.x; job < njobs; job += gridDim.x, ++jl) {
            const int a = jl & 1;
            prefetch_c(job + gridDim.x);
            if (!xg_mbar_wait(&acc_full[a], (uint32_t)(jl >> 1) & 1)) {
                if (lane == 0) atomicOr(status, XG_ST_TIMEOUT);
                break;
            }
            xg_tc_fence_after();
            const XgObJob J = xg_ob_decode(job, nt, ts, band, k, part);
            float *C = T32 + xg_slot32(J.i, J.j, nt, band) * (long long)ts * ts +
                       (long long)(J.bm * XG_OB_BM + lg * 32 + lane) * ts + J.bn * XG_OB_BN;
#pragma unroll 1
            for (int cc = 0; cc < XG_OB_BN / 32; ++cc) {
                uint32_t r[32];
                xg_tmem_ld_32x32b_x32(tmem + (uint32_t)(a * XG_OB_BN + cc * 32) + ((uint32_t)(lg * 32) << 16), r);
                xg_tmem_ld_wait();
                float4 *pc = reinterpret_cast<float4 *>(C + cc * 32);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    float4 cv = pc[q];
                    cv.x -= __uint_as_float(r[4 * q + 0]);
                    cv.y -= __uint_as_float(r[4 * q + 1]);
                    cv.z -= __uint_as_float(r[4 * q + 2]);
                    cv.w -= __uint_as_float(r[4 * q + 3]);
                    pc[q] = cv;
                }
            }
            xg_tc_fence_before();
            __syncwarp();
            if (lane == 0) xg_mbar_arrive(&acc_empty[a]);
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

size_t xg_trsm32_smem_bytes(int ts) { return ((size_t)XG_T32_SR * (ts + 4) + 32 * 33) * sizeof(double); }

cudaError_t xg_mixed_kernels_configure()
{
    cudaError_t e = cudaFuncSetAttribute(xg_offband_gemm_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         XgObCfg<1>::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(xg_offband_gemm_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 XgObCfg<3>::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(xg_trsm_panel32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)xg_trsm32_smem_bytes(XG_MAX_TS));
    return e;
}

void xg_launch_gen_mixed(const XgTileArgs &T, const int2 *tile_ij, long long ntiles, const double *x, const double *y,
                         int n, const XgMaternParams &p, int metric, cudaStream_t st)
{
    xg_gen_mixed_kernel<<<(unsigned)(ntiles * (T.ts / XG_MG_ROWS)), 256, 0, st>>>(T, tile_ij, x, y, n, p, metric);
}

void xg_launch_trsm_panel32(const XgTileArgs &T, int k, double *v, int with_rhs, const int *status, cudaStream_t st)
{
    const int i0 = k + T.band;
    const int n = T.nt - i0;
    if (n <= 0) return;
    xg_trsm_panel32_kernel<<<n * (T.ts / XG_T32_SR), XG_T32_THREADS, xg_trsm32_smem_bytes(T.ts), st>>>(T, k, i0, v,
                                                                                                      with_rhs, status);
}

void xg_launch_panel_prep(const XgTileArgs &T, int k, double *p64, float *phi, float *plo, int passes,
                          const int *status, cudaStream_t st)
{
    const int n = T.nt - k - 1;
    if (n <= 0) return;
    xg_panel_prep_kernel<<<dim3(32, n), 256, 0, st>>>(T, k, p64, phi, plo, passes, status);
}

void xg_launch_offband_gemm(const XgMixedMaps &maps, const XgTileArgs &T, int k, int part, int passes, int sm_count,
                            int *status, cudaStream_t st)
{
    const int j0 = (part == 2) ? k + 2 : k + 1;
    const long long rows = (long long)T.nt - j0 - T.band; /* tiles in the first target column */
    if (rows <= 0) return;
    const long long pairs = (part == 1) ? rows : rows * (rows + 1) / 2;
    const long long njobs = pairs * (T.ts / XG_OB_BM) * (T.ts / XG_OB_BN);
    const unsigned grid = (unsigned)(njobs < sm_count ? njobs : sm_count);
    if (passes == 3)
        xg_offband_gemm_kernel<3><<<grid, XG_OB_THREADS, XgObCfg<3>::SMEM, st>>>(
            maps.ahi, maps.bhi, maps.alo, maps.blo, T.data32, T.nt, T.ts, T.band, k, part, njobs, status);
    else
        xg_offband_gemm_kernel<1><<<grid, XG_OB_THREADS, XgObCfg<1>::SMEM, st>>>(
            maps.ahi, maps.bhi, maps.alo, maps.blo, T.data32, T.nt, T.ts, T.band, k, part, njobs, status);
}
