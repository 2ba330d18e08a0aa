/*
 * Shared device helpers: lower-tile indexing, error words, and the sm_100a
 * PTX wrappers (mbarrier, TMA bulk-tensor loads, FP64 DMMA).
 */
#ifndef EXAGEOSTAT_B200_COMMON_CUH
#define EXAGEOSTAT_B200_COMMON_CUH

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

/* ---- status word bits (device int written by kernels, read by the host) ---- */
#define XG_ST_NOT_SPD 1   /* a non-positive or NaN pivot; info holds the 1-based column */
#define XG_ST_TIMEOUT 2   /* a bounded wait gave up (pipeline stall) */
#define XG_ST_BAD_ARG 4

/* Lower tile (i, j), j <= i, of an nt x nt tile grid in column-packed order. */
__host__ __device__ inline long long xg_tile_index(int i, int j, int nt)
{
    return (long long)j * nt - (long long)j * (j - 1) / 2 + (i - j);
}

__host__ __device__ inline long long xg_num_lower_tiles(int nt) { return (long long)nt * (nt + 1) / 2; }

/* pair index p = ii (ii + 1) / 2 + jj, jj <= ii  ->  (ii, jj) */
__device__ inline void xg_pair_decode(long long p, int *ii, int *jj)
{
    int i = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while ((long long)(i + 1) * (i + 2) / 2 <= p) ++i;
    while ((long long)i * (i + 1) / 2 > p) --i;
    *ii = i;
    *jj = (int)(p - (long long)i * (i + 1) / 2);
}

__device__ inline uint32_t xg_smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ inline uint64_t xg_globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

/* CTA-uniform read of the device status word: thread 0 reads it once and the
 * whole CTA takes the same branch (kernels that use __syncthreads must not
 * let a few threads leave early). */
__device__ inline bool xg_cta_should_skip(const int *status, bool extra = false)
{
    __shared__ int s_skip;
    __syncthreads();
    if (threadIdx.x == 0) s_skip = (extra || *(volatile const int *)status != 0) ? 1 : 0;
    __syncthreads();
    return s_skip != 0;
}

/* ---- mbarrier ---- */
__device__ inline void xg_mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(xg_smem_u32(bar)), "r"(count) : "memory");
}

__device__ inline void xg_fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ inline void xg_fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ inline void xg_mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(xg_smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ inline void xg_mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(xg_smem_u32(bar)) : "memory");
}

__device__ inline bool xg_mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(xg_smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

/* Waits for the phase with the given parity; gives up after `limit_ns`
 * nanoseconds of wall time and returns false (the caller records a timeout). */
__device__ inline bool xg_mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = 2000000000ull)
{
    if (xg_mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = xg_globaltimer_ns();
    for (uint32_t it = 0;; ++it) {
        if (xg_mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 255u && xg_globaltimer_ns() - t0 > limit_ns) return false;
    }
}

/* ---- TMA: 2-D tiled bulk-tensor load into shared memory ---- */
__device__ inline void xg_tma_load_2d(void *smem_dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            xg_smem_u32(smem_dst)),
        "l"(map), "r"(x), "r"(y), "r"(xg_smem_u32(bar))
        : "memory");
}

/* ---- untiled bulk copy, global -> this CTA's shared memory, completing on an
 * mbarrier (both addresses 16-byte aligned, bytes a multiple of 16) ---- */
__device__ inline void xg_bulk_load(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     xg_smem_u32(smem_dst)),
                 "l"(gsrc), "r"(bytes), "r"(xg_smem_u32(bar))
                 : "memory");
}

__device__ inline void xg_prefetch_tensormap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

/* ---- FP64 tensor-core MMA (DMMA), D = A * B + D, m16n8k4 ----
 * Fragment ownership (g = lane / 4, t = lane % 4):
 *   A (16x4, row):  a0 = A[g][t],  a1 = A[g+8][t]
 *   B (4x8, col):   b0 = B[t][g]
 *   C (16x8):       c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1] */
__device__ inline void xg_dmma_16x8x4(double &c0, double &c1, double &c2, double &c3, double a0, double a1, double b0)
{
    asm("mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, {%0,%1,%2,%3};"
                 : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
                 : "d"(a0), "d"(a1), "d"(b0));
}

/* 128-byte swizzled row-major staging (TMA SWIZZLE_128B): element (row, k) of a
 * [rows][16] FP64 box lives at byte row*128 + (((k>>1) ^ (row&7)) << 4) + (k&1)*8. */
__device__ inline int xg_swz128_off(int row, int k) { return (row << 7) + ((((k >> 1) ^ (row & 7))) << 4) + ((k & 1) << 3); }

#endif
