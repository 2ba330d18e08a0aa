/*
 * sm_100a tensor-core (tcgen05) helpers: TMEM allocation, shared-memory
 * matrix descriptors, the kind::tf32 and kind::i8 MMAs, commit-to-mbarrier
 * and TMEM loads.
 * Only single-CTA (cta_group::1) forms are used.
 */
#ifndef EXAGEOSTAT_B200_TCGEN05_CUH
#define EXAGEOSTAT_B200_TCGEN05_CUH

#include <stdint.h>

#include "xg_common.cuh"

/* Shared-memory matrix descriptor for a K-major operand staged by TMA with
 * the 128-byte swizzle: rows of 128 B, 8-row (1024 B) swizzle atoms stacked
 * along M/N.  Fields: start address >> 4 [0,14), leading byte offset >> 4
 * [16,30) (unused for swizzled K-major, set to 1), stride byte offset >> 4
 * [32,46) = 1024 B between 8-row groups, version [46,48) = 1, base offset
 * [49,52) = 0 (atoms are 1024-B aligned), layout [61,64) = 2 (128-byte swizzle). */
__device__ inline uint64_t xg_umma_desc_sw128(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)2u << 61;
    return d;
}

/* The same for a K-major operand staged with the 64-byte swizzle: rows of
 * 64 B, 8-row (512 B) atoms, stride byte offset 512 B, layout [61,64) = 4. */
__device__ inline uint64_t xg_umma_desc_sw64(uint32_t smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;
    d |= (uint64_t)((512u >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    d |= (uint64_t)4u << 61;
    return d;
}

/* Instruction descriptor, kind::i8: D = S32 (2 at [4,6)), A = B = signed
 * 8-bit (1 at [7,10) and [10,13)), both K-major, no saturation, dense;
 * N >> 3 at [17,23), M >> 4 at [24,29). */
__host__ __device__ constexpr uint32_t xg_idesc_i8(int M, int N)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

/* Instruction descriptor, kind::tf32: D = F32, A = B = TF32, both K-major,
 * no negation, dense; N >> 3 at [17,23), M >> 4 at [24,29). */
__host__ __device__ constexpr uint32_t xg_idesc_tf32(int M, int N)
{
    return (1u << 4)            /* D format F32 */
           | (2u << 7)          /* A format TF32 */
           | (2u << 10)         /* B format TF32 */
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ inline void xg_tmem_alloc(uint32_t *smem_result, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(xg_smem_u32(smem_result)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ inline void xg_tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ inline void xg_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ inline void xg_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

/* D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread */
__device__ inline void xg_umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

/* D[tmem] (+)= A[smem] * B[smem]^T on signed 8-bit operands, S32 accumulators
 * (exact: no rounding, wraps only past 2^31) */
__device__ inline void xg_umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

/* arrives (once) on the mbarrier when every MMA this thread issued so far is complete */
__device__ inline void xg_umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(xg_smem_u32(bar))
                 : "memory");
}

/* 32 lanes x 32 consecutive 32-bit columns: thread t of the warp gets lane
 * (base lane + t), columns col .. col + 31 */
__device__ inline void xg_tmem_ld_32x32b_x32(uint32_t taddr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
}

/* 32 lanes x 8 consecutive 32-bit columns */
__device__ inline void xg_tmem_ld_32x32b_x8(uint32_t taddr, uint32_t (&r)[8])
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr)
                 : "memory");
}

/* 32 lanes x 16 consecutive 32-bit columns */
__device__ inline void xg_tmem_ld_32x32b_x16(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}

__device__ inline void xg_tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

/* FP32 -> TF32 (round to nearest, ties away), kept in an FP32 container */
__device__ inline float xg_to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

#endif
