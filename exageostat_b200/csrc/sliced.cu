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
 * Schedule (left-looking): the target tiles of column j receive the whole
 * update A_ij -= sum_{k<j} L_ik L_jk^T in one pass, chunk by chunk over the
 * panels k; the S32 levels restart for every chunk (each panel row has its
 * own scale) and the scaled chunk products accumulate in FP64 registers, so
 * every FP64 tile is read and written once per column instead of once per
 * step (the right-looking order would move 16 bytes per trailing element
 * per step, ~5 TB at N = 100,000).  The digit planes of every factored panel
 * tile are kept (tile-packed, 4 bytes per element).
 *
 * Kernels:
 *   xg_slice_panel_kernel : panel tiles (i, k), i > k (or the slots (k, a), a <= k, of the
 *                           inverse factor) -> four digit planes + row scales
 *   xg_sliced_left_kernel : persistent update of the targets (i, j), i >= j, from the
 *                           panels k0 <= k < k1; 128 x 128 jobs; warp 0 TMA, warp 1 MMA
 *                           issue + TMEM (4 levels x 128 columns = all 512), warps 4-11
 *                           epilogue (FP64 combine per chunk into 64 sums per thread,
 *                           one C -= update per job); setmaxnreg moves the registers of
 *                           warpgroup 0 to the epilogue.
 *                           The MMA computes the transposed block so that a TMEM lane
 *                           holds a column of C and the accesses to C are coalesced.
 */
#include <stdint.h>

#include "xg_common.cuh"
#include "xg_kernels.h"
#include "xg_tcgen05.cuh"

#define XG_SL_BM 128 /* C rows per job (rows of the A operand, the MMA's N) */
#define XG_SL_BN 128 /* C columns per job (rows of the B operand, the MMA's M) */
#define XG_SL_BK 64  /* int8 per 64-byte swizzled row */
#define XG_SL_SLICES 4
#define XG_SL_LEVELS 4 /* level sums |L_t| <= (t + 1) 127^2 ts stay exact in S32 */
#define XG_SL_EPI_WARPS 8
#define XG_SL_THREADS 384 /* warpgroup 0: TMA, MMA, 2 idle warps; warpgroups 1-2: epilogue */
/* register split (setmaxnreg): launched at 168 per thread (64,512 in all);
 * warpgroup 0 drops to 40, the epilogue warpgroups rise to 232:
 * 128 x 40 + 256 x 232 = 64,512 */
#define XG_SL_REG_LOW 40
#define XG_SL_REG_HIGH 232
#define XG_SL_STAGES 3
#define XG_SL_ABOX_BYTES (XG_SL_BM * XG_SL_BK)                                  /* one digit plane, 128 rows */
#define XG_SL_BBOX_BYTES (XG_SL_BN * XG_SL_BK)                                  /* one digit plane, 128 rows */
#define XG_SL_STAGE_BYTES (XG_SL_SLICES * (XG_SL_ABOX_BYTES + XG_SL_BBOX_BYTES)) /* 64 KB */
/* per panel chunk, the 128 A-row and 128 B-row scales, double-buffered */
#define XG_SL_SCALE_BYTES (2 * 2 * 128 * 8)
#define XG_SL_SMEM (XG_SL_STAGES * XG_SL_STAGE_BYTES + XG_SL_SCALE_BYTES + 1024 + 256)
#define XG_SL_RADIX 254.0
#define XG_SL_TOP 127.0
#define XG_SL_INV_RADIX3 (1.0 / (254.0 * 254.0 * 254.0))

/* Exact integer -> FP64 by the magic-number method: the integer is added to
 * the low mantissa bits of a double with a fixed exponent and the constant is
 * subtracted (one integer add and one FP64 add, no conversion instruction). */
/* |x| < 2^51 */
__device__ __forceinline__ double xg_i64_to_f64(long long x)
{
    /* (2^52 + 2^51 + x) - (2^52 + 2^51) */
    return __longlong_as_double(0x4338000000000000LL + x) - 6755399441055744.0;
}

/* ========================================================================== */
/* panel slicing                                                              */
/* ========================================================================== */

/* One warp per panel row: rows of tiles k+1 .. nt-1 of column k.  Lane l owns
 * elements c * 128 + 4 l .. + 3 for every 128-column chunk c, so each load
 * instruction reads 1 KB of the row and each digit store writes 128 bytes. */
__global__ void __launch_bounds__(256) xg_slice_panel_kernel(XgTileArgs T, int k, int row_mode,
                                                             int8_t *__restrict__ dig, double *__restrict__ scale,
                                                             long long plane, const int *status)
{
    if (*(volatile const int *)status) return;
    const int ts = T.ts;
    const int lane = threadIdx.x & 31;
    const long long row = (long long)blockIdx.x * 8 + (threadIdx.x >> 5);
    /* column mode: tiles (i, k), i > k; row mode: slots (k, a), a <= k */
    const long long nrows = (long long)(row_mode ? k + 1 : T.nt - k - 1) * ts;
    if (row >= nrows) return;
    const int u = (int)(row / ts), r = (int)(row % ts);
    const long long slot = row_mode ? xg_tile_index(k, u, T.nt) : xg_tile_index(k + 1 + u, k, T.nt);
    const double *src = T.data + (slot * ts + r) * (long long)ts;
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
    const long long grow = slot * ts + r; /* tile-packed row index */
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

/* One job: a 128 x 128 block (bm, bn) of an output tile, summed over the
 * panel chunks k0 <= k < k1; operand tiles are packed slots of the digit
 * stores and the output a packed slot of the FP64 store. */
struct XgSlJob {
    int ta, tb;       /* tile rows (A) and columns (B) index the operand slots */
    int bm, bn, k0, k1;
    long long c_slot;
};

/* job -> (output tile, block, chunk range) per mode (see XgSlTask); false
 * for a block with nothing to do (entirely above the diagonal of a diagonal
 * tile, or an empty chunk range).  Jobs are ordered longest first. */
__device__ __forceinline__ bool xg_sl_job(const XgSlTask &S, long long job, int nt, int ts, XgSlJob &J)
{
    const int bpt = ts / XG_SL_BM;
    const int per = bpt * bpt;
    const long long unit = job / per;
    const int blk = (int)(job % per);
    J.bm = blk / bpt;
    J.bn = blk % bpt;
    bool diag = false;
    if (S.mode == XG_SL_FACTOR) { /* targets (i, j), i >= j, of column j */
        J.ta = S.col + (int)unit;
        J.tb = S.col;
        J.k0 = S.k0;
        J.k1 = S.k1;
        J.c_slot = xg_tile_index(J.ta, J.tb, nt);
        diag = J.ta == J.tb;
    } else if (S.mode == XG_SL_INVERSE) { /* X(a, b), a < b = col, from chunks a <= c < b (within [k0, k1)) */
        J.ta = (int)unit;
        J.tb = S.col;
        J.k0 = J.ta > S.k0 ? J.ta : S.k0;
        J.k1 = S.col < S.k1 ? S.col : S.k1;
        J.c_slot = xg_tile_index(J.tb, J.ta, nt);
    } else { /* SYRK: S(a, b), a >= b, from chunks a <= c < nt */
        int ii, jj;
        xg_pair_decode(unit, &ii, &jj);
        J.ta = ii;
        J.tb = jj;
        J.k0 = ii;
        J.k1 = nt;
        J.c_slot = xg_tile_index(ii, jj, nt);
        diag = ii == jj;
    }
    if (diag && J.bm * XG_SL_BM + XG_SL_BM - 1 < J.bn * XG_SL_BN) return false;
    return J.k1 > J.k0;
}

/* packed slot of the A / B operand tile of chunk k */
__device__ __forceinline__ long long xg_sl_slot_a(const XgSlTask &S, const XgSlJob &J, int k, int nt)
{
    return S.mode == XG_SL_FACTOR ? xg_tile_index(J.ta, k, nt) : xg_tile_index(k, J.ta, nt); /* L(i,k) | X(a,k) */
}
__device__ __forceinline__ long long xg_sl_slot_b(const XgSlTask &S, const XgSlJob &J, int k, int nt)
{
    return S.mode == XG_SL_SYRK ? xg_tile_index(k, J.tb, nt) : xg_tile_index(J.tb, k, nt); /* X(b,k) | L(j,k) */
}

__global__ void __launch_bounds__(XG_SL_THREADS, 1)
    xg_sliced_left_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                          const double *__restrict__ scale_a, const double *__restrict__ scale_b, XgTileArgs T,
                          XgSlTask S, long long njobs, int plane_rows, int *status)
{
    extern __shared__ __align__(1024) unsigned char xg_smem_raw[];
    unsigned char *smem = (unsigned char *)(((uintptr_t)xg_smem_raw + 1023) & ~(uintptr_t)1023);
    double *sscale = (double *)(smem + XG_SL_STAGES * XG_SL_STAGE_BYTES); /* [2][A 128 | B 128] */
    uint64_t *full = (uint64_t *)(smem + XG_SL_STAGES * XG_SL_STAGE_BYTES + XG_SL_SCALE_BYTES);
    uint64_t *empty = full + XG_SL_STAGES;
    uint64_t *acc_full = empty + XG_SL_STAGES;
    uint64_t *acc_empty = acc_full + 1;
    uint64_t *drain = acc_empty + 1;
    uint64_t *sfull = drain + 1;  /* [2] the chunk's row scales have landed */
    uint64_t *sempty = sfull + 2; /* [2] the epilogue is done with them */
    uint32_t *tmem_slot = (uint32_t *)(sempty + 2);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ts = T.ts, nt = T.nt;
    if (xg_cta_should_skip(status)) return;
    if (tid == 0) {
        for (int s = 0; s < XG_SL_STAGES; ++s) {
            xg_mbar_init(&full[s], 1);
            xg_mbar_init(&empty[s], 1);
        }
        xg_mbar_init(acc_full, 1);
        xg_mbar_init(acc_empty, XG_SL_EPI_WARPS);
        xg_mbar_init(drain, 1);
        for (int b = 0; b < 2; ++b) {
            xg_mbar_init(&sfull[b], 1);
            xg_mbar_init(&sempty[b], XG_SL_EPI_WARPS);
        }
        xg_fence_barrier_init();
    }
    if (warp == 1) xg_tmem_alloc(tmem_slot, 512); /* four 128-lane x 128-column S32 levels */
    xg_tc_fence_before();
    __syncthreads();
    xg_tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int KT = ts / XG_SL_BK;
    bool ok = true;

    if (warp < 4) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(XG_SL_REG_LOW));
    if (warp == 0) {
        /* ---- TMA producer: per panel chunk the 128 + 128 row scales of the
         * job's A and B blocks (one bulk copy each, into a double buffer the
         * epilogue reads), then per stage the four A and four B digit boxes ---- */
        if (lane == 0) {
            xg_prefetch_tensormap(&map_a);
            xg_prefetch_tensormap(&map_b);
            long long it = 0, cs = 0;
            for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x) {
                XgSlJob J;
                if (!xg_sl_job(S, job, nt, ts, J)) continue;
                for (int k = J.k0; k < J.k1 && ok; ++k, ++cs) {
                    const long long slot_a = xg_sl_slot_a(S, J, k, nt), slot_b = xg_sl_slot_b(S, J, k, nt);
                    const int rowA = (int)(slot_a * ts) + J.bm * XG_SL_BM;
                    const int rowB = (int)(slot_b * ts) + J.bn * XG_SL_BN;
                    {
                        const int sb = (int)(cs & 1);
                        if (cs >= 2 && !xg_mbar_wait(&sempty[sb], (uint32_t)((cs >> 1) - 1) & 1)) {
                            ok = false;
                            break;
                        }
                        xg_mbar_arrive_expect_tx(&sfull[sb], 2 * XG_SL_BM * 8);
                        xg_bulk_load(sscale + sb * 256, scale_a + slot_a * ts + J.bm * XG_SL_BM, XG_SL_BM * 8,
                                     &sfull[sb]);
                        xg_bulk_load(sscale + sb * 256 + 128, scale_b + slot_b * ts + J.bn * XG_SL_BN, XG_SL_BN * 8,
                                     &sfull[sb]);
                    }
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
                            xg_tma_load_2d(st + t * XG_SL_ABOX_BYTES, &map_a, kb * XG_SL_BK, t * plane_rows + rowA,
                                           &full[s]);
                            xg_tma_load_2d(st + XG_SL_SLICES * XG_SL_ABOX_BYTES + t * XG_SL_BBOX_BYTES, &map_b,
                                           kb * XG_SL_BK, t * plane_rows + rowB, &full[s]);
                        }
                    }
                }
            }
            if (!ok) atomicOr(status, XG_ST_TIMEOUT);
            /* copies still in flight land before the CTA may exit */
            const long long first = it > XG_SL_STAGES ? it - XG_SL_STAGES : 0;
            for (long long q = first; q < it; ++q)
                xg_mbar_wait(&full[q % XG_SL_STAGES], (uint32_t)(q / XG_SL_STAGES) & 1);
            for (long long q = cs > 2 ? cs - 2 : 0; q < cs; ++q) xg_mbar_wait(&sfull[q & 1], (uint32_t)(q >> 1) & 1);
        }
    } else if (warp == 1) {
        /* ---- MMA issuer: one accumulation (4 levels) per (job, panel chunk) ---- */
        if (lane == 0) {
            constexpr uint32_t idesc = xg_idesc_i8(XG_SL_BN, XG_SL_BM); /* M = 128 (C columns), N = 128 (C rows) */
            const uint32_t sbase = xg_smem_u32(smem);
            long long it = 0, cc = 0;
            for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x) {
                XgSlJob J;
                if (!xg_sl_job(S, job, nt, ts, J)) continue;
                for (int k = J.k0; k < J.k1 && ok; ++k, ++cc) {
                    if (cc >= 1 && !xg_mbar_wait(acc_empty, (uint32_t)(cc - 1) & 1)) {
                        ok = false;
                        break;
                    }
                    xg_tc_fence_after();
                    const uint32_t dt = tmem;
                    for (int kb = 0; kb < KT; ++kb, ++it) {
                        const int s = (int)(it % XG_SL_STAGES);
                        if (!xg_mbar_wait(&full[s], (uint32_t)(it / XG_SL_STAGES) & 1)) {
                            ok = false;
                            break;
                        }
                        xg_tc_fence_after();
                        const uint32_t sa = sbase + s * XG_SL_STAGE_BYTES;
                        const uint32_t sb = sa + XG_SL_SLICES * XG_SL_ABOX_BYTES;
#pragma unroll
                        for (int kk = 0; kk < XG_SL_BK / 32; ++kk) {
                            /* K = 32 int8 = 32 bytes per MMA inside the 64-byte swizzled row */
#pragma unroll
                            for (int p = 0; p < 10; ++p) {
                                int a, b;
                                xg_sl_pair(p, a, b);
                                const uint64_t ad = xg_umma_desc_sw64(sa + a * XG_SL_ABOX_BYTES + kk * 32);
                                const uint64_t bd = xg_umma_desc_sw64(sb + b * XG_SL_BBOX_BYTES + kk * 32);
                                const bool starts = (p == 0 || p == 1 || p == 3 || p == 6);
                                /* the transposed block E_b D_a^T: TMEM lane = column of
                                 * C, TMEM column = row of C */
                                xg_umma_i8(dt + (uint32_t)((a + b) * XG_SL_BM), bd, ad, idesc,
                                           (kb | kk) != 0 || !starts);
                            }
                        }
                        xg_umma_commit(&empty[s]);
                    }
                    if (!ok) break;
                    xg_umma_commit(acc_full);
                }
            }
            if (!ok) atomicOr(status, XG_ST_TIMEOUT);
            xg_umma_commit(drain);
            xg_mbar_wait(drain, 0);
        }
    }
    } else {
        asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(XG_SL_REG_HIGH));
        /* ---- epilogue: warps 4-11.  Thread (quarter q = warp % 4, lane l) owns
         * C column 32 q + l of the job's block (TMEM lane 32 q + l) and the 64
         * rows h * 64 .. + 63, h = (warp - 4) / 4 (TMEM columns of each level).
         * Per chunk k it adds s_A(row) s_B(col) sum_t 254^-t level_t to 64 FP64
         * sums; after the last chunk C -= sums. ---- */
        const int q = warp & 3, h = (warp - 4) >> 2;
        long long cc = 0;
        for (long long job = blockIdx.x; job < njobs && ok; job += gridDim.x) {
            XgSlJob J;
            if (!xg_sl_job(S, job, nt, ts, J)) continue;
            const int col = J.bn * XG_SL_BN + q * 32 + lane; /* C column (row of the B operand) */
            const int row0 = J.bm * XG_SL_BM + h * 64;       /* first C row (row of the A operand) */
            double *Cc = T.data + J.c_slot * (long long)ts * ts + (long long)row0 * ts + col;
            {
                /* the C block is read once, after all chunks: lane l brings rows
                 * row0 + 2 l, + 1, this quarter's 32 columns (two 128-byte lines
                 * each), into L2 */
                const double *pf = Cc + (long long)(2 * lane) * ts - lane;
                asm volatile("prefetch.global.L2 [%0];" ::"l"(pf));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(pf + 16));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(pf + ts));
                asm volatile("prefetch.global.L2 [%0];" ::"l"(pf + ts + 16));
            }
            double res[64];
#pragma unroll
            for (int u = 0; u < 64; ++u) res[u] = 0.0;
            for (int k = J.k0; k < J.k1; ++k, ++cc) {
                const int sb = (int)(cc & 1);
                if (!xg_mbar_wait(&sfull[sb], (uint32_t)(cc >> 1) & 1) || !xg_mbar_wait(acc_full, (uint32_t)cc & 1)) {
                    if (lane == 0) atomicOr(status, XG_ST_TIMEOUT);
                    ok = false;
                    break;
                }
                xg_tc_fence_after();
                /* s_B (this thread's column) with 254^-3 folded in: the levels are
                 * combined as the exact integer v = L0 254^3 + L1 254^2 + L2 254 + L3
                 * (|v| < 2^48) and converted once.  The row scales come from the
                 * shared-memory copy the producer staged for this chunk. */
                const double sc = sscale[sb * 256 + 128 + q * 32 + lane] * (S.sign * XG_SL_INV_RADIX3);
                const double2 *sr2 = reinterpret_cast<const double2 *>(sscale + sb * 256 + h * 64);
                const uint32_t base = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * 64);
                /* 8 batches per chunk: (columns c * 16 .. + 15, levels 0-1 or 2-3),
                 * software-pipelined -- the next batch's TMEM loads are issued
                 * before the current one is processed, so every wait::ld covers
                 * a load issued one batch earlier */
                uint32_t A0[16], A1[16], B0[16], B1[16];
                int hi[16];
                xg_tmem_ld_32x32b_x16(base + 0u, A0);
                xg_tmem_ld_32x32b_x16(base + (uint32_t)XG_SL_BM, A1);
                xg_tmem_ld_wait();
#pragma unroll
                for (int b = 0; b < 8; ++b) {
                    const int c = b >> 1, half = b & 1;
                    uint32_t(&C0)[16] = (b & 1) ? B0 : A0; /* current batch */
                    uint32_t(&C1)[16] = (b & 1) ? B1 : A1;
                    uint32_t(&N0)[16] = (b & 1) ? A0 : B0; /* next batch */
                    uint32_t(&N1)[16] = (b & 1) ? A1 : B1;
                    if (b < 7) {
                        const int nc = (b + 1) >> 1, nl = 2 * ((b + 1) & 1);
                        xg_tmem_ld_32x32b_x16(base + (uint32_t)(nl * XG_SL_BM + nc * 16), N0);
                        xg_tmem_ld_32x32b_x16(base + (uint32_t)((nl + 1) * XG_SL_BM + nc * 16), N1);
                    }
                    if (half == 0) {
                        /* |L0| <= 127^2 ts, |L1| <= 2 127^2 ts: L0 254 + L1 fits int32 for ts <= 512 */
#pragma unroll
                        for (int w = 0; w < 16; ++w) hi[w] = (int)C0[w] * 254 + (int)C1[w];
                    } else {
#pragma unroll
                        for (int u = 0; u < 16; u += 2) {
                            const double2 s2 = sr2[(c * 16 + u) >> 1]; /* same address in every lane: a broadcast */
#pragma unroll
                            for (int e = 0; e < 2; ++e) {
                                const int w = u + e;
                                /* v = (L0 254 + L1) 254^2 + L2 254 + L3, exact in int64 (< 2^48) */
                                const long long v =
                                    (long long)hi[w] * 64516 + ((long long)(int)C0[w] * 254 + (int)C1[w]);
                                const double sr = e ? s2.y : s2.x;
                                res[c * 16 + w] = fma(sr * sc, xg_i64_to_f64(v), res[c * 16 + w]);
                            }
                        }
                    }
                    if (b < 7) xg_tmem_ld_wait();
                    if (b == 6) {
                        /* every TMEM load of this chunk is complete: the
                         * accumulators are free for the next chunk while the
                         * last batch is combined */
                        xg_tc_fence_before();
                        __syncwarp();
                        if (lane == 0) xg_mbar_arrive(acc_empty);
                    }
                }
                /* this chunk's scale buffer may be refilled */
                __syncwarp();
                if (lane == 0) xg_mbar_arrive(&sempty[sb]);
            }
            if (!ok) break;
            /* C += sign U (or C = sign U): each warp instruction touches 32
             * consecutive doubles of a row; 16 rows are loaded before any is stored, so 16 loads per
             * thread are in flight (a load after a store through the same
             * pointer would wait for it); L2-only accesses (.cg): the few KB
             * of L1 left beside the shared-memory stages would only thrash */
#pragma unroll
            for (int u0 = 0; u0 < 64; u0 += 16) {
                double cv[16];
#pragma unroll
                for (int u = 0; u < 16; ++u) cv[u] = S.overwrite ? 0.0 : __ldcg(Cc + (long long)u * ts);
#pragma unroll
                for (int u = 0; u < 16; ++u) __stcg(Cc + (long long)u * ts, cv[u] + res[u0 + u]);
                Cc += 16LL * ts;
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
    return cudaFuncSetAttribute(xg_sliced_left_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, XG_SL_SMEM);
}

void xg_launch_slice_panel(const XgTileArgs &T, int k, int row_mode, int8_t *dig, double *scale, long long plane,
                           const int *status, cudaStream_t st)
{
    const long long rows = (long long)(row_mode ? k + 1 : T.nt - k - 1) * T.ts;
    if (rows <= 0) return;
    xg_slice_panel_kernel<<<(unsigned)((rows + 7) / 8), 256, 0, st>>>(T, k, row_mode, dig, scale, plane, status);
}

void xg_launch_sliced(const CUtensorMap &map_a, const CUtensorMap &map_b, const double *scale_a,
                      const double *scale_b, const XgTileArgs &T, const XgSlTask &S, int plane_rows, int max_ctas,
                      int *status, cudaStream_t st)
{
    if (S.k1 <= S.k0 || S.col >= T.nt) return;
    const long long per = (long long)(T.ts / XG_SL_BM) * (T.ts / XG_SL_BN);
    long long units;
    if (S.mode == XG_SL_FACTOR) units = T.nt - S.col;
    else if (S.mode == XG_SL_INVERSE) units = S.col;
    else units = (long long)T.nt * (T.nt + 1) / 2;
    const long long njobs = units * per;
    if (njobs <= 0) return;
    const unsigned grid = (unsigned)(njobs < max_ctas ? njobs : max_ctas);
    xg_sliced_left_kernel<<<grid, XG_SL_THREADS, XG_SL_SMEM, st>>>(map_a, map_b, scale_a, scale_b, T, S, njobs,
                                                                   plane_rows, status);
}
