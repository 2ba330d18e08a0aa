/*
 * Log-likelihood evaluation that allocates no device memory.
 *
 * Some callers cannot call cudaMalloc: code running inside another
 * framework's memory pool or allocator (which owns every device allocation
 * and may forbid or interpose foreign ones), and code that has to keep
 * working while the device heap is exhausted.  For them
 * exageostat_b200_dmle_device_noalloc() evaluates the exact Matern
 * log-likelihood for up to XG_NOALLOC_MAX_N locations using only caller
 * buffers (device x, y, z and result) plus one file-scope device array,
 * xg_noalloc_scratch, that the library carries for every GPU that loads it
 * (about 18 MB) until the process exits.
 *
 * The call is synchronous: it enqueues its work on the caller's stream, then
 * reads the device status word back and waits for the stream before it
 * returns.  d_out is written only when the evaluation succeeded; on any
 * error its contents are left as they were.
 *
 * The scratch array is shared by all calls on a device and keeps the
 * previous call's contents; every buffer inside it that must start at zero
 * (solve-vector padding, status word) is cleared by each call, and the tile
 * table is rebuilt.  Calls whose work overlaps on the GPU (other streams,
 * other host threads) race on the array: serialise them.  The scratch
 * address is cached per device ordinal, so only the primary context of each
 * device (the runtime API's default) is supported.
 */
#include <stdint.h>
#include <string.h>

#include <mutex>

#include "../../include/exageostat_b200.h"
#include "xg_common.cuh"
#include "xg_engine.h"
#include "xg_kernels.h"

#define XG_NOALLOC_MAX_N 2048
#define XG_NOALLOC_TS 128
#define XG_NOALLOC_MAX_NT (XG_NOALLOC_MAX_N / XG_NOALLOC_TS)
#define XG_NOALLOC_MAX_TILES (XG_NOALLOC_MAX_NT * (XG_NOALLOC_MAX_NT + 1) / 2)
#define XG_NOALLOC_TILE_DOUBLES ((size_t)XG_NOALLOC_MAX_TILES * XG_NOALLOC_TS * XG_NOALLOC_TS)
/* layout in doubles: tiles | v [MAX_N] | part [2 MAX_NT] | out [8] | status (2 ints) | tile table (MAX_TILES int2) */
#define XG_NOALLOC_OFF_V XG_NOALLOC_TILE_DOUBLES
#define XG_NOALLOC_OFF_PART (XG_NOALLOC_OFF_V + XG_NOALLOC_MAX_N)
#define XG_NOALLOC_OFF_OUT (XG_NOALLOC_OFF_PART + 2 * XG_NOALLOC_MAX_NT)
#define XG_NOALLOC_OFF_STATUS (XG_NOALLOC_OFF_OUT + 8)
#define XG_NOALLOC_OFF_TABLE (XG_NOALLOC_OFF_STATUS + 1)
#define XG_NOALLOC_DOUBLES (XG_NOALLOC_OFF_TABLE + XG_NOALLOC_MAX_TILES)

static __device__ __align__(256) double xg_noalloc_scratch[XG_NOALLOC_DOUBLES];

#define XG_NOALLOC_MAX_DEVICES 64
static std::mutex g_noalloc_mu;
static double *g_noalloc_ptr[XG_NOALLOC_MAX_DEVICES];

typedef CUresult (*XgEncodeFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                               const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                               CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static XgEncodeFn g_noalloc_encode = nullptr;

/* (i, j) of every packed lower tile for nt tiles per side */
__global__ void xg_noalloc_table_kernel(int2 *table, int nt)
{
    for (int j = 0; j < nt; ++j)
        for (int i = j + threadIdx.x; i < nt; i += blockDim.x) table[xg_tile_index(i, j, nt)] = make_int2(i, j);
}

/* One-time set-up on the current device: device address of the scratch
 * array (host code cannot use the symbol itself), kernel attributes and the
 * tensor-map encoder.  Returns the scratch address or nullptr. */
static double *xg_noalloc_setup(int *rc)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *rc = xg_fail(XG_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
        return nullptr;
    }
    if (dev < 0 || dev >= XG_NOALLOC_MAX_DEVICES) {
        *rc = xg_fail(XG_ERR_UNSUPPORTED, "device ordinal %d is beyond %d", dev, XG_NOALLOC_MAX_DEVICES);
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_ptr[dev]) return g_noalloc_ptr[dev];
    int major = 0;
    e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e != cudaSuccess) {
        *rc = xg_fail(XG_ERR_CUDA, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e));
        return nullptr;
    }
    if (major != 10) {
        *rc = xg_fail(XG_ERR_UNSUPPORTED, "device %d is sm_%dx; the library is built for sm_100a (B200) only", dev,
                      major);
        return nullptr;
    }
    void *ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, xg_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        *rc = xg_fail(XG_ERR_CUDA, "cudaGetSymbolAddress(xg_noalloc_scratch): %s", cudaGetErrorString(e));
        return nullptr;
    }
    e = xg_kernels_configure();
    if (e != cudaSuccess) {
        *rc = xg_fail(XG_ERR_CUDA, "kernel attribute setup: %s", cudaGetErrorString(e));
        return nullptr;
    }
    if (!g_noalloc_encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || !fn || q != cudaDriverEntryPointSuccess) {
            *rc = xg_fail(XG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
            return nullptr;
        }
        g_noalloc_encode = (XgEncodeFn)fn;
    }
    g_noalloc_ptr[dev] = (double *)ptr;
    return (double *)ptr;
}

extern "C" int exageostat_b200_dmle_device_noalloc(int n, const double *d_x, const double *d_y, const double *d_z,
                                                   const double *theta, int kernel, int metric, double *d_out,
                                                   void *stream)
{
    if (n <= 0 || n > XG_NOALLOC_MAX_N)
        return xg_fail(XG_ERR_BAD_ARGUMENT,
                       "n = %d is outside [1, %d], the size the no-allocation entry point's static scratch holds",
                       n, XG_NOALLOC_MAX_N);
    if (!d_x || !d_y || !d_z || !d_out || !theta)
        return xg_fail(XG_ERR_BAD_ARGUMENT, "a buffer argument is NULL");
    if (kernel != 0 && kernel != 1) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    if (metric != 0 && metric != 1)
        return xg_fail(XG_ERR_BAD_ARGUMENT, "metric %d (0 Euclidean, 1 great circle)", metric);
    int rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    rc = XG_OK;
    double *base = xg_noalloc_setup(&rc);
    if (!base) return rc;

    cudaStream_t st = (cudaStream_t)stream;
    XgTileMatrix M;
    M.N = n;
    M.ts = XG_NOALLOC_TS;
    M.nt = (n + XG_NOALLOC_TS - 1) / XG_NOALLOC_TS;
    M.ntiles = xg_num_lower_tiles(M.nt);
    M.d = base;
    M.ij = (int2 *)(base + XG_NOALLOC_OFF_TABLE);
    double *v = base + XG_NOALLOC_OFF_V;
    double *part = base + XG_NOALLOC_OFF_PART;
    double *out = base + XG_NOALLOC_OFF_OUT;
    int *status = (int *)(base + XG_NOALLOC_OFF_STATUS);
    cuuint64_t dims[2] = {(cuuint64_t)M.ts, (cuuint64_t)M.ntiles * M.ts};
    cuuint64_t strides[1] = {(cuuint64_t)M.ts * sizeof(double)};
    cuuint32_t box[2] = {16, 128};
    cuuint32_t estr[2] = {1, 1};
    CUresult cr = g_noalloc_encode(&M.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, M.d, dims, strides, box, estr,
                                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return xg_fail(XG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)cr);

    const size_t np = (size_t)M.nt * M.ts;
    cudaError_t e = cudaMemsetAsync(status, 0, 2 * sizeof(int), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(v, 0, np * sizeof(double), st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(v, d_z, n * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "scratch initialisation: %s", cudaGetErrorString(e));
    xg_noalloc_table_kernel<<<1, 32, 0, st>>>(M.ij, M.nt);
    const XgMaternParams p = xg_params(theta, kernel);
    XgTileArgs T{M.d, M.ts, M.nt};
    xg_launch_gen(T, M.ij, M.ntiles, d_x, d_y, d_x, d_y, n, n, p, metric, 1, st);
    xg_factor(M, v, part, status, status + 1, st);
    xg_launch_finalize(part, part + M.nt, M.nt, n, out, status, status + 1, st);
    e = cudaGetLastError();
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "launch: %s", cudaGetErrorString(e));
    int sv[2] = {0, 0};
    e = cudaMemcpyAsync(sv, status, sizeof sv, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "no-allocation evaluation: %s", cudaGetErrorString(e));
    if (sv[0] & XG_ST_NOT_SPD) return xg_fail(XG_ERR_NOT_SPD, "the covariance is not positive definite (pivot %d)", sv[1]);
    if (sv[0]) return xg_fail(XG_ERR_TIMEOUT, "device status word 0x%x", sv[0]);
    /* the result reaches the caller's buffer only once the status is clean */
    e = cudaMemcpyAsync(d_out, out, 3 * sizeof(double), cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "no-allocation result copy: %s", cudaGetErrorString(e));
    return XG_OK;
}
