/*
 * Diagnostic of the bounded-wait path (no counterpart in the reference).
 *
 * Every pipeline wait in the library's kernels goes through xg_mbar_wait,
 * which gives up after a wall-time limit and lets the kernel record
 * XG_ST_TIMEOUT in its status word instead of spinning forever.  This entry
 * point runs that path on purpose: one thread waits on a shared-memory
 * mbarrier that nothing ever arrives on, with a short limit, records the
 * timeout bit and returns normally, so the host sees XG_ERR_TIMEOUT and the
 * CUDA context stays usable for the next call.
 */
#include <stdint.h>

#include "../../include/exageostat_b200.h"
#include "xg_common.cuh"
#include "xg_engine.h"

__global__ void xg_diag_wait_kernel(uint64_t limit_ns, int *status, unsigned long long *waited_ns)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        xg_mbar_init(&bar, 1);
        xg_fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint64_t t0 = xg_globaltimer_ns();
        /* phase 0 of a fresh barrier never completes: no thread arrives */
        const bool ok = xg_mbar_wait(&bar, 0, limit_ns);
        *waited_ns = (unsigned long long)(xg_globaltimer_ns() - t0);
        if (!ok) atomicOr(status, XG_ST_TIMEOUT);
    }
}

extern "C" int exageostat_b200_diag_wait_timeout(double limit_us, double *waited_us)
{
    if (!(limit_us >= 1.0 && limit_us <= 1.0e6))
        return xg_fail(XG_ERR_BAD_ARGUMENT, "limit %g us is outside [1, 1e6]", limit_us);
    int rc = xg_context_require();
    if (rc) return rc;
    cudaStream_t st = g_xg.stream;
    void *buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, 16);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "bounded-wait diagnostic: %s", cudaGetErrorString(e));
    int *status = (int *)buf;
    unsigned long long *waited = (unsigned long long *)((char *)buf + 8);
    e = cudaMemsetAsync(buf, 0, 16, st);
    if (e == cudaSuccess) {
        xg_diag_wait_kernel<<<1, 32, 0, st>>>((uint64_t)(limit_us * 1e3), status, waited);
        e = cudaGetLastError();
    }
    unsigned long long h[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, buf, 16, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "bounded-wait diagnostic: %s", cudaGetErrorString(e));
    if (waited_us) *waited_us = (double)h[1] * 1e-3;
    const int sv = (int)(h[0] & 0xffffffffu);
    if (sv & XG_ST_TIMEOUT) return xg_fail(XG_ERR_TIMEOUT, "a device pipeline wait timed out (diagnostic)");
    if (sv) return xg_fail(XG_ERR_CUDA, "device status word 0x%x", sv);
    return XG_OK;
}
