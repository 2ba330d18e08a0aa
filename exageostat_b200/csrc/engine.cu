/*
 * Host engine behind the reference C API (capi.cpp).
 *
 * One process-wide context (exageostat_init) owns the CUDA stream.  Each
 * MLE_data owns one XgField (stored in data->descC): the device locations,
 * z, the lower-tile covariance / factor and the solve buffers.  An
 * evaluation is a fixed launch sequence on the context stream:
 *
 *   generate Sigma(theta) tiles -> for k: POTRF(k,k) [+ log-det, + z block
 *   solve] -> TRSM panel k [+ z update] -> trailing update k -> finalize
 *
 * and one device-to-host copy of the result.  Nothing here calls exit().
 */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/exageostat_b200.h"
#include "kbessel.cuh"
#include "xg_common.cuh"
#include "xg_engine.h"
#include "xg_kernels.h"

/* ------------------------------------------------------------------------- */
/* errors                                                                    */
/* ------------------------------------------------------------------------- */

static thread_local std::string g_last_error;

int xg_fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

static int xg_cuda_fail(cudaError_t e, const char *what)
{
    return xg_fail(XG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define XG_CU(call)                                                                                                    \
    do {                                                                                                               \
        cudaError_t _e = (call);                                                                                       \
        if (_e != cudaSuccess) return xg_cuda_fail(_e, #call);                                                         \
    } while (0)

extern "C" const char *exageostat_last_error(void) { return g_last_error.c_str(); }

/* ------------------------------------------------------------------------- */
/* context                                                                   */
/* ------------------------------------------------------------------------- */

XgContext g_xg;

typedef CUresult (*XgEncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                     const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                     CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static XgEncodeTiledFn g_encode = nullptr;

int xg_context_start(int dts)
{
    std::lock_guard<std::mutex> lk(g_xg.mu);
    if (g_xg.initialized) return XG_OK;
    int dev = 0;
    XG_CU(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    XG_CU(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10)
        return xg_fail(XG_ERR_UNSUPPORTED, "device %d (%s, sm_%d%d) is not a B200-class sm_100 GPU", dev, prop.name,
                       prop.major, prop.minor);
    XG_CU(cudaStreamCreateWithFlags(&g_xg.stream, cudaStreamNonBlocking));
    int prio_least = 0, prio_greatest = 0;
    XG_CU(cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest));
    XG_CU(cudaStreamCreateWithPriority(&g_xg.stream_hi, cudaStreamNonBlocking, prio_greatest));
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    XG_CU(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (!fn || q != cudaDriverEntryPointSuccess)
        return xg_fail(XG_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    g_encode = (XgEncodeTiledFn)fn;
    cudaError_t e = xg_kernels_configure();
    if (e == cudaSuccess) e = xg_gradient_kernels_configure();
    if (e == cudaSuccess) e = xg_mixed_kernels_configure();
    if (e == cudaSuccess) e = xg_sliced_kernels_configure();
    if (e != cudaSuccess) return xg_cuda_fail(e, "kernel attribute setup");
    g_xg.device = dev;
    g_xg.sm_count = prop.multiProcessorCount;
    g_xg.dts = dts;
    g_xg.initialized = true;
    return XG_OK;
}

int xg_context_require()
{
    if (g_xg.initialized) return XG_OK;
    /* The reference requires exageostat_init first; starting lazily keeps
     * the one-shot entry points usable on their own. */
    return xg_context_start(0);
}

/* tile size: a multiple of 128 in [128, XG_MAX_TS]; 0 picks by problem size */
int xg_choose_ts(int N, int dts)
{
    if (dts <= 0) {
        if (N <= 1024) return 128;
        if (N <= 8192) return 256;
        return 512;
    }
    int ts = ((dts + 127) / 128) * 128;
    if (ts < 128) ts = 128;
    if (ts > XG_MAX_TS) ts = XG_MAX_TS;
    return ts;
}

/* ------------------------------------------------------------------------- */
/* lower-tile matrices                                                       */
/* ------------------------------------------------------------------------- */

int xg_tm_alloc(XgTileMatrix &M, int N, int ts)
{
    M.N = N;
    M.ts = ts;
    M.nt = (N + ts - 1) / ts;
    M.ntiles = xg_num_lower_tiles(M.nt);
    const size_t bytes = (size_t)M.ntiles * ts * ts * sizeof(double);
    cudaError_t e = cudaMalloc(&M.d, bytes);
    if (e != cudaSuccess) {
        M.d = nullptr;
        return xg_fail(XG_ERR_NO_MEMORY, "cannot allocate %.2f GB for %lld covariance tiles: %s", bytes / 1e9,
                       M.ntiles, cudaGetErrorString(e));
    }
    int2 *hij = (int2 *)malloc(sizeof(int2) * M.ntiles);
    for (int j = 0; j < M.nt; ++j)
        for (int i = j; i < M.nt; ++i) hij[xg_tile_index(i, j, M.nt)] = make_int2(i, j);
    e = cudaMalloc(&M.ij, sizeof(int2) * M.ntiles);
    if (e == cudaSuccess) e = cudaMemcpy(M.ij, hij, sizeof(int2) * M.ntiles, cudaMemcpyHostToDevice);
    free(hij);
    if (e != cudaSuccess) return xg_cuda_fail(e, "tile index table");
    e = cudaMalloc(&M.dinv, sizeof(double) * (size_t)ts * 32);
    if (e != cudaSuccess) {
        M.dinv = nullptr;
        return xg_cuda_fail(e, "diagonal-block inverses");
    }
    return xg_encode_tiles(&M.map, M.d, M.ntiles, ts);
}

/* TMA view of a lower-tile store: a 2-D FP64 tensor [ntiles * ts rows][ts
 * columns], boxes of 128 rows x 16 columns (128 bytes, swizzled) */
int xg_encode_tiles(CUtensorMap *map, double *base, long long ntiles, int ts)
{
    cuuint64_t dims[2] = {(cuuint64_t)ts, (cuuint64_t)ntiles * ts};
    cuuint64_t strides[1] = {(cuuint64_t)ts * sizeof(double)};
    cuuint32_t box[2] = {16, 128};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, base, dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return xg_fail(XG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return XG_OK;
}

void xg_tm_free(XgTileMatrix &M)
{
    if (M.d) cudaFree(M.d);
    if (M.ij) cudaFree(M.ij);
    if (M.dinv) cudaFree(M.dinv);
    M.d = nullptr;
    M.ij = nullptr;
    M.dinv = nullptr;
}

XgMaternParams xg_params(const double *theta, int kernel)
{
    XgMaternParams p;
    p.bivariate = 0;
    p.sigma2b = p.nu2 = p.con2 = p.nu12 = p.con12 = p.cross0 = 0.0;
    p.beta2 = p.beta12 = 0.0;
    if (kernel == 3) {
        /* theta = (a_1, a_2, ., ., nu_1, nu_2, ., ., ., ., .): the constants of
         * core_dcmg_bivariate_flexible (core_zcmg.c:1524-1556), in its order;
         * at zero distance the reference stores theta[0], theta[1] and rho
         * (:1565-1568) */
        const double scale1 = theta[0], scale2 = theta[1], nu1 = theta[4], nu2 = theta[5];
        const double scale12 = pow(0.5 * (pow(scale1, -2) + pow(scale2, -2)) + theta[2] * (1 - theta[3]), -0.5);
        const double nu12 = 0.5 * (nu1 + nu2) + theta[6] * (1 - theta[7]);
        const double rho = theta[8] * theta[9] * theta[10] * pow(scale12, 2 * theta[6] + (nu1 + nu2)) *
                           tgamma(0.5 * (nu1 + nu2) + 1) * tgamma(nu12) / tgamma(nu12 + 1);
        const double s11 = theta[8] * theta[8] * pow(scale1, 2 * theta[6] + nu1 + nu1) * tgamma(nu1);
        const double s22 = theta[9] * theta[9] * pow(scale2, 2 * theta[6] + nu2 + nu2) * tgamma(nu2);
        p.bivariate = 1;
        p.sigma2 = theta[0];
        p.sigma2b = theta[1];
        p.cross0 = rho;
        p.beta = scale1;
        p.beta2 = scale2;
        p.beta12 = scale12;
        p.nu = nu1;
        p.nu2 = nu2;
        p.nu12 = nu12;
        p.nugget = 0.0;
        p.half_integer = -1;
        double con1 = pow(2, (nu1 - 1)) * tgamma(nu1);
        con1 = 1.0 / con1;
        p.con = s11 * con1;
        double con2 = pow(2, (nu2 - 1)) * tgamma(nu2);
        con2 = 1.0 / con2;
        p.con2 = s22 * con2;
        double con12 = pow(2, (nu12 - 1)) * tgamma(nu12);
        con12 = 1.0 / con12;
        p.con12 = rho * con12;
        p.tm = xg_temme_consts(nu1);
        return p;
    }
    if (kernel == 2) {
        /* theta = (sigma_1^2, sigma_2^2, beta, nu_1, nu_2, rho): the constants of
         * core_dcmg_bivariate_parsimonious (core_zcmg.c:1637-1651), in its order */
        p.bivariate = 1;
        p.sigma2 = theta[0];
        p.sigma2b = theta[1];
        p.beta = theta[2];
        p.nu = theta[3];
        p.nu2 = theta[4];
        p.nugget = 0.0;
        p.half_integer = -1;
        double con1 = pow(2, (theta[3] - 1)) * tgamma(theta[3]);
        con1 = 1.0 / con1;
        p.con = theta[0] * con1;
        double con2 = pow(2, (theta[4] - 1)) * tgamma(theta[4]);
        con2 = 1.0 / con2;
        p.con2 = theta[1] * con2;
        p.nu12 = 0.5 * (theta[3] + theta[4]);
        const double rho = theta[5] * sqrt((tgamma(theta[3] + 1) * tgamma(theta[4] + 1)) /
                                           (tgamma(theta[3]) * tgamma(theta[4]))) *
                           tgamma(p.nu12) / tgamma(p.nu12 + 1);
        double con12 = pow(2, (p.nu12 - 1)) * tgamma(p.nu12);
        con12 = 1.0 / con12;
        p.con12 = rho * sqrt(theta[0] * theta[1]) * con12;
        p.cross0 = rho * sqrt(theta[0] * theta[1]);
        p.beta2 = p.beta12 = p.beta;
        p.tm = xg_temme_consts(p.nu);
        return p;
    }
    p.sigma2 = theta[0];
    p.beta = theta[1];
    p.nu = theta[2];
    p.nugget = (kernel == 1) ? theta[3] : 0.0;
    /* core_zcmg.c:976-978 */
    double con = pow(2, (theta[2] - 1)) * tgamma(theta[2]);
    con = 1.0 / con;
    p.con = theta[0] * con;
    p.half_integer = (theta[2] == 0.5) ? 0 : (theta[2] == 1.5) ? 1 : (theta[2] == 2.5) ? 2 : -1;
    p.tm = xg_temme_consts(theta[2]);
    return p;
}

int xg_check_theta(const double *theta, int kernel)
{
    if (kernel == 3) {
        for (int i = 0; i < 11; ++i)
            if (!isfinite(theta[i])) return xg_fail(XG_ERR_BAD_ARGUMENT, "theta[%d] is not finite", i);
        const int pos[4] = {0, 1, 4, 5}; /* the two scales and smoothnesses */
        for (int i : pos)
            if (!(theta[i] > 0)) return xg_fail(XG_ERR_BAD_ARGUMENT, "theta[%d] = %g must be positive", i, theta[i]);
        if (theta[4] > 25.0 || theta[5] > 25.0)
            return xg_fail(XG_ERR_BAD_ARGUMENT, "smoothness above the supported maximum 25");
        return XG_OK;
    }
    if (kernel == 2) {
        for (int i = 0; i < 6; ++i)
            if (!isfinite(theta[i])) return xg_fail(XG_ERR_BAD_ARGUMENT, "theta[%d] is not finite", i);
        for (int i = 0; i < 5; ++i)
            if (!(theta[i] > 0)) return xg_fail(XG_ERR_BAD_ARGUMENT, "theta[%d] = %g must be positive", i, theta[i]);
        if (theta[3] > 25.0 || theta[4] > 25.0)
            return xg_fail(XG_ERR_BAD_ARGUMENT, "smoothness above the supported maximum 25");
        return XG_OK;
    }
    const int np = kernel == 1 ? 4 : 3;
    for (int i = 0; i < np; ++i)
        if (!isfinite(theta[i])) return xg_fail(XG_ERR_BAD_ARGUMENT, "theta[%d] is not finite", i);
    if (!(theta[0] > 0) || !(theta[1] > 0) || !(theta[2] > 0))
        return xg_fail(XG_ERR_BAD_ARGUMENT, "theta = (%g, %g, %g) must be positive", theta[0], theta[1], theta[2]);
    if (theta[2] > 25.0)
        return xg_fail(XG_ERR_BAD_ARGUMENT, "smoothness nu = %g is above the supported maximum 25", theta[2]);
    if (kernel == 1 && theta[3] < 0) return xg_fail(XG_ERR_BAD_ARGUMENT, "nugget %g must be >= 0", theta[3]);
    return XG_OK;
}

/* Cholesky of M in place; with v != nullptr also v <- L^-1 v and the per-tile
 * partial sums (log-det in part[0:nt], |v_k|^2 in part[nt:2nt]). */
/* Right-looking tile Cholesky with the fused z solve.  Per step k:
 *   panel   : POTRF(k,k) [+ log-det, + L_kk v_k = v_k]  ->  TRSM(i,k) [+ v_i -= L_ik v_k]
 *   trailing: A_ij -= L_ik L_jk^T, j >= k+1
 * With fs.st_hi the panel of step k+1 runs on the high-priority stream as soon
 * as column k+1 has received the step-k update (the trailing update is split
 * into "column k+1" and "the rest"), so it overlaps the rest of step k.
 * Profiling events (5 per step): panel start, after POTRF, after TRSM,
 * trailing start, trailing end. */
void xg_factor_lookahead(XgTileMatrix &M, double *v, double *part, int *status, int *info, const XgFactorStreams &fs)
{
    XgTileArgs T{M.d, M.ts, M.nt};
    T.dinv = M.dinv;
    const bool la = fs.st_hi != nullptr;
    cudaStream_t sp = la ? fs.st_hi : fs.st; /* panel stream */
    cudaEvent_t *pev = fs.pev;
    const int rhs = v != nullptr;
    if (la) {
        cudaEventRecord(fs.ev_upd, fs.st); /* the generated matrix */
    }
    for (int k = 0; k < M.nt; ++k) {
        if (la) cudaStreamWaitEvent(sp, fs.ev_upd, 0);
        if (pev) cudaEventRecord(pev[5 * k], sp);
        xg_launch_potrf_tiled(M.map, T, k, v, part, part + M.nt, rhs, status, info, sp);
        if (pev) cudaEventRecord(pev[5 * k + 1], sp);
        if (T.dinv)
            xg_launch_trsm_gemm(M.map, T, k, v, rhs, status, sp);
        else
            xg_launch_trsm_panel(T, k, v, rhs, status, sp);
        if (pev) cudaEventRecord(pev[5 * k + 2], sp);
        if (la) {
            cudaEventRecord(fs.ev_panel, sp);
            cudaStreamWaitEvent(fs.st, fs.ev_panel, 0);
        }
        if (pev) cudaEventRecord(pev[5 * k + 3], fs.st);
        if (k + 1 < M.nt) {
            if (la) {
                xg_launch_syrk_gemm(M.map, T, k, status, fs.st, 1);
                cudaEventRecord(fs.ev_upd, fs.st);
                xg_launch_syrk_gemm(M.map, T, k, status, fs.st, 2);
            } else {
                xg_launch_syrk_gemm(M.map, T, k, status, fs.st, 0);
            }
        }
        if (pev) cudaEventRecord(pev[5 * k + 4], fs.st);
    }
}

void xg_factor(XgTileMatrix &M, double *v, double *part, int *status, int *info, cudaStream_t st, cudaEvent_t *pev)
{
    XgFactorStreams fs;
    fs.st = st;
    fs.pev = pev;
    xg_factor_lookahead(M, v, part, status, info, fs);
}

/* Algorithmic flops of the trailing update after step k: a GEMM (2 ts^3) per
 * off-diagonal tile pair and a SYRK (ts^2 (ts + 1)) per diagonal tile. */
double xg_trailing_flops(int nt, int ts, int k)
{
    const double n = nt - k - 1;
    const double t = ts;
    return n * (n - 1) / 2 * 2 * t * t * t + n * t * t * (t + 1);
}

int xg_field_set_profiling(XgField *f, int on)
{
    if (on && !f->pev) {
        const int n = 8 * f->C.nt;
        f->pev = (cudaEvent_t *)calloc(n, sizeof(cudaEvent_t));
        for (int i = 0; i < n; ++i)
            if (cudaEventCreate(&f->pev[i]) != cudaSuccess) return xg_fail(XG_ERR_CUDA, "profiling events");
    }
    f->profiling = on != 0;
    for (int i = 0; i < 12; ++i) f->prof[i] = 0;
    return XG_OK;
}

static void xg_field_collect_profile(XgField *f)
{
    float ms = 0;
    const int nt = f->C.nt;
    cudaEventElapsedTime(&ms, f->ev[0], f->ev[1]);
    f->prof[0] += ms * 1e-3;
    for (int k = 0; k < nt; ++k) {
        cudaEventElapsedTime(&ms, f->pev[5 * k], f->pev[5 * k + 1]);
        f->prof[1] += ms * 1e-3;
        cudaEventElapsedTime(&ms, f->pev[5 * k + 1], f->pev[5 * k + 2]);
        f->prof[2] += ms * 1e-3;
        if (k + 1 < nt) {
            cudaEventElapsedTime(&ms, f->pev[5 * k + 3], f->pev[5 * k + 4]);
            f->prof[3] += ms * 1e-3;
            f->prof[4] += xg_trailing_flops(nt, f->C.ts, k);
        }
    }
    cudaEventElapsedTime(&ms, f->ev[0], f->ev[2]);
    f->prof[7] += ms * 1e-3;
    /* launches: generation, the sub-block POTRF sequence per step, TRSM and two
     * trailing launches per step but the last (the first trailing launch of
     * the last step but one covers one column and the second is empty),
     * finalize */
    double launches = 1 + (double)nt * xg_potrf_tiled_launches(f->C.ts) + 1;
    for (int k = 0; k + 1 < nt; ++k) launches += 1 + 1 + (k + 2 < nt ? 1 : 0);
    f->prof[5] += launches;
    f->prof[6] += 1;
}

int xg_field_set_data(XgField *f, const double *x, const double *y, const double *z)
{
    cudaStream_t st = g_xg.stream;
    const int nloc = xg_bivariate(f->kernel) ? f->N / 2 : f->N; /* bivariate: two variables per location */
    if (x) XG_CU(cudaMemcpyAsync(f->x, x, nloc * sizeof(double), cudaMemcpyHostToDevice, st));
    if (y) XG_CU(cudaMemcpyAsync(f->y, y, nloc * sizeof(double), cudaMemcpyHostToDevice, st));
    if (z) XG_CU(cudaMemcpyAsync(f->z, z, f->N * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaStreamSynchronize(st));
    if (z) f->have_z = true;
    return XG_OK;
}

/* ------------------------------------------------------------------------- */
/* fields                                                                    */
/* ------------------------------------------------------------------------- */

static int xg_dev_alloc(double **p, size_t n)
{
    cudaError_t e = cudaMalloc(p, n * sizeof(double));
    if (e != cudaSuccess) return xg_fail(XG_ERR_NO_MEMORY, "cudaMalloc(%zu doubles): %s", n, cudaGetErrorString(e));
    return cudaMemset(*p, 0, n * sizeof(double)) == cudaSuccess ? XG_OK : XG_ERR_CUDA;
}

void xg_field_destroy(XgField *f)
{
    if (!f) return;
    xg_tm_free(f->C);
    double *bufs[] = {f->x, f->y, f->z, f->v, f->e, f->part, f->out};
    for (double *b : bufs)
        if (b) cudaFree(b);
    if (f->status) cudaFree(f->status);
    if (f->h_out) cudaFreeHost(f->h_out);
    if (f->pev) {
        for (int i = 0; i < 8 * f->C.nt; ++i)
            if (f->pev[i]) cudaEventDestroy(f->pev[i]);
        free(f->pev);
    }
    if (f->ev_panel) cudaEventDestroy(f->ev_panel);
    if (f->ev_upd) cudaEventDestroy(f->ev_upd);
    xg_tm_free(f->X);
    if (f->mx) xg_mixed_destroy(f->mx);
    if (f->sl) xg_sliced_destroy(f->sl);
    if (f->gpart) cudaFree(f->gpart);
    if (f->gout) cudaFree(f->gout);
    for (int i = 0; i < 4; ++i)
        if (f->ev[i]) cudaEventDestroy(f->ev[i]);
    delete f;
}

int xg_field_create(XgField **out, int N, int ts, const double *x, const double *y, int kernel, int metric)
{
    *out = nullptr;
    int rc = xg_context_require();
    if (rc) return rc;
    if (N <= 0) return xg_fail(XG_ERR_BAD_ARGUMENT, "N = %d must be positive", N);
    if (!x || !y) return xg_fail(XG_ERR_BAD_ARGUMENT, "locations are NULL");
    if (xg_bivariate(kernel) && (N & 1))
        return xg_fail(XG_ERR_BAD_ARGUMENT, "bivariate kernel: N = %d must be 2 x the number of locations", N);
    /* bivariate: N / 2 locations, two variables each */
    const int nloc = xg_bivariate(kernel) ? N / 2 : N;
    XgField *f = new XgField();
    f->N = N;
    f->kernel = kernel;
    f->metric = metric;
    rc = xg_tm_alloc(f->C, N, xg_choose_ts(N, ts));
    const size_t Np = (size_t)f->C.nt * f->C.ts;
    if (!rc) rc = xg_dev_alloc(&f->x, Np);
    if (!rc) rc = xg_dev_alloc(&f->y, Np);
    if (!rc) rc = xg_dev_alloc(&f->z, Np);
    if (!rc) rc = xg_dev_alloc(&f->v, Np);
    if (!rc) rc = xg_dev_alloc(&f->e, Np);
    if (!rc) rc = xg_dev_alloc(&f->part, 2 * (size_t)f->C.nt);
    if (!rc) rc = xg_dev_alloc(&f->out, 8);
    if (!rc && cudaMalloc(&f->status, 2 * sizeof(int)) != cudaSuccess) rc = xg_fail(XG_ERR_NO_MEMORY, "status word");
    if (!rc && cudaMallocHost(&f->h_out, 8 * sizeof(double)) != cudaSuccess)
        rc = xg_fail(XG_ERR_NO_MEMORY, "pinned result buffer");
    for (int i = 0; i < 4 && !rc; ++i)
        if (cudaEventCreate(&f->ev[i]) != cudaSuccess) rc = xg_fail(XG_ERR_CUDA, "event");
    if (!rc && (cudaEventCreateWithFlags(&f->ev_panel, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&f->ev_upd, cudaEventDisableTiming) != cudaSuccess))
        rc = xg_fail(XG_ERR_CUDA, "lookahead events");
    if (!rc && cudaMemcpy(f->x, x, nloc * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = xg_fail(XG_ERR_CUDA, "upload x");
    if (!rc && cudaMemcpy(f->y, y, nloc * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        rc = xg_fail(XG_ERR_CUDA, "upload y");
    if (rc) {
        xg_field_destroy(f);
        return rc;
    }
    f->info = f->status + 1;
    *out = f;
    return XG_OK;
}

int xg_field_set_z(XgField *f, const double *z)
{
    cudaStream_t st = g_xg.stream;
    XG_CU(cudaMemcpyAsync(f->z, z, f->N * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaStreamSynchronize(st));
    f->have_z = true;
    return XG_OK;
}

static int xg_read_status(XgField *f)
{
    const int st = (int)f->h_out[3];
    if (st & XG_ST_NOT_SPD)
        return xg_fail(XG_ERR_NOT_SPD, "the covariance is not positive definite (pivot %d)", (int)f->h_out[4]);
    if (st & XG_ST_TIMEOUT) return xg_fail(XG_ERR_TIMEOUT, "a device pipeline wait timed out");
    if (st) return xg_fail(XG_ERR_CUDA, "device status word 0x%x", st);
    return XG_OK;
}

/* log-likelihood at theta; res[0..2] = loglik, logdet, dotp; times[0..1] =
 * generation and factorisation+solve seconds (CUDA events). */
int xg_field_loglik(XgField *f, const double *theta, double *res, double *times)
{
    int rc = xg_check_theta(theta, f->kernel);
    if (rc) return rc;
    if (!f->have_z) return xg_fail(XG_ERR_BAD_ARGUMENT, "no observations: call MLE_zvg or set z first");
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, f->C.ts, f->C.nt};
    const XgMaternParams p = xg_params(theta, f->kernel);
    const size_t Np = (size_t)f->C.nt * f->C.ts;
    XG_CU(cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st));
    XG_CU(cudaMemcpyAsync(f->v, f->z, Np * sizeof(double), cudaMemcpyDeviceToDevice, st));
    XG_CU(cudaEventRecord(f->ev[0], st));
    xg_launch_gen(T, f->C.ij, f->C.ntiles, f->x, f->y, f->x, f->y, f->N, f->N, p, f->metric, 1, st);
    XG_CU(cudaEventRecord(f->ev[1], st));
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = f->ev_panel;
    fs.ev_upd = f->ev_upd;
    fs.pev = f->profiling ? f->pev : nullptr;
    xg_factor_lookahead(f->C, f->v, f->part, f->status, f->info, fs);
    xg_launch_finalize(f->part, f->part + f->C.nt, f->C.nt, f->N, f->out, f->status, f->info, st);
    XG_CU(cudaEventRecord(f->ev[2], st));
    XG_CU(cudaMemcpyAsync(f->h_out, f->out, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    XG_CU(cudaGetLastError());
    XG_CU(cudaStreamSynchronize(st));
    if (times) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, f->ev[0], f->ev[1]);
        cudaEventElapsedTime(&b, f->ev[1], f->ev[2]);
        times[0] = a * 1e-3;
        times[1] = b * 1e-3;
    }
    if (f->profiling) xg_field_collect_profile(f);
    rc = xg_read_status(f);
    if (rc) return rc;
    res[0] = f->h_out[0];
    res[1] = f->h_out[1];
    res[2] = f->h_out[2];
    return XG_OK;
}

/* z = chol(Sigma(theta)) e, e = nrand (N host doubles) */
int xg_field_zvg(XgField *f, const double *theta, const double *nrand, double *times)
{
    int rc = xg_check_theta(theta, f->kernel);
    if (rc) return rc;
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, f->C.ts, f->C.nt};
    const XgMaternParams p = xg_params(theta, f->kernel);
    XG_CU(cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st));
    XG_CU(cudaMemcpyAsync(f->e, nrand, f->N * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaEventRecord(f->ev[0], st));
    xg_launch_gen(T, f->C.ij, f->C.ntiles, f->x, f->y, f->x, f->y, f->N, f->N, p, f->metric, 1, st);
    XG_CU(cudaEventRecord(f->ev[1], st));
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = f->ev_panel;
    fs.ev_upd = f->ev_upd;
    xg_factor_lookahead(f->C, nullptr, f->part, f->status, f->info, fs);
    xg_launch_trmv_lower(T, f->e, f->z, f->status, st);
    XG_CU(cudaEventRecord(f->ev[2], st));
    XG_CU(cudaGetLastError());
    XG_CU(cudaStreamSynchronize(st));
    /* status and info are ints on the device: widen them into the slots
     * xg_read_status reads */
    int sv[2];
    XG_CU(cudaMemcpy(sv, f->status, sizeof sv, cudaMemcpyDeviceToHost));
    f->h_out[3] = sv[0];
    f->h_out[4] = sv[1];
    if (times) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, f->ev[0], f->ev[1]);
        cudaEventElapsedTime(&b, f->ev[1], f->ev[2]);
        times[0] = a * 1e-3;
        times[1] = b * 1e-3;
    }
    rc = xg_read_status(f);
    if (rc) return rc;
    f->have_z = true;
    return XG_OK;
}

/* digamma: upward recurrence to x >= 10, then the asymptotic series
 * psi(x) = ln x - 1/(2x) - sum_k B_2k / (2k x^2k) (Abramowitz & Stegun 6.3.18) */
double xg_digamma(double x)
{
    double r = 0.0;
    while (x < 10.0) {
        r -= 1.0 / x;
        x += 1.0;
    }
    const double i2 = 1.0 / (x * x);
    const double series =
        i2 * (1.0 / 12 - i2 * (1.0 / 120 - i2 * (1.0 / 252 - i2 * (1.0 / 240 - i2 * (1.0 / 132 - i2 * (691.0 / 32760 - i2 / 12))))));
    return r + log(x) - 0.5 / x - series;
}

/* Without a nugget the Matern covariance is linear in sigma^2
 * (Sigma = sigma^2 R(beta, nu)), so dSigma/dsigma^2 = Sigma / sigma^2 and
 *   dl/dsigma^2 = (z^T Sigma^-1 z - N) / (2 sigma^2)
 * exactly, from the quadratic form of the evaluation itself; that component
 * replaces the contraction's (on the INT8-sliced path the quadratic form is
 * good to ~1e-9 while the trace of the sliced inverse is not). */
static void xg_exact_sigma2_grad(const XgField *f, const double *theta, const double *res, double *grad)
{
    if (f->kernel == 0) grad[0] = 0.5 * (res[2] - (double)f->N) / theta[0];
}

/* The gradient's inverse-factor store and contraction partials, each
 * allocated on first use (the Fisher path allocates only the store). */
static int xg_grad_workspace(XgField *f)
{
    if (!f->X.d) {
        int rc = xg_tm_alloc(f->X, f->N, f->C.ts);
        if (rc) return rc;
    }
    const long long blocks = xg_grad_contract_blocks(f->C.ntiles, f->C.ts);
    if (!f->gpart && cudaMalloc(&f->gpart, 4 * (size_t)blocks * sizeof(double)) != cudaSuccess) {
        f->gpart = nullptr;
        return xg_fail(XG_ERR_NO_MEMORY, "gradient workspace");
    }
    if (!f->gout && cudaMalloc(&f->gout, 4 * sizeof(double)) != cudaSuccess) {
        f->gout = nullptr;
        return xg_fail(XG_ERR_NO_MEMORY, "gradient workspace");
    }
    return XG_OK;
}

/* log-likelihood and its gradient (see gradient_fp64.cu for the steps);
 * grad has 3 entries (4 for the nugget kernel) */
int xg_field_loglik_grad(XgField *f, const double *theta, double *res, double *grad, double *times)
{
    int rc = xg_grad_workspace(f);
    if (rc) return rc;
    rc = xg_field_loglik(f, theta, res, times);
    if (rc) return rc;
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, f->C.ts, f->C.nt};
    const XgMaternParams p = xg_params(theta, f->kernel);
    const double dlogcon = -(log(2.0) + xg_digamma(theta[2]));
    XG_CU(cudaEventRecord(f->ev[0], st));
    for (int k = f->C.nt - 1; k >= 0; --k) xg_launch_trsv_lower_t_step(T, k, f->v, f->status, st);
    xg_launch_inverse_factor(f->X.map, f->C.map, f->X.d, f->C.d, f->C.nt, f->C.ts, f->status, st);
    xg_launch_inverse_syrk(f->X.map, f->C.d, f->C.nt, f->C.ts, f->status, st);
    xg_launch_grad_contract(f->C.d, f->C.ij, f->C.ntiles, f->C.nt, f->C.ts, f->x, f->y, f->v, f->N, p, f->kernel,
                            f->metric, dlogcon, f->gpart, f->gout, st);
    XG_CU(cudaEventRecord(f->ev[3], st));
    double g4[4];
    int sv[2];
    XG_CU(cudaGetLastError());
    XG_CU(cudaMemcpyAsync(g4, f->gout, sizeof g4, cudaMemcpyDeviceToHost, st));
    XG_CU(cudaMemcpyAsync(sv, f->status, sizeof sv, cudaMemcpyDeviceToHost, st));
    XG_CU(cudaStreamSynchronize(st));
    if (sv[0]) {
        f->h_out[3] = sv[0];
        f->h_out[4] = sv[1];
        return xg_read_status(f);
    }
    if (times) {
        float ms = 0;
        cudaEventElapsedTime(&ms, f->ev[0], f->ev[3]);
        times[2] = ms * 1e-3;
    }
    const int np = f->kernel == 1 ? 4 : 3;
    for (int i = 0; i < np; ++i) grad[i] = g4[i];
    /* the contraction kernel accumulates the nugget term in slot 3 */
    xg_exact_sigma2_grad(f, theta, res, grad);
    return XG_OK;
}

/* ------------------------------------------------------------------------- */
/* banded mixed precision                                                    */
/* ------------------------------------------------------------------------- */

/* SMs left free by the persistent trailing-update kernels (one CTA per SM,
 * ~197 KB of shared memory each) while the lookahead panel of the next step
 * (POTRF, TRSM, panel conversion) runs on the high-priority stream: resident
 * CTAs are never preempted, so without free SMs the panel would wait for the
 * whole update. */
#define XG_PANEL_SMS 16

static int xg_encode(CUtensorMap *map, CUtensorMapDataType dt, size_t esize, void *base, cuuint64_t cols,
                     cuuint64_t rows, cuuint32_t box_cols, cuuint32_t box_rows,
                     CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_128B)
{
    cuuint64_t dims[2] = {cols, rows};
    cuuint64_t strides[1] = {cols * esize};
    cuuint32_t box[2] = {box_cols, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g_encode(map, dt, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          swz, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? XG_OK : xg_fail(XG_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
}

void xg_mixed_destroy(XgMixed *m)
{
    if (!m) return;
    if (m->T.data) cudaFree(m->T.data);
    if (m->T.data32) cudaFree(m->T.data32);
    for (int b = 0; b < 2; ++b) {
        if (m->p64[b]) cudaFree(m->p64[b]);
        if (m->phi[b]) cudaFree(m->phi[b]);
        if (m->plo[b]) cudaFree(m->plo[b]);
    }
    delete m;
}

static int xg_mixed_create(XgMixed **out, int N, int ts, int band, int passes)
{
    *out = nullptr;
    if (ts % 256 != 0) return xg_fail(XG_ERR_BAD_ARGUMENT, "mixed precision needs a tile size multiple of 256 (got %d)", ts);
    if (band < 1) band = 1;
    if (passes != 1 && passes != 3) return xg_fail(XG_ERR_BAD_ARGUMENT, "TF32 passes must be 1 or 3 (got %d)", passes);
    XgMixed *m = new XgMixed();
    const int nt = (N + ts - 1) / ts;
    if (band > nt) band = nt;
    m->band = band;
    m->passes = passes;
    m->T.ts = ts;
    m->T.nt = nt;
    m->T.band = band;
    const size_t tile = (size_t)ts * ts;
    const size_t np = (size_t)nt * ts;
    int rc = XG_OK;
    double *d64 = nullptr;
    float *d32 = nullptr;
    const long long noff = xg_num_offband_tiles(nt, band);
    if (cudaMalloc(&d64, (size_t)nt * band * tile * sizeof(double)) != cudaSuccess)
        rc = xg_fail(XG_ERR_NO_MEMORY, "mixed band tiles");
    if (!rc && noff > 0 && cudaMalloc(&d32, (size_t)noff * tile * sizeof(float)) != cudaSuccess)
        rc = xg_fail(XG_ERR_NO_MEMORY, "mixed off-band tiles (%.2f GB)", noff * tile * 4.0 / 1e9);
    m->T.data = d64;
    m->T.data32 = d32;
    for (int b = 0; b < 2 && !rc; ++b) {
        if (cudaMalloc(&m->p64[b], np * ts * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&m->phi[b], np * ts * sizeof(float)) != cudaSuccess ||
            cudaMalloc(&m->plo[b], np * ts * sizeof(float)) != cudaSuccess) {
            rc = xg_fail(XG_ERR_NO_MEMORY, "mixed panel buffers");
            break;
        }
        rc = xg_encode(&m->maps[b].p64, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, m->p64[b], ts, np, 16, 128);
        if (!rc) rc = xg_encode(&m->maps[b].ahi, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, m->phi[b], ts, np, 32, 128);
        if (!rc) rc = xg_encode(&m->maps[b].bhi, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, m->phi[b], ts, np, 32, 256);
        if (!rc) rc = xg_encode(&m->maps[b].alo, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, m->plo[b], ts, np, 32, 128);
        if (!rc) rc = xg_encode(&m->maps[b].blo, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, m->plo[b], ts, np, 32, 256);
    }
    if (rc) {
        xg_mixed_destroy(m);
        return rc;
    }
    *out = m;
    return XG_OK;
}

/* Mixed factorisation with the z solve fused (v), lookahead as in the FP64
 * path: the panel of step k+1 (POTRF, band TRSM, FP32 TRSM, panel prep) runs
 * on the high-priority stream under the rest of step k's trailing update. */
static void xg_factor_mixed(XgMixed *m, double *v, double *part, int *status, int *info, const XgFactorStreams &fs)
{
    const XgTileArgs &T = m->T;
    const int nt = T.nt;
    const bool la = fs.st_hi != nullptr;
    cudaStream_t sp = la ? fs.st_hi : fs.st;
    /* profiling events, 8 per step: panel start, after POTRF, after TRSM and
     * panel prep, trailing start, after band part 1, after off-band part 1,
     * after band part 2, trailing end */
    cudaEvent_t *pev = fs.pev;
    auto rec = [&](int k, int e, cudaStream_t s) {
        if (pev) cudaEventRecord(pev[8 * k + e], s);
    };
    if (la) cudaEventRecord(fs.ev_upd, fs.st);
    for (int k = 0; k < nt; ++k) {
        const int b = k & 1;
        if (la) cudaStreamWaitEvent(sp, fs.ev_upd, 0);
        rec(k, 0, sp);
        xg_launch_potrf_diag(T, k, v, part, part + nt, v != nullptr, status, info, sp);
        rec(k, 1, sp);
        xg_launch_trsm_panel(T, k, v, v != nullptr, status, sp, k + T.band);
        xg_launch_trsm_panel32(T, k, v, v != nullptr, status, sp);
        if (k + 1 < nt) xg_launch_panel_prep(T, k, m->p64[b], m->phi[b], m->plo[b], m->passes, status, sp);
        rec(k, 2, sp);
        if (la) {
            cudaEventRecord(fs.ev_panel, sp);
            cudaStreamWaitEvent(fs.st, fs.ev_panel, 0);
        }
        rec(k, 3, fs.st);
        if (k + 1 < nt) {
            xg_launch_band_gemm(m->maps[b].p64, T, k, la ? 1 : 0, status, fs.st);
            rec(k, 4, fs.st);
            xg_launch_offband_gemm(m->maps[b], T, k, la ? 1 : 0, m->passes, g_xg.sm_count, status, fs.st);
            rec(k, 5, fs.st);
            if (la) {
                cudaEventRecord(fs.ev_upd, fs.st);
                xg_launch_band_gemm(m->maps[b].p64, T, k, 2, status, fs.st);
                rec(k, 6, fs.st);
                xg_launch_offband_gemm(m->maps[b], T, k, 2, m->passes, g_xg.sm_count - XG_PANEL_SMS, status, fs.st);
            } else {
                rec(k, 6, fs.st);
            }
        } else {
            rec(k, 4, fs.st);
            rec(k, 5, fs.st);
            rec(k, 6, fs.st);
        }
        rec(k, 7, fs.st);
    }
}

/* per-step algorithmic flops of the mixed trailing update: band targets
 * (FP64 DMMA: SYRK ts^2 (ts+1) on the diagonal tile, GEMM 2 ts^3 otherwise)
 * and off-band targets (TF32 tensor cores, 2 ts^3 each) */
static void xg_mixed_step_flops(int nt, int ts, int band, int k, double *band_flops, double *off_flops)
{
    const double t = ts;
    double bf = 0, of = 0;
    for (int j = k + 1; j < nt; ++j) {
        const int rows = nt - j; /* tiles i = j .. nt-1 in column j */
        const int nb = rows < band ? rows : band;
        bf += t * t * (t + 1) + (nb - 1) * 2 * t * t * t;
        if (rows > band) of += (double)(rows - band) * 2 * t * t * t;
    }
    *band_flops = bf;
    *off_flops = of;
}

/* Per-kernel-class times of a banded factorisation (mixed or sliced), from
 * the 8 events per step; launches_per_step counts the panel and trailing
 * launches of one step. */
void xg_field_collect_profile_banded(XgField *f, int band, double launches_per_step)
{
    const int nt = f->C.nt;
    float ms = 0;
    auto el = [&](int a, int b) {
        cudaEventElapsedTime(&ms, f->pev[a], f->pev[b]);
        return ms * 1e-3;
    };
    cudaEventElapsedTime(&ms, f->ev[0], f->ev[1]);
    f->prof[0] += ms * 1e-3;
    for (int k = 0; k < nt; ++k) {
        const int e = 8 * k;
        f->prof[1] += el(e, e + 1);
        f->prof[2] += el(e + 1, e + 2);
        if (k + 1 < nt) {
            f->prof[3] += el(e + 3, e + 7);
            double bfl, ofl;
            xg_mixed_step_flops(nt, f->C.ts, band, k, &bfl, &ofl);
            f->prof[4] += bfl + ofl;
            f->prof[8] += el(e + 4, e + 5) + el(e + 6, e + 7);
            f->prof[9] += ofl;
            f->prof[10] += el(e + 3, e + 4) + el(e + 5, e + 6);
            f->prof[11] += bfl;
        }
    }
    cudaEventElapsedTime(&ms, f->ev[0], f->ev[2]);
    f->prof[7] += ms * 1e-3;
    /* generation and finalize, then per step (upper bound: empty launches are
     * skipped on the host) */
    f->prof[5] += 2 + launches_per_step * nt;
    f->prof[6] += 1;
}

void xg_field_collect_profile_mixed(XgField *f)
{
    /* POTRF, band TRSM, FP32 TRSM, panel prep, two band and two off-band launches */
    xg_field_collect_profile_banded(f, f->mx->band, 8.0);
}

int xg_field_set_mixed(XgField *f, int band, int passes)
{
    if (f->mx && f->mx->band == band && f->mx->passes == passes) return XG_OK;
    if (f->mx) {
        xg_mixed_destroy(f->mx);
        f->mx = nullptr;
    }
    return xg_mixed_create(&f->mx, f->N, f->C.ts, band, passes);
}

int xg_field_loglik_mixed(XgField *f, const double *theta, double *res, double *times)
{
    int rc = xg_check_theta(theta, f->kernel);
    if (rc) return rc;
    if (!f->have_z) return xg_fail(XG_ERR_BAD_ARGUMENT, "no observations: call MLE_zvg or set z first");
    if (!f->mx) {
        rc = xg_field_set_mixed(f, 1, 3);
        if (rc) return rc;
    }
    XgMixed *m = f->mx;
    cudaStream_t st = g_xg.stream;
    const XgMaternParams p = xg_params(theta, f->kernel);
    const size_t Np = (size_t)f->C.nt * f->C.ts;
    XG_CU(cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st));
    XG_CU(cudaMemcpyAsync(f->v, f->z, Np * sizeof(double), cudaMemcpyDeviceToDevice, st));
    XG_CU(cudaEventRecord(f->ev[0], st));
    xg_launch_gen_mixed(m->T, f->C.ij, f->C.ntiles, f->x, f->y, f->N, p, f->metric, st);
    XG_CU(cudaEventRecord(f->ev[1], st));
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = f->ev_panel;
    fs.ev_upd = f->ev_upd;
    fs.pev = f->profiling ? f->pev : nullptr;
    xg_factor_mixed(m, f->v, f->part, f->status, f->info, fs);
    xg_launch_finalize(f->part, f->part + f->C.nt, f->C.nt, f->N, f->out, f->status, f->info, st);
    XG_CU(cudaEventRecord(f->ev[2], st));
    XG_CU(cudaMemcpyAsync(f->h_out, f->out, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    XG_CU(cudaGetLastError());
    XG_CU(cudaStreamSynchronize(st));
    if (times) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, f->ev[0], f->ev[1]);
        cudaEventElapsedTime(&b, f->ev[1], f->ev[2]);
        times[0] = a * 1e-3;
        times[1] = b * 1e-3;
    }
    if (f->profiling) xg_field_collect_profile_mixed(f);
    rc = xg_read_status(f);
    if (rc) return rc;
    res[0] = f->h_out[0];
    res[1] = f->h_out[1];
    res[2] = f->h_out[2];
    return XG_OK;
}

/* Dense mixed factor L (row-major n x n, zeros above the diagonal) for the
 * parity tests: FP64 band tiles and FP32 off-band tiles widened. */
int xg_mixed_factor_dense(int n, const double *x, const double *y, const double *theta, int kernel, int metric, int ts,
                          int band, int passes, double *out)
{
    XgField *f = nullptr;
    int rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    rc = xg_field_create(&f, n, ts, x, y, kernel, metric);
    if (rc) return rc;
    rc = xg_field_set_mixed(f, band, passes);
    if (rc) {
        xg_field_destroy(f);
        return rc;
    }
    XgMixed *m = f->mx;
    cudaStream_t st = g_xg.stream;
    cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st);
    xg_launch_gen_mixed(m->T, f->C.ij, f->C.ntiles, f->x, f->y, n, xg_params(theta, kernel), metric, st);
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = f->ev_panel;
    fs.ev_upd = f->ev_upd;
    xg_factor_mixed(m, nullptr, f->part, f->status, f->info, fs);
    cudaError_t e = cudaGetLastError();
    const int nt = m->T.nt, tsz = m->T.ts;
    const size_t tile = (size_t)tsz * tsz;
    std::vector<double> h64((size_t)nt * m->band * tile);
    const long long noff = xg_num_offband_tiles(nt, m->band);
    std::vector<float> h32((size_t)noff * tile);
    int sv[2] = {0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h64.data(), m->T.data, h64.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess && noff)
        e = cudaMemcpyAsync(h32.data(), m->T.data32, h32.size() * sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sv, f->status, sizeof sv, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = xg_cuda_fail(e, "mixed factor");
    if (!rc && sv[0]) rc = xg_fail(sv[0] & XG_ST_NOT_SPD ? XG_ERR_NOT_SPD : XG_ERR_TIMEOUT, "status 0x%x", sv[0]);
    if (!rc)
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                double val = 0.0;
                if (c <= r) {
                    const int i = r / tsz, j = c / tsz;
                    const size_t off = (size_t)(r % tsz) * tsz + (c % tsz);
                    if (i - j < m->band)
                        val = h64[(size_t)xg_slot64(m->T, i, j) * tile + off];
                    else
                        val = h32[(size_t)xg_slot32(i, j, nt, m->band) * tile + off];
                }
                out[(size_t)r * n + c] = val;
            }
    xg_field_destroy(f);
    return rc;
}

/* Copies the lower-tile store of f to a dense row-major n x n array (zeros
 * above the diagonal), after the stream's work; reads the status word. */
static int xg_tiles_to_dense(XgField *f, int n, double *out)
{
    cudaStream_t st = g_xg.stream;
    int rc = XG_OK;
    cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return xg_cuda_fail(le, "dense copy launch");
    const int tsz = f->C.ts;
    const size_t tile_elems = (size_t)tsz * tsz;
    double *h = (double *)malloc(f->C.ntiles * tile_elems * sizeof(double));
    if (!h) return xg_fail(XG_ERR_NO_MEMORY, "host copy of the tiles");
    int sv[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, f->C.d, f->C.ntiles * tile_elems * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(sv, f->status, sizeof sv, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = xg_cuda_fail(e, "tile download");
    if (!rc && (sv[0] & XG_ST_NOT_SPD)) rc = xg_fail(XG_ERR_NOT_SPD, "not positive definite (pivot %d)", sv[1]);
    if (!rc && sv[0]) rc = xg_fail(XG_ERR_TIMEOUT, "device status word 0x%x", sv[0]);
    if (!rc) {
        for (int r = 0; r < n; ++r)
            for (int c = 0; c < n; ++c) {
                double val = 0.0;
                if (c <= r) {
                    const int i = r / tsz, j = c / tsz;
                    val = h[xg_tile_index(i, j, f->C.nt) * tile_elems + (size_t)(r % tsz) * tsz + (c % tsz)];
                }
                out[(size_t)r * n + c] = val;
            }
    }
    free(h);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* FP64 tiles, INT8-sliced off-band updates                                  */
/* ------------------------------------------------------------------------- */

void xg_sliced_destroy(XgSliced *s)
{
    if (!s) return;
    if (s->dig) cudaFree(s->dig);
    if (s->scale) cudaFree(s->scale);
    if (s->xdig) cudaFree(s->xdig);
    if (s->xscale) cudaFree(s->xscale);
    if (s->ev_a) cudaEventDestroy(s->ev_a);
    for (int b = 0; b < 2; ++b)
        if (s->ev_p[b]) cudaEventDestroy(s->ev_p[b]);
    delete s;
}

int xg_field_set_sliced(XgField *f)
{
    if (f->sl) return XG_OK;
    const int ts = f->C.ts;
    if (ts % 128 != 0) return xg_fail(XG_ERR_BAD_ARGUMENT, "the sliced path needs a tile size multiple of 128");
    XgSliced *s = new XgSliced();
    s->plane_rows = f->C.ntiles * ts;
    const size_t plane = (size_t)s->plane_rows * ts;
    int rc = XG_OK;
    if (4 * s->plane_rows > 0x7fffffffLL)
        rc = xg_fail(XG_ERR_BAD_ARGUMENT, "N = %d is beyond the sliced path's 2^31-row digit store", f->N);
    if (!rc && (cudaMalloc(&s->dig, 4 * plane) != cudaSuccess ||
                cudaMalloc(&s->scale, (size_t)s->plane_rows * sizeof(double)) != cudaSuccess))
        rc = xg_fail(XG_ERR_NO_MEMORY, "digit planes (%.2f GB)", 4.0 * plane / 1e9);
    /* both operands are staged in boxes of 128 rows x 64 bytes */
    if (!rc)
        rc = xg_encode(&s->map_a, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, s->dig, ts, 4 * s->plane_rows, 64, 128,
                       CU_TENSOR_MAP_SWIZZLE_64B);
    if (!rc) s->map_b = s->map_a;
    if (!rc && (cudaEventCreateWithFlags(&s->ev_a, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&s->ev_p[0], cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&s->ev_p[1], cudaEventDisableTiming) != cudaSuccess))
        rc = xg_fail(XG_ERR_CUDA, "sliced lookahead events");
    if (rc) {
        xg_sliced_destroy(s);
        return rc;
    }
    f->sl = s;
    return XG_OK;
}

/* Left-looking factorisation with FP64 tiles and INT8-sliced updates.  For
 * each column j:
 *   update  : A_ij -= sum_{k<j} L_ik L_jk^T for i >= j (xg_sliced_left_kernel)
 *   panel   : POTRF(j, j) [+ log-det, + z block solve] -> TRSM(i, j) [+ z update]
 *             -> slicing of the tiles (i, j), i > j, into digit planes
 * With fs.st_hi the update of column j+1 is split: chunks k < j (needing
 * panels already sliced) run on the main stream on all but xg_panel_share(j)
 * SMs while the panel chain of column j runs on the high-priority stream, and
 * chunk k = j joins the panel chain of column j+1.  Profiling events (8 per
 * column): panel stream before / after the last-chunk update, after POTRF,
 * after TRSM + slicing; main stream before / after the split update. */
static XgSlTask factor_task(int col, int k0, int k1)
{
    XgSlTask S;
    S.mode = XG_SL_FACTOR;
    S.col = col;
    S.k0 = k0;
    S.k1 = k1;
    S.sign = -1.0;
    S.overwrite = 0;
    return S;
}

/* SMs given to the panel chain of column j (last-chunk update, POTRF, TRSM,
 * slicing) while the split update of column j+1 runs on the others.  The
 * chain's work grows like nt - j and the split update's like j (nt - j), so
 * the chain gets sms K / (K + j), clamped to [XG_PANEL_SMS, sms -
 * XG_PANEL_SMS].  K = 4 (EXAGEOSTAT_B200_PANEL_K overrides it) measured best
 * at N = 100 000 with the 128-column-block TRSM: 1.589-1.644 s per
 * evaluation against 1.614-1.665 s for K = 2, 3, 6, 8, 1.624 s for a cost
 * model balancing the chain against the update, and 1.639 s for that model
 * with the update's round count in it (each compared within one GPU
 * session; the sessions differ by up to 3 %). */
static int xg_panel_k()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("EXAGEOSTAT_B200_PANEL_K");
        v = e ? atoi(e) : 0;
        if (v < 1 || v > 64) v = 4;
    }
    return v;
}

static int xg_panel_share(int j, int sms)
{
    const int K = xg_panel_k();
    int r = (int)((long long)sms * K / (K + j));
    if (r < XG_PANEL_SMS) r = XG_PANEL_SMS;
    if (r > sms - XG_PANEL_SMS) r = sms - XG_PANEL_SMS;
    return r;
}

/* How the SMs are divided between the panel chain and the split update.
 * "static" (default): the split update runs as a persistent launch on
 * sms - xg_panel_share(j) CTAs, leaving the rest to the panel chain.
 * "dynamic" (EXAGEOSTAT_B200_SL_SHARE=dynamic): both updates launch one CTA
 * per job, so CTAs retire throughout the update and the hardware hands each
 * freed SM to the pending panel kernels first (higher stream priority), the
 * SMs the chain does not need staying with the update. */
static bool xg_sl_dynamic_share()
{
    static int v = -1;
    if (v < 0) {
        const char *e = getenv("EXAGEOSTAT_B200_SL_SHARE");
        v = (e && strcmp(e, "dynamic") == 0) ? 1 : 0;
    }
    return v == 1;
}

static void xg_factor_sliced(XgField *f, double *v, const XgFactorStreams &fs)
{
    XgSliced *sl = f->sl;
    XgTileMatrix &M = f->C;
    XgTileArgs T{M.d, M.ts, M.nt};
    T.dinv = M.dinv;
    const int nt = M.nt;
    const long long plane = sl->plane_rows * M.ts;
    const int pr = (int)sl->plane_rows;
    const bool la = fs.st_hi != nullptr;
    cudaStream_t sp = la ? fs.st_hi : fs.st;
    cudaEvent_t *pev = fs.pev;
    auto rec = [&](int k, int e, cudaStream_t s) {
        if (pev) cudaEventRecord(pev[8 * k + e], s);
    };
    const int rhs = v != nullptr;
    const int sms = g_xg.sm_count;
    const bool dyn = xg_sl_dynamic_share();
    const int all = 1 << 30; /* one CTA per job */
    if (la) cudaEventRecord(sl->ev_a, fs.st); /* the generated matrix */
    for (int j = 0; j < nt; ++j) {
        if (la) cudaStreamWaitEvent(sp, sl->ev_a, 0); /* chunks k < j-1 of column j */
        rec(j, 0, sp);
        const int band_ctas = xg_panel_share(j, sms), upd_ctas = sms - band_ctas;
        if (la) {
            if (j >= 1) xg_launch_sliced(sl->map_a, sl->map_b, sl->scale, sl->scale, T, factor_task(j, j - 1, j), pr,
                                         dyn ? all : band_ctas, f->status, sp);
        } else {
            xg_launch_sliced(sl->map_a, sl->map_b, sl->scale, sl->scale, T, factor_task(j, 0, j), pr, sms, f->status,
                             sp);
        }
        rec(j, 1, sp);
        xg_launch_potrf_tiled(M.map, T, j, v, f->part, f->part + nt, rhs, f->status, f->info, sp);
        rec(j, 2, sp);
        if (T.dinv)
            xg_launch_trsm_gemm(M.map, T, j, v, rhs, f->status, sp);
        else
            xg_launch_trsm_panel(T, j, v, rhs, f->status, sp);
        if (j + 1 < nt) xg_launch_slice_panel(T, j, 0, sl->dig, sl->scale, plane, f->status, sp);
        rec(j, 3, sp);
        if (la) {
            cudaEventRecord(sl->ev_p[j & 1], sp);
            /* chunks k < j of column j+1, behind the slicing of panel j-1 */
            if (j >= 1 && j + 1 < nt) cudaStreamWaitEvent(fs.st, sl->ev_p[(j - 1) & 1], 0);
            rec(j, 4, fs.st);
            if (j >= 1 && j + 1 < nt)
                xg_launch_sliced(sl->map_a, sl->map_b, sl->scale, sl->scale, T, factor_task(j + 1, 0, j), pr,
                                 dyn ? all : upd_ctas, f->status, fs.st);
            rec(j, 5, fs.st);
            cudaEventRecord(sl->ev_a, fs.st);
        } else {
            rec(j, 4, fs.st);
            rec(j, 5, fs.st);
        }
        rec(j, 6, fs.st);
        rec(j, 7, fs.st);
    }
    if (la) {
        cudaEventRecord(fs.ev_panel, sp);
        cudaStreamWaitEvent(fs.st, fs.ev_panel, 0);
    }
}

/* Per-kernel-class times of the sliced factorisation from its events:
 * prof[8], prof[9] = seconds and algorithmic flops of the split updates on
 * the main stream (chunks k < j-1 of column j: nearly all the work);
 * prof[10], prof[11] = the same for the last-chunk updates on the panel
 * stream (all chunks of a column without the lookahead). */
static void xg_field_collect_profile_sliced(XgField *f, bool lookahead)
{
    const int nt = f->C.nt;
    const double t = f->C.ts;
    float ms = 0;
    auto el = [&](int a, int b) {
        cudaEventElapsedTime(&ms, f->pev[a], f->pev[b]);
        return ms * 1e-3;
    };
    /* algorithmic flops of `chunks` panel chunks applied to column j */
    auto col_flops = [&](int j, int chunks) {
        return (double)chunks * ((nt - j - 1) * 2.0 * t * t * t + t * t * (t + 1));
    };
    cudaEventElapsedTime(&ms, f->ev[0], f->ev[1]);
    f->prof[0] += ms * 1e-3;
    for (int j = 0; j < nt; ++j) {
        const int e = 8 * j;
        f->prof[1] += el(e + 1, e + 2);
        f->prof[2] += el(e + 2, e + 3);
        const double tb = el(e, e + 1), ta = el(e + 4, e + 5);
        f->prof[3] += ta + tb;
        f->prof[4] += col_flops(j, j);
        if (lookahead) {
            f->prof[10] += tb;
            f->prof[11] += j >= 1 ? col_flops(j, 1) : 0.0;
            f->prof[8] += ta;
            f->prof[9] += (j >= 1 && j + 1 < nt) ? col_flops(j + 1, j) : 0.0;
        } else {
            f->prof[8] += tb;
            f->prof[9] += col_flops(j, j);
        }
    }
    cudaEventElapsedTime(&ms, f->ev[0], f->ev[2]);
    f->prof[7] += ms * 1e-3;
    /* generation, finalize; per column two update launches, the sub-block POTRF
     * sequence, TRSM, slicing */
    f->prof[5] += 2 + (4.0 + xg_potrf_tiled_launches(f->C.ts)) * nt;
    f->prof[6] += 1;
}

int xg_field_loglik_sliced(XgField *f, const double *theta, double *res, double *times)
{
    int rc = xg_check_theta(theta, f->kernel);
    if (rc) return rc;
    if (!f->have_z) return xg_fail(XG_ERR_BAD_ARGUMENT, "no observations: call MLE_zvg or set z first");
    if (!f->sl) {
        rc = xg_field_set_sliced(f);
        if (rc) return rc;
    }
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, f->C.ts, f->C.nt};
    const XgMaternParams p = xg_params(theta, f->kernel);
    const size_t Np = (size_t)f->C.nt * f->C.ts;
    XG_CU(cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st));
    XG_CU(cudaMemcpyAsync(f->v, f->z, Np * sizeof(double), cudaMemcpyDeviceToDevice, st));
    XG_CU(cudaEventRecord(f->ev[0], st));
    xg_launch_gen(T, f->C.ij, f->C.ntiles, f->x, f->y, f->x, f->y, f->N, f->N, p, f->metric, 1, st);
    XG_CU(cudaEventRecord(f->ev[1], st));
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = f->ev_panel;
    fs.ev_upd = f->ev_upd;
    fs.pev = f->profiling ? f->pev : nullptr;
    xg_factor_sliced(f, f->v, fs);
    xg_launch_finalize(f->part, f->part + f->C.nt, f->C.nt, f->N, f->out, f->status, f->info, st);
    XG_CU(cudaEventRecord(f->ev[2], st));
    XG_CU(cudaMemcpyAsync(f->h_out, f->out, 5 * sizeof(double), cudaMemcpyDeviceToHost, st));
    XG_CU(cudaGetLastError());
    XG_CU(cudaStreamSynchronize(st));
    if (times) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, f->ev[0], f->ev[1]);
        cudaEventElapsedTime(&b, f->ev[1], f->ev[2]);
        times[0] = a * 1e-3;
        times[1] = b * 1e-3;
    }
    if (f->profiling) xg_field_collect_profile_sliced(f, fs.st_hi != nullptr);
    rc = xg_read_status(f);
    if (rc) return rc;
    res[0] = f->h_out[0];
    res[1] = f->h_out[1];
    res[2] = f->h_out[2];
    return XG_OK;
}

/* Dense factor L (row-major n x n, zeros above the diagonal) of the sliced
 * path, for the parity tests. */
int xg_sliced_factor_dense(int n, const double *x, const double *y, const double *theta, int kernel, int metric,
                           int ts, double *out)
{
    XgField *f = nullptr;
    int rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    rc = xg_field_create(&f, n, ts, x, y, kernel, metric);
    if (!rc) rc = xg_field_set_sliced(f);
    if (rc) {
        xg_field_destroy(f);
        return rc;
    }
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, f->C.ts, f->C.nt};
    cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st);
    xg_launch_gen(T, f->C.ij, f->C.ntiles, f->x, f->y, f->x, f->y, n, n, xg_params(theta, kernel), metric, 1, st);
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = f->ev_panel;
    fs.ev_upd = f->ev_upd;
    xg_factor_sliced(f, nullptr, fs);
    rc = xg_tiles_to_dense(f, n, out);
    xg_field_destroy(f);
    return rc;
}

/* Gradient with the sliced path: the forward factorisation as
 * xg_field_loglik_sliced, alpha = L^-T v in FP64, the inverse factor
 * X = L^-T column by column (INT8-sliced update from the digit planes of L and
 * of the already finished columns of X, then the FP64 triangular solve with
 * L_bb^T and the slicing of column b of X), S = X X^T by one sliced launch
 * written over the factor, and the FP64 contraction with dSigma/dtheta. */
int xg_field_loglik_grad_sliced(XgField *f, const double *theta, double *res, double *grad, double *times)
{
    int rc = XG_OK;
    if (!f->sl && (rc = xg_field_set_sliced(f))) return rc;
    XgSliced *sl = f->sl;
    if ((rc = xg_grad_workspace(f))) return rc;
    const int ts = f->C.ts, nt = f->C.nt;
    const size_t plane = (size_t)sl->plane_rows * ts;
    if (!sl->xdig) {
        if (cudaMalloc(&sl->xdig, 4 * plane) != cudaSuccess ||
            cudaMalloc(&sl->xscale, (size_t)sl->plane_rows * sizeof(double)) != cudaSuccess)
            return xg_fail(XG_ERR_NO_MEMORY, "digit planes of the inverse factor (%.2f GB)", 4.0 * plane / 1e9);
        rc = xg_encode(&sl->xmap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, sl->xdig, ts, 4 * sl->plane_rows, 64, 128,
                       CU_TENSOR_MAP_SWIZZLE_64B);
        if (rc) return rc;
    }
    rc = xg_field_loglik_sliced(f, theta, res, times);
    if (rc) return rc;
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, ts, nt};
    XgTileArgs TX{f->X.d, ts, nt};
    const int pr = (int)sl->plane_rows;
    const XgMaternParams p = xg_params(theta, f->kernel);
    const double dlogcon = -(log(2.0) + xg_digamma(theta[2]));
    XG_CU(cudaEventRecord(f->ev[0], st));
    for (int k = nt - 1; k >= 0; --k) xg_launch_trsv_lower_t_step(T, k, f->v, f->status, st);
    xg_launch_identity_x(f->X.d, nt, ts, st);
    /* X = L^-T column by column: the update of column b from the finished
     * columns c < b (INT8-sliced), the FP64 solve with L_bb, the slicing of
     * column b.  (Overlapping the solve and slicing of column b with the
     * update of column b + 1 on two streams, as the factorisation does, was
     * measured at the same 5.87 s per gradient at N = 100 000: the update
     * dominates each column.) */
    for (int b = 0; b < nt; ++b) {
        if (b >= 1) {
            XgSlTask S;
            S.mode = XG_SL_INVERSE;
            S.col = b;
            S.k0 = 0;
            S.k1 = b;
            S.sign = -1.0;
            S.overwrite = 0;
            xg_launch_sliced(sl->xmap, sl->map_b, sl->xscale, sl->scale, TX, S, pr, g_xg.sm_count, f->status, st);
        }
        xg_launch_xtrsm(f->X.d, f->C.d, nt, ts, b, f->status, st);
        xg_launch_slice_panel(TX, b, 1, sl->xdig, sl->xscale, (long long)plane, f->status, st);
    }
    XgSlTask S;
    S.mode = XG_SL_SYRK;
    S.col = 0;
    S.k0 = 0;
    S.k1 = nt;
    S.sign = 1.0;
    S.overwrite = 1;
    xg_launch_sliced(sl->xmap, sl->xmap, sl->xscale, sl->xscale, T, S, pr, g_xg.sm_count, f->status, st);
    xg_launch_grad_contract(f->C.d, f->C.ij, f->C.ntiles, nt, ts, f->x, f->y, f->v, f->N, p, f->kernel, f->metric,
                            dlogcon, f->gpart, f->gout, st);
    XG_CU(cudaEventRecord(f->ev[3], st));
    double g4[4];
    int sv[2];
    XG_CU(cudaGetLastError());
    XG_CU(cudaMemcpyAsync(g4, f->gout, sizeof g4, cudaMemcpyDeviceToHost, st));
    XG_CU(cudaMemcpyAsync(sv, f->status, sizeof sv, cudaMemcpyDeviceToHost, st));
    XG_CU(cudaStreamSynchronize(st));
    if (sv[0]) {
        f->h_out[3] = sv[0];
        f->h_out[4] = sv[1];
        return xg_read_status(f);
    }
    if (times) {
        float ms = 0;
        cudaEventElapsedTime(&ms, f->ev[0], f->ev[3]);
        times[2] = ms * 1e-3;
    }
    const int np = f->kernel == 1 ? 4 : 3;
    for (int i = 0; i < np; ++i) grad[i] = g4[i];
    xg_exact_sigma2_grad(f, theta, res, grad);
    return XG_OK;
}

/* ------------------------------------------------------------------------- */
/* autotuner                                                                 */
/* ------------------------------------------------------------------------- */

/* seconds (CUDA events, generation to result) of one evaluation of f in the
 * given precision after a warm-up one; < 0 on failure; res receives loglik */
static double xg_time_eval(XgField *f, const double *theta, int precision, double *ll)
{
    double res[3], t[3] = {0, 0, 0};
    for (int rep = 0; rep < 2; ++rep) {
        const int rc = precision == 2   ? xg_field_loglik_mixed(f, theta, res, t)
                       : precision == 3 ? xg_field_loglik_sliced(f, theta, res, t)
                                        : xg_field_loglik(f, theta, res, t);
        if (rc) return -1.0;
    }
    if (ll) *ll = res[0];
    return t[0] + t[1];
}

/* Tile size (and, for precision 2, band width) chosen by timing.  Tile
 * sizes 128, 256, 384, 512 (multiples of 256 for precision 2) up to the
 * field size are timed on temporary fields with the same locations and
 * observations; *pf is rebuilt with the fastest.  For precision 2 the band
 * widths 1, 2, 4, 8 are then timed and the fastest whose |dl| / |l| against
 * one FP64 evaluation is <= tol is kept (the most accurate if none is).
 * report receives (ts, seconds) pairs, 4 entries at most. */
int xg_autotune_field(XgField **pf, const double *x, const double *y, const double *theta, int precision, double tol,
                      int *ts_out, int *band_out, double *report)
{
    XgField *f = *pf;
    if (precision == 2 && xg_bivariate(f->kernel))
        return xg_fail(XG_ERR_UNSUPPORTED, "banded mixed precision with bivariate_matern_parsimonious");
    const int N = f->N;
    std::vector<double> z(N);
    int rc = xg_field_get_z(f, z.data(), N);
    if (rc) return rc;
    const int cands[4] = {128, 256, 384, 512};
    int best_ts = f->C.ts, nrep = 0;
    double best_t = -1.0;
    for (int c = 0; c < 4; ++c) {
        const int ts = cands[c];
        if (precision == 2 && ts % 256) continue;
        if (ts > 128 && ts / 2 >= N) continue; /* a single half-empty tile */
        XgField *t = nullptr;
        if (xg_field_create(&t, N, ts, x, y, f->kernel, f->metric)) continue;
        double sec = -1.0;
        if (!xg_field_set_z(t, z.data()) &&
            (precision != 2 || !xg_field_set_mixed(t, f->mx ? f->mx->band : 1, 3)) &&
            (precision != 3 || !xg_field_set_sliced(t)))
            sec = xg_time_eval(t, theta, precision, nullptr);
        xg_field_destroy(t);
        if (sec < 0) continue;
        if (report && nrep < 4) {
            report[2 * nrep] = ts;
            report[2 * nrep + 1] = sec;
            ++nrep;
        }
        if (best_t < 0 || sec < best_t) {
            best_t = sec;
            best_ts = ts;
        }
    }
    if (best_t < 0) return xg_fail(XG_ERR_CUDA, "autotune: no tile size could be timed");
    if (best_ts != f->C.ts) {
        XgField *g = nullptr;
        rc = xg_field_create(&g, N, best_ts, x, y, f->kernel, f->metric);
        if (!rc) rc = xg_field_set_z(g, z.data());
        if (rc) {
            if (g) xg_field_destroy(g);
            return rc;
        }
        g->profiling = false;
        xg_field_destroy(f);
        *pf = f = g;
    }
    *ts_out = best_ts;
    *band_out = 0;
    if (precision == 2) {
        double ll64 = 0;
        if (xg_time_eval(f, theta, 0, &ll64) < 0) return xg_fail(XG_ERR_CUDA, "autotune: FP64 reference evaluation");
        int best_band = 1, acc_band = 1;
        double bt = -1.0, best_err = 1e300;
        const int bands[4] = {1, 2, 4, 8};
        for (int b = 0; b < 4; ++b) {
            if (bands[b] > f->C.nt) break;
            if (xg_field_set_mixed(f, bands[b], 3)) continue;
            double ll = 0;
            const double sec = xg_time_eval(f, theta, 2, &ll);
            if (sec < 0) continue;
            const double err = fabs(ll - ll64) / fabs(ll64);
            if (err <= tol && (bt < 0 || sec < bt)) {
                bt = sec;
                best_band = bands[b];
            }
            if (err < best_err) {
                best_err = err;
                acc_band = bands[b];
            }
        }
        const int band = bt >= 0 ? best_band : acc_band;
        rc = xg_field_set_mixed(f, band, 3);
        if (rc) return rc;
        *band_out = band;
    }
    return XG_OK;
}

int xg_field_get_z(XgField *f, double *z, int n)
{
    if (!f->have_z) return xg_fail(XG_ERR_BAD_ARGUMENT, "no observations generated yet");
    if (n > f->N) n = f->N;
    XG_CU(cudaMemcpy(z, f->z, n * sizeof(double), cudaMemcpyDeviceToHost));
    return XG_OK;
}

/* ------------------------------------------------------------------------- */
/* kriging                                                                   */
/* ------------------------------------------------------------------------- */

void xg_predict_destroy(XgPredict *q)
{
    if (!q) return;
    xg_tm_free(q->C22);
    double *bufs[] = {q->xm, q->ym, q->xo, q->yo, q->v, q->zact, q->zmiss, q->part, q->out};
    for (double *b : bufs)
        if (b) cudaFree(b);
    if (q->status) cudaFree(q->status);
    if (q->ev_panel) cudaEventDestroy(q->ev_panel);
    if (q->ev_upd) cudaEventDestroy(q->ev_upd);
    delete q;
}

int xg_predict_create(XgPredict **out, int nmiss, int nobs, int ts)
{
    *out = nullptr;
    int rc = xg_context_require();
    if (rc) return rc;
    if (nmiss <= 0 || nobs <= 0) return xg_fail(XG_ERR_BAD_ARGUMENT, "nZmiss = %d, nZobs = %d", nmiss, nobs);
    XgPredict *q = new XgPredict();
    q->nmiss = nmiss;
    q->nobs = nobs;
    rc = xg_tm_alloc(q->C22, nobs, xg_choose_ts(nobs, ts));
    const size_t Np = (size_t)q->C22.nt * q->C22.ts;
    if (!rc) rc = xg_dev_alloc(&q->xo, Np);
    if (!rc) rc = xg_dev_alloc(&q->yo, Np);
    if (!rc) rc = xg_dev_alloc(&q->v, Np);
    if (!rc) rc = xg_dev_alloc(&q->xm, nmiss);
    if (!rc) rc = xg_dev_alloc(&q->ym, nmiss);
    if (!rc) rc = xg_dev_alloc(&q->zact, nmiss);
    if (!rc) rc = xg_dev_alloc(&q->zmiss, nmiss);
    if (!rc) rc = xg_dev_alloc(&q->part, 2 * (size_t)q->C22.nt);
    if (!rc) rc = xg_dev_alloc(&q->out, 8);
    if (!rc && cudaMalloc(&q->status, 2 * sizeof(int)) != cudaSuccess) rc = xg_fail(XG_ERR_NO_MEMORY, "status");
    if (!rc && (cudaEventCreateWithFlags(&q->ev_panel, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventCreateWithFlags(&q->ev_upd, cudaEventDisableTiming) != cudaSuccess))
        rc = xg_fail(XG_ERR_CUDA, "lookahead events");
    if (rc) {
        xg_predict_destroy(q);
        return rc;
    }
    *out = q;
    return XG_OK;
}

int xg_predict_run(XgPredict *q, const double *theta, int kernel, int metric, const double *xm, const double *ym,
                   const double *xo, const double *yo, const double *zobs, const double *zactual, double *zmiss,
                   double *mse, double *mse_parts)
{
    int rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    if (xg_bivariate(kernel) && ((q->nmiss | q->nobs) & 1))
        return xg_fail(XG_ERR_BAD_ARGUMENT, "bivariate kriging: nZmiss = %d and nZobs = %d must be even (2 x locations)",
                       q->nmiss, q->nobs);
    cudaStream_t st = g_xg.stream;
    const int nmiss = q->nmiss, nobs = q->nobs;
    /* bivariate: nmiss and nobs count matrix rows, two per location */
    const int lmiss = xg_bivariate(kernel) ? nmiss / 2 : nmiss, lobs = xg_bivariate(kernel) ? nobs / 2 : nobs;
    XgTileArgs T{q->C22.d, q->C22.ts, q->C22.nt};
    const XgMaternParams p = xg_params(theta, kernel);
    const size_t Np = (size_t)q->C22.nt * q->C22.ts;
    XG_CU(cudaMemsetAsync(q->status, 0, 2 * sizeof(int), st));
    XG_CU(cudaMemsetAsync(q->v, 0, Np * sizeof(double), st));
    XG_CU(cudaMemcpyAsync(q->xo, xo, lobs * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaMemcpyAsync(q->yo, yo, lobs * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaMemcpyAsync(q->v, zobs, nobs * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaMemcpyAsync(q->xm, xm, lmiss * sizeof(double), cudaMemcpyHostToDevice, st));
    XG_CU(cudaMemcpyAsync(q->ym, ym, lmiss * sizeof(double), cudaMemcpyHostToDevice, st));
    if (zactual) XG_CU(cudaMemcpyAsync(q->zact, zactual, nmiss * sizeof(double), cudaMemcpyHostToDevice, st));
    /* C22 = Sigma(obs, obs); POSV: L L^T alpha = zobs */
    xg_launch_gen(T, q->C22.ij, q->C22.ntiles, q->xo, q->yo, q->xo, q->yo, nobs, nobs, p, metric, 1, st);
    XgFactorStreams fs;
    fs.st = st;
    fs.st_hi = g_xg.stream_hi;
    fs.ev_panel = q->ev_panel;
    fs.ev_upd = q->ev_upd;
    xg_factor_lookahead(q->C22, q->v, q->part, q->status, q->info(), fs);
    for (int k = q->C22.nt - 1; k >= 0; --k) xg_launch_trsv_lower_t_step(T, k, q->v, q->status, st);
    /* zmiss = Sigma(miss, obs) alpha, C12 generated on the fly */
    xg_launch_predict_cross(q->xm, q->ym, nmiss, q->xo, q->yo, nobs, q->v, p, metric, q->zmiss, st);
    if (zactual) xg_launch_mse(q->zact, q->zmiss, nmiss, q->out, st);
    XG_CU(cudaGetLastError());
    int sv[2];
    XG_CU(cudaMemcpyAsync(sv, q->status, sizeof sv, cudaMemcpyDeviceToHost, st));
    XG_CU(cudaMemcpyAsync(zmiss, q->zmiss, nmiss * sizeof(double), cudaMemcpyDeviceToHost, st));
    double m[3] = {-1, -1, -1};
    if (zactual) XG_CU(cudaMemcpyAsync(m, q->out, sizeof m, cudaMemcpyDeviceToHost, st));
    XG_CU(cudaStreamSynchronize(st));
    if (sv[0] & XG_ST_NOT_SPD) return xg_fail(XG_ERR_NOT_SPD, "C22 is not positive definite (pivot %d)", sv[1]);
    if (sv[0]) return xg_fail(XG_ERR_TIMEOUT, "device status word 0x%x", sv[0]);
    *mse = zactual ? m[0] : -1.0;
    if (mse_parts) {
        mse_parts[0] = zactual ? m[1] : -1.0;
        mse_parts[1] = zactual ? m[2] : -1.0;
    }
    return XG_OK;
}

/* ------------------------------------------------------------------------- */
/* dense diagnostics                                                         */
/* ------------------------------------------------------------------------- */

int xg_covariance_dense(int n, const double *x, const double *y, const double *theta, int kernel, int metric, int ts,
                        int factor, double *out)
{
    XgField *f = nullptr;
    int rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    rc = xg_field_create(&f, n, ts, x, y, kernel, metric);
    if (rc) return rc;
    cudaStream_t st = g_xg.stream;
    XgTileArgs T{f->C.d, f->C.ts, f->C.nt};
    const XgMaternParams p = xg_params(theta, kernel);
    cudaMemsetAsync(f->status, 0, 2 * sizeof(int), st);
    xg_launch_gen(T, f->C.ij, f->C.ntiles, f->x, f->y, f->x, f->y, n, n, p, metric, 1, st);
    if (factor) xg_factor(f->C, nullptr, f->part, f->status, f->info, st);
    rc = xg_tiles_to_dense(f, n, out);
    xg_field_destroy(f);
    return rc;
}

int xg_bessel_knu_host(int n, const double *nu, const double *x, double *out)
{
    int rc = xg_context_require();
    if (rc) return rc;
    if (n <= 0) return XG_OK;
    double *d = nullptr;
    XG_CU(cudaMalloc(&d, 3 * (size_t)n * sizeof(double)));
    cudaStream_t st = g_xg.stream;
    cudaMemcpyAsync(d, nu, n * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d + n, x, n * sizeof(double), cudaMemcpyHostToDevice, st);
    xg_launch_bessel(d, d + n, n, d + 2 * (size_t)n, st);
    cudaMemcpyAsync(out, d + 2 * (size_t)n, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return xg_cuda_fail(e, "bessel");
    return XG_OK;
}

int xg_matern_pairs_host(int n, const double *x1, const double *y1, const double *x2, const double *y2,
                         const double *theta, int kernel, int metric, double *out)
{
    int rc = xg_context_require();
    if (rc) return rc;
    rc = xg_check_theta(theta, kernel);
    if (rc) return rc;
    if (n <= 0) return XG_OK;
    double *d = nullptr;
    XG_CU(cudaMalloc(&d, 5 * (size_t)n * sizeof(double)));
    cudaStream_t st = g_xg.stream;
    const double *src[4] = {x1, y1, x2, y2};
    for (int i = 0; i < 4; ++i)
        cudaMemcpyAsync(d + (size_t)i * n, src[i], n * sizeof(double), cudaMemcpyHostToDevice, st);
    xg_launch_matern_pairs(d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, n, xg_params(theta, kernel), metric,
                           d + 4 * (size_t)n, st);
    if (cudaGetLastError() != cudaSuccess) {
        cudaFree(d);
        return xg_fail(XG_ERR_CUDA, "matern pairs launch failed");
    }
    cudaMemcpyAsync(out, d + 4 * (size_t)n, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return xg_cuda_fail(e, "matern pairs");
    return XG_OK;
}
