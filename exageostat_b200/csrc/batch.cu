/*
 * Many independent regional fields in one graph launch.
 *
 * The reference evaluates one field per MLE_data; a study of many regions
 * loops over the exact path.  Here every field of a batch shares one lower-tile
 * store (fields packed one after the other, one TMA tensor over all of them).
 * Generation is one launch over every tile of every field; the whole
 * factorisation (with the fused log-det and z solve) of all fields is ONE
 * persistent launch driven by a device-resident tile scheduler
 * (xg_batch_sched_kernel): the task list -- every POTRF, TRSM and trailing
 * tile update of every field, in one topological order built here -- is
 * taken by persistent CTAs, each task waiting (bounded) on per-tile
 * dependency counters and publishing its completion, so the fields' steps
 * interleave freely instead of proceeding in lock-step.  The reduction to
 * log-likelihoods is a third launch.  The memsets and the three launches are
 * captured once into a CUDA graph; each evaluation uploads the fields'
 * parameters (computed on the host exactly as for a single field) and replays
 * the graph.  Every field has its own status word, so a field whose
 * covariance is not positive definite reports -inf without stopping the
 * others.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <functional>
#include <queue>
#include <vector>

#include "../../include/exageostat_b200.h"
#include "xg_common.cuh"
#include "xg_engine.h"
#include "xg_kernels.h"

#define XG_CU(call)                                                                                                    \
    do {                                                                                                               \
        cudaError_t _e = (call);                                                                                       \
        if (_e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e));                   \
    } while (0)

struct XgBTable {
    std::vector<int> fields;
    std::vector<long long> start; /* nact + 1 */
    XgBStep dev;                   /* device view (pointers into the batch's table buffer) */
    long long blocks = 0;
};

struct XgBatch {
    int nfields = 0, ts = 0, kernel = 0, metric = 0, maxnt = 0;
    long long total_tiles = 0, total_vec = 0, total_part = 0, total_cnt = 0;
    std::vector<XgBField> F;
    XgBField *F_dev = nullptr, *F_pinned = nullptr;
    double *tiles = nullptr, *x = nullptr, *y = nullptr, *z = nullptr, *v = nullptr, *part = nullptr,
           *out = nullptr, *h_out = nullptr;
    int *status = nullptr, *h_status = nullptr;
    void *table_buf = nullptr;
    XgBTable gen;
    /* device tile scheduler: task list, counters, next-task index, abort flag */
    int4 *tasks = nullptr;
    long long ntasks = 0;
    int *cnt = nullptr;
    unsigned long long *next = nullptr;
    int *abort_flag = nullptr;
    double *dinv = nullptr; /* per scheduler CTA: ts x 32 inverted diagonal blocks */
    CUtensorMap map;
    cudaGraphExec_t graph = nullptr;
    /* gradients (allocated on the first request): per stream an inverse-factor
     * store for the largest field and contraction partials; per field a TMA
     * view of its tiles; one (i, j) table per tile count; 4 sums per field */
    static const int GS = 8;
    cudaStream_t gst[GS] = {};
    XgTileMatrix gX[GS];
    double *gpart[GS] = {};
    double *gout = nullptr, *h_gout = nullptr;
    std::vector<CUtensorMap> fmap;
    std::vector<int2 *> ij_by_nt;
};

static void xg_batch_free(XgBatch *b)
{
    if (!b) return;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    for (int s = 0; s < XgBatch::GS; ++s) {
        xg_tm_free(b->gX[s]);
        if (b->gpart[s]) cudaFree(b->gpart[s]);
        if (b->gst[s]) cudaStreamDestroy(b->gst[s]);
    }
    for (int2 *p : b->ij_by_nt)
        if (p) cudaFree(p);
    if (b->gout) cudaFree(b->gout);
    if (b->h_gout) cudaFreeHost(b->h_gout);
    void *dev[] = {b->F_dev, b->tiles, b->x, b->y, b->z, b->v, b->part, b->out, b->status, b->table_buf,
                   b->tasks, b->cnt, b->next, b->abort_flag, b->dinv};
    for (void *p : dev)
        if (p) cudaFree(p);
    if (b->F_pinned) cudaFreeHost(b->F_pinned);
    if (b->h_out) cudaFreeHost(b->h_out);
    if (b->h_status) cudaFreeHost(b->h_status);
    delete b;
}

/* builds the host side of a table from per-field CTA counts (0 = inactive) */
static void xg_table_fill(XgBTable &t, const std::vector<long long> &cnt)
{
    t.fields.clear();
    t.start.assign(1, 0);
    for (size_t f = 0; f < cnt.size(); ++f)
        if (cnt[f] > 0) {
            t.fields.push_back((int)f);
            t.start.push_back(t.start.back() + cnt[f]);
        }
    t.blocks = t.start.back();
}

/* ------------------------------------------------------------------------- */
/* task order of the device scheduler                                        */
/* ------------------------------------------------------------------------- */

/* Relative durations of the scheduler's task bodies on one SM (units of a
 * tile update, 2 ts^3 DMMA flops): a TRSM task solves the tile's ts / 32 row
 * strips one after the other; a POTRF task is latency-bound. */
#define XG_PLAN_GEMM 1.0
#define XG_PLAN_TRSM 1.05
#define XG_PLAN_POTRF 0.5

/* Bottom levels (longest path to the end of the field's DAG, the task's own
 * duration included) of every task of a tile Cholesky with nt tiles per side,
 * under the scheduler's dependencies: POTRF(k) <- the k updates of (k, k);
 * TRSM(i, k) <- POTRF(k) and the k updates of (i, k); update (i, j) <- k <-
 * TRSM(i, k), TRSM(j, k) and the update (i, j) <- k - 1. */
struct XgPlanLevels {
    int nt = 0;
    std::vector<double> p, t, g; /* p[k], t[i * nt + k], g[(i * nt + j) * nt + k] */
};

static void xg_plan_levels(int nt, XgPlanLevels &L)
{
    L.nt = nt;
    L.p.assign(nt, 0.0);
    L.t.assign((size_t)nt * nt, 0.0);
    L.g.assign((size_t)nt * nt * nt, 0.0);
    auto G = [&](int i, int j, int k) -> double & { return L.g[((size_t)i * nt + j) * nt + k]; };
    auto T = [&](int i, int k) -> double & { return L.t[(size_t)i * nt + k]; };
    for (int k = nt - 1; k >= 0; --k) {
        for (int j = k + 1; j < nt; ++j)
            for (int i = j; i < nt; ++i) {
                const double next = k + 1 < j ? G(i, j, k + 1) : (i == j ? L.p[j] : T(i, j));
                G(i, j, k) = XG_PLAN_GEMM + next;
            }
        for (int i = k + 1; i < nt; ++i) {
            double m = 0.0;
            for (int j = k + 1; j <= i; ++j) m = std::max(m, G(i, j, k));
            for (int i2 = i; i2 < nt; ++i2) m = std::max(m, G(i2, i, k));
            T(i, k) = XG_PLAN_TRSM + m;
        }
        double m = 0.0;
        for (int i = k + 1; i < nt; ++i) m = std::max(m, T(i, k));
        L.p[k] = XG_PLAN_POTRF + m;
    }
}

/* The task list of a batch for `workers` persistent CTAs that take tasks in
 * list order: a list-scheduling simulation in which every free worker starts
 * the ready task of largest bottom level (critical path first), with the
 * durations above; the list is the order in which tasks start.  A task
 * starts only after every task it waits on has finished, so the list is a
 * topological order and the device scheduler cannot deadlock on it. */
static void xg_batch_plan(const std::vector<int> &nts, int workers, std::vector<int4> &tl)
{
    struct Task {
        int f, type, i, j, k;
        double bl;
    };
    const int nf = (int)nts.size();
    std::vector<const XgPlanLevels *> lev(nf);
    std::vector<XgPlanLevels> cache;
    {
        std::vector<int> distinct(nts.begin(), nts.end());
        std::sort(distinct.begin(), distinct.end());
        distinct.erase(std::unique(distinct.begin(), distinct.end()), distinct.end());
        cache.resize(distinct.size());
        for (size_t d = 0; d < distinct.size(); ++d) xg_plan_levels(distinct[d], cache[d]);
        for (int f = 0; f < nf; ++f)
            lev[f] = &cache[std::lower_bound(distinct.begin(), distinct.end(), nts[f]) - distinct.begin()];
    }
    /* per field: update counts and TRSM completion per lower tile, POTRF completion per step */
    std::vector<long long> off(nf + 1, 0);
    for (int f = 0; f < nf; ++f) off[f + 1] = off[f] + xg_num_lower_tiles(nts[f]);
    std::vector<int> ucnt(off[nf], 0);
    std::vector<char> tdone(off[nf], 0);
    std::vector<long long> poff(nf + 1, 0);
    for (int f = 0; f < nf; ++f) poff[f + 1] = poff[f] + nts[f];
    std::vector<char> pdone(poff[nf], 0);

    std::vector<Task> tasks;
    auto cmp = [&](int a, int b) { /* max-heap on bottom level, then the earlier task */
        if (tasks[a].bl != tasks[b].bl) return tasks[a].bl < tasks[b].bl;
        return a > b;
    };
    std::priority_queue<int, std::vector<int>, decltype(cmp)> ready(cmp);
    auto push = [&](int f, int type, int i, int j, int k) {
        const XgPlanLevels &L = *lev[f];
        const int nt = L.nt;
        double bl = type == XG_TASK_POTRF ? L.p[k]
                    : type == XG_TASK_TRSM ? L.t[(size_t)i * nt + k]
                                           : L.g[((size_t)i * nt + j) * nt + k];
        tasks.push_back(Task{f, type, i, j, k, bl});
        ready.push((int)tasks.size() - 1);
    };
    for (int f = 0; f < nf; ++f) push(f, XG_TASK_POTRF, 0, 0, 0);
    typedef std::pair<double, int> Ev; /* finish time, task */
    std::priority_queue<Ev, std::vector<Ev>, std::greater<Ev>> running;
    double now = 0.0;
    int idle = workers;
    tl.clear();
    while (!ready.empty() || !running.empty()) {
        while (idle > 0 && !ready.empty()) {
            const int id = ready.top();
            ready.pop();
            const Task &t = tasks[id];
            tl.push_back(make_int4(t.type | (t.f << 2), t.i, t.j, t.k));
            const double d = t.type == XG_TASK_POTRF ? XG_PLAN_POTRF : t.type == XG_TASK_TRSM ? XG_PLAN_TRSM
                                                                                                 : XG_PLAN_GEMM;
            running.push(Ev(now + d, id));
            --idle;
        }
        if (running.empty()) break;
        /* complete the next task and release what it unblocks */
        const Ev ev = running.top();
        running.pop();
        now = ev.first;
        ++idle;
        const Task t = tasks[ev.second];
        const int f = t.f, nt = nts[f];
        auto U = [&](int i, int j) -> int & { return ucnt[off[f] + xg_tile_index(i, j, nt)]; };
        auto TD = [&](int i, int j) -> char & { return tdone[off[f] + xg_tile_index(i, j, nt)]; };
        if (t.type == XG_TASK_POTRF) {
            pdone[poff[f] + t.k] = 1;
            for (int i = t.k + 1; i < nt; ++i)
                if (U(i, t.k) == t.k) push(f, XG_TASK_TRSM, i, t.k, t.k);
        } else if (t.type == XG_TASK_TRSM) {
            const int i = t.i, k = t.k;
            TD(i, k) = 1;
            for (int j = k + 1; j <= i; ++j) /* update (i, j) <- k: A operand L_ik, B operand L_jk */
                if (TD(j, k) && U(i, j) == k) push(f, XG_TASK_GEMM, i, j, k);
            for (int i2 = i + 1; i2 < nt; ++i2) /* update (i2, i) <- k: B operand L_ik */
                if (TD(i2, k) && U(i2, i) == k) push(f, XG_TASK_GEMM, i2, i, k);
        } else {
            const int i = t.i, j = t.j, k = t.k;
            const int u = ++U(i, j);
            if (u < j) {
                if (TD(i, u) && TD(j, u)) push(f, XG_TASK_GEMM, i, j, u);
            } else if (i == j) {
                push(f, XG_TASK_POTRF, j, j, j);
            } else if (pdone[poff[f] + j]) {
                push(f, XG_TASK_TRSM, i, j, j);
            }
        }
    }
}

/* The planned task list of a batch of fields with nt[f] tiles per side, for
 * `workers` CTAs: writes 4 ints per task (type | field << 2, i, j, k) to out
 * when out is not null and returns the number of tasks.  Host-only. */
extern "C" long long exageostat_b200_batch_plan(int nfields, const int *nt, int workers, int *out)
{
    if (nfields <= 0 || !nt || workers <= 0) return 0;
    std::vector<int> nts(nt, nt + nfields);
    std::vector<int4> tl;
    xg_batch_plan(nts, workers, tl);
    if (out)
        for (size_t q = 0; q < tl.size(); ++q) {
            out[4 * q] = tl[q].x;
            out[4 * q + 1] = tl[q].y;
            out[4 * q + 2] = tl[q].z;
            out[4 * q + 3] = tl[q].w;
        }
    return (long long)tl.size();
}

extern "C" int exageostat_b200_batch_create(int nfields, const int *n, const double *x, const double *y,
                                            const double *z, int kernel, int metric, int ts, void **handle)
{
    *handle = nullptr;
    int rc = xg_context_require();
    if (rc) return rc;
    if (nfields <= 0 || !n || !x || !y || !z) return xg_fail(XG_ERR_BAD_ARGUMENT, "empty batch");
    if (kernel != 0 && kernel != 1) return xg_fail(XG_ERR_BAD_ARGUMENT, "kernel %d", kernel);
    XgBatch *b = new XgBatch();
    b->nfields = nfields;
    b->ts = ts > 0 ? xg_choose_ts(1 << 20, ts) : 256;
    b->kernel = kernel;
    b->metric = metric;
    b->F.resize(nfields);
    for (int f = 0; f < nfields; ++f) {
        if (n[f] <= 0) {
            xg_batch_free(b);
            return xg_fail(XG_ERR_BAD_ARGUMENT, "field %d has %d locations", f, n[f]);
        }
        XgBField &fd = b->F[f];
        memset(&fd, 0, sizeof fd);
        fd.N = n[f];
        fd.nt = (n[f] + b->ts - 1) / b->ts;
        fd.kernel = kernel;
        fd.tile_off = b->total_tiles;
        fd.vec_off = b->total_vec;
        fd.part_off = b->total_part;
        fd.sched_off = b->total_cnt;
        b->total_tiles += xg_num_lower_tiles(fd.nt);
        b->total_vec += (long long)fd.nt * b->ts;
        b->total_part += 2LL * fd.nt;
        b->total_cnt += fd.nt + 2 * xg_num_lower_tiles(fd.nt);
        if (fd.nt > b->maxnt) b->maxnt = fd.nt;
    }
    const size_t tile = (size_t)b->ts * b->ts;
    cudaError_t e = cudaMalloc(&b->tiles, (size_t)b->total_tiles * tile * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->x, b->total_vec * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->y, b->total_vec * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->z, b->total_vec * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->v, b->total_vec * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->part, b->total_part * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->out, 2 * (size_t)nfields * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&b->status, 2 * (size_t)nfields * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&b->F_dev, nfields * sizeof(XgBField));
    if (e == cudaSuccess) e = cudaMallocHost(&b->F_pinned, nfields * sizeof(XgBField));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_out, 2 * (size_t)nfields * sizeof(double));
    if (e == cudaSuccess) e = cudaMallocHost(&b->h_status, 2 * (size_t)nfields * sizeof(int));
    if (e != cudaSuccess) {
        xg_batch_free(b);
        return xg_fail(XG_ERR_NO_MEMORY, "batch buffers (%.2f GB of tiles): %s",
                       b->total_tiles * tile * 8.0 / 1e9, cudaGetErrorString(e));
    }
    /* locations and observations, zero padded per field */
    std::vector<double> hx(b->total_vec, 0.0), hy(b->total_vec, 0.0), hz(b->total_vec, 0.0);
    long long src = 0;
    for (int f = 0; f < nfields; ++f) {
        const XgBField &fd = b->F[f];
        memcpy(&hx[fd.vec_off], x + src, fd.N * sizeof(double));
        memcpy(&hy[fd.vec_off], y + src, fd.N * sizeof(double));
        memcpy(&hz[fd.vec_off], z + src, fd.N * sizeof(double));
        src += fd.N;
    }
    cudaMemcpy(b->x, hx.data(), b->total_vec * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(b->y, hy.data(), b->total_vec * sizeof(double), cudaMemcpyHostToDevice);
    cudaMemcpy(b->z, hz.data(), b->total_vec * sizeof(double), cudaMemcpyHostToDevice);
    /* generation table: the CTAs of every field's tiles */
    std::vector<long long> cnt(nfields);
    for (int f = 0; f < nfields; ++f) cnt[f] = xg_num_lower_tiles(b->F[f].nt) * (b->ts / 8);
    xg_table_fill(b->gen, cnt);
    /* the scheduler's task list: a critical-path-first list schedule over
     * every field's tasks for the launch's CTAs (xg_batch_plan) */
    {
        std::vector<int> nts(nfields);
        for (int f = 0; f < nfields; ++f) nts[f] = b->F[f].nt;
        std::vector<int4> tl;
        xg_batch_plan(nts, g_xg.sm_count, tl);
        b->ntasks = (long long)tl.size();
        e = cudaMalloc(&b->tasks, tl.size() * sizeof(int4));
        if (e == cudaSuccess) e = cudaMemcpy(b->tasks, tl.data(), tl.size() * sizeof(int4), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMalloc(&b->cnt, (size_t)b->total_cnt * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&b->next, sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMalloc(&b->abort_flag, sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&b->dinv, (size_t)g_xg.sm_count * b->ts * 32 * sizeof(double));
        if (e != cudaSuccess) {
            xg_batch_free(b);
            return xg_fail(XG_ERR_NO_MEMORY, "batch task list (%lld tasks): %s", (long long)tl.size(),
                           cudaGetErrorString(e));
        }
    }
    /* one device buffer for the table(s): fields (int) then starts (long long) */
    std::vector<XgBTable *> all;
    all.push_back(&b->gen);
    size_t bytes = 0;
    for (XgBTable *t : all) bytes += t->start.size() * sizeof(long long) + ((t->fields.size() * sizeof(int) + 7) & ~7ULL);
    std::vector<unsigned char> hbuf(bytes);
    e = cudaMalloc(&b->table_buf, bytes);
    if (e != cudaSuccess) {
        xg_batch_free(b);
        return xg_fail(XG_ERR_NO_MEMORY, "batch tables");
    }
    size_t off = 0;
    for (XgBTable *t : all) {
        memcpy(&hbuf[off], t->start.data(), t->start.size() * sizeof(long long));
        t->dev.blk_start = (const long long *)((unsigned char *)b->table_buf + off);
        off += t->start.size() * sizeof(long long);
        memcpy(&hbuf[off], t->fields.data(), t->fields.size() * sizeof(int));
        t->dev.fields = (const int *)((unsigned char *)b->table_buf + off);
        off += (t->fields.size() * sizeof(int) + 7) & ~7ULL;
        t->dev.nact = (int)t->fields.size();
    }
    cudaMemcpy(b->table_buf, hbuf.data(), bytes, cudaMemcpyHostToDevice);
    /* TMA view over the whole batch store */
    rc = xg_encode_tiles(&b->map, b->tiles, b->total_tiles, b->ts);
    if (rc) {
        xg_batch_free(b);
        return rc;
    }
    *handle = b;
    return XG_OK;
}

static void xg_batch_record(XgBatch *b, cudaStream_t st)
{
    XgTileArgs base{b->tiles, b->ts, 0};
    cudaMemsetAsync(b->status, 0, 2 * (size_t)b->nfields * sizeof(int), st);
    cudaMemsetAsync(b->cnt, 0, (size_t)b->total_cnt * sizeof(int), st);
    cudaMemsetAsync(b->next, 0, sizeof(unsigned long long), st);
    cudaMemsetAsync(b->abort_flag, 0, sizeof(int), st);
    cudaMemcpyAsync(b->v, b->z, b->total_vec * sizeof(double), cudaMemcpyDeviceToDevice, st);
    xg_launch_batch_gen(base, b->F_dev, b->gen.dev, b->gen.blocks, b->x, b->y, b->metric, st);
    XgSched sch;
    sch.tasks = b->tasks;
    sch.ntasks = b->ntasks;
    sch.next = b->next;
    sch.abort = b->abort_flag;
    sch.cnt = b->cnt;
    sch.dinv = b->dinv;
    const int ctas = (int)std::min<long long>(g_xg.sm_count, b->ntasks);
    xg_launch_batch_sched(b->map, base, b->F_dev, sch, ctas, b->v, b->part, b->status, st);
    xg_launch_batch_finalize(b->F_dev, b->nfields, b->part, b->out, st);
}

extern "C" int exageostat_b200_batch_loglik(void *handle, const double *theta, double *loglik)
{
    XgBatch *b = (XgBatch *)handle;
    if (!b || !theta || !loglik) return xg_fail(XG_ERR_BAD_ARGUMENT, "NULL argument");
    const int np = b->kernel == 1 ? 4 : 3;
    for (int f = 0; f < b->nfields; ++f) {
        int rc = xg_check_theta(theta + (size_t)f * np, b->kernel);
        if (rc) return xg_fail(rc, "field %d: %s", f, exageostat_last_error());
        b->F[f].p = xg_params(theta + (size_t)f * np, b->kernel);
    }
    memcpy(b->F_pinned, b->F.data(), b->nfields * sizeof(XgBField));
    cudaStream_t st = g_xg.stream;
    cudaError_t e = cudaMemcpyAsync(b->F_dev, b->F_pinned, b->nfields * sizeof(XgBField), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "batch parameters: %s", cudaGetErrorString(e));
    if (!b->graph) {
        cudaGraph_t g;
        e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            xg_batch_record(b, st);
            e = cudaStreamEndCapture(st, &g);
        }
        if (e == cudaSuccess) {
            e = cudaGraphInstantiate(&b->graph, g, 0);
            cudaGraphDestroy(g);
        }
        if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(e));
    }
    e = cudaGraphLaunch(b->graph, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_out, b->out, 2 * (size_t)b->nfields * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b->h_status, b->status, 2 * (size_t)b->nfields * sizeof(int), cudaMemcpyDeviceToHost,
                            st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return xg_fail(XG_ERR_CUDA, "batch evaluation: %s", cudaGetErrorString(e));
    int failed = 0;
    for (int f = 0; f < b->nfields; ++f) {
        const int stf = b->h_status[2 * f];
        if (stf & XG_ST_TIMEOUT) return xg_fail(XG_ERR_TIMEOUT, "field %d: a device wait timed out", f);
        if (stf) {
            loglik[f] = -INFINITY;
            ++failed;
        } else {
            loglik[f] = b->h_out[2 * f];
        }
    }
    if (failed) xg_fail(XG_ERR_NOT_SPD, "%d of %d fields are not positive definite (their loglik is -inf)", failed,
                        b->nfields);
    return XG_OK;
}

/* gradient workspace of a batch (first gradient request) */
static int xg_batch_grad_workspace(XgBatch *b)
{
    if (b->gout) return XG_OK;
    const int ts = b->ts;
    long long maxblocks = 0;
    b->ij_by_nt.assign(b->maxnt + 1, nullptr);
    for (int nt = 1; nt <= b->maxnt; ++nt) {
        const long long ntl = xg_num_lower_tiles(nt);
        std::vector<int2> h(ntl);
        for (int j = 0; j < nt; ++j)
            for (int i = j; i < nt; ++i) h[xg_tile_index(i, j, nt)] = make_int2(i, j);
        XG_CU(cudaMalloc(&b->ij_by_nt[nt], sizeof(int2) * ntl));
        XG_CU(cudaMemcpy(b->ij_by_nt[nt], h.data(), sizeof(int2) * ntl, cudaMemcpyHostToDevice));
        maxblocks = std::max(maxblocks, xg_grad_contract_blocks(ntl, ts));
    }
    for (int s = 0; s < XgBatch::GS; ++s) {
        int rc = xg_tm_alloc(b->gX[s], b->maxnt * ts, ts);
        if (rc) return rc;
        XG_CU(cudaMalloc(&b->gpart[s], 4 * (size_t)maxblocks * sizeof(double)));
        XG_CU(cudaStreamCreateWithFlags(&b->gst[s], cudaStreamNonBlocking));
    }
    b->fmap.resize(b->nfields);
    for (int f = 0; f < b->nfields; ++f) {
        const XgBField &fd = b->F[f];
        int rc = xg_encode_tiles(&b->fmap[f], b->tiles + fd.tile_off * (long long)ts * ts, xg_num_lower_tiles(fd.nt),
                                 ts);
        if (rc) return rc;
    }
    XG_CU(cudaMalloc(&b->gout, 4 * (size_t)b->nfields * sizeof(double)));
    XG_CU(cudaMallocHost(&b->h_gout, 4 * (size_t)b->nfields * sizeof(double)));
    return XG_OK;
}

/* Log-likelihoods and their gradients of every field: the batched
 * factorisation (the graph of exageostat_b200_batch_loglik), then per field,
 * round-robin over eight streams, the adjoint of the single-field path on
 * that field's tiles -- alpha = L^-T v by backward tile solves, X = L^-T,
 * Sigma^-1 = X X^T over the factor, and the fused contraction with the
 * on-the-fly dSigma/dtheta tiles.  A field that is not positive definite
 * gets loglik -inf and a NaN gradient. */
extern "C" int exageostat_b200_batch_loglik_grad(void *handle, const double *theta, double *loglik, double *grad)
{
    XgBatch *b = (XgBatch *)handle;
    if (!b || !theta || !loglik || !grad) return xg_fail(XG_ERR_BAD_ARGUMENT, "NULL argument");
    int rc = xg_batch_grad_workspace(b);
    if (rc) return rc;
    rc = exageostat_b200_batch_loglik(handle, theta, loglik);
    if (rc) return rc;
    const int ts = b->ts;
    const int np = b->kernel == 1 ? 4 : 3;
    for (int f = 0; f < b->nfields; ++f) {
        if (!std::isfinite(loglik[f])) continue;
        const XgBField &fd = b->F[f];
        const int s = f % XgBatch::GS;
        cudaStream_t st = b->gst[s];
        XgTileArgs T{b->tiles + fd.tile_off * (long long)ts * ts, ts, fd.nt};
        double *vf = b->v + fd.vec_off;
        int *stf = b->status + 2 * f;
        for (int k = fd.nt - 1; k >= 0; --k) xg_launch_trsv_lower_t_step(T, k, vf, stf, st);
        xg_launch_inverse_factor(b->gX[s].map, b->fmap[f], b->gX[s].d, T.data, fd.nt, ts, stf, st);
        xg_launch_inverse_syrk(b->gX[s].map, T.data, fd.nt, ts, stf, st);
        const double dlogcon = -(log(2.0) + xg_digamma(fd.p.nu));
        xg_launch_grad_contract(T.data, b->ij_by_nt[fd.nt], xg_num_lower_tiles(fd.nt), fd.nt, ts, b->x + fd.vec_off,
                                b->y + fd.vec_off, vf, fd.N, fd.p, b->kernel, b->metric, dlogcon, b->gpart[s],
                                b->gout + 4 * (size_t)f, st);
    }
    XG_CU(cudaGetLastError());
    for (int s = 0; s < XgBatch::GS; ++s) XG_CU(cudaStreamSynchronize(b->gst[s]));
    XG_CU(cudaMemcpy(b->h_gout, b->gout, 4 * (size_t)b->nfields * sizeof(double), cudaMemcpyDeviceToHost));
    XG_CU(cudaMemcpy(b->h_status, b->status, 2 * (size_t)b->nfields * sizeof(int), cudaMemcpyDeviceToHost));
    for (int f = 0; f < b->nfields; ++f) {
        const bool ok = std::isfinite(loglik[f]) && b->h_status[2 * f] == 0;
        if (!ok && std::isfinite(loglik[f]) && (b->h_status[2 * f] & XG_ST_TIMEOUT))
            return xg_fail(XG_ERR_TIMEOUT, "field %d: a device wait timed out", f);
        for (int i = 0; i < np; ++i) grad[(size_t)f * np + i] = ok ? b->h_gout[4 * (size_t)f + i] : NAN;
    }
    return XG_OK;
}

extern "C" int exageostat_b200_batch_destroy(void *handle)
{
    xg_batch_free((XgBatch *)handle);
    return XG_OK;
}

/* Tile size of a batch chosen by timing: the batch is built with tile sizes
 * 128, 256, 384 and 512 in turn, each timed on one evaluation at theta after
 * the one that captures its graph, and the fastest is returned in *handle
 * (*ts_out its tile size; report receives (ts, seconds) pairs, 4 at most). */
extern "C" int exageostat_b200_batch_autotune(int nfields, const int *n, const double *x, const double *y,
                                              const double *z, int kernel, int metric, const double *theta,
                                              int *ts_out, double *report, void **handle)
{
    *handle = nullptr;
    const int cands[4] = {128, 256, 384, 512};
    void *best = nullptr;
    double best_t = -1.0;
    int best_ts = 0, nrep = 0;
    std::vector<double> ll(nfields);
    for (int c = 0; c < 4; ++c) {
        void *h = nullptr;
        if (exageostat_b200_batch_create(nfields, n, x, y, z, kernel, metric, cands[c], &h)) continue;
        double sec = -1.0;
        if (!exageostat_b200_batch_loglik(h, theta, ll.data())) {
            const auto t0 = std::chrono::steady_clock::now();
            if (!exageostat_b200_batch_loglik(h, theta, ll.data()))
                sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        if (sec >= 0 && report && nrep < 4) {
            report[2 * nrep] = cands[c];
            report[2 * nrep + 1] = sec;
            ++nrep;
        }
        if (sec >= 0 && (best_t < 0 || sec < best_t)) {
            if (best) exageostat_b200_batch_destroy(best);
            best = h;
            best_t = sec;
            best_ts = cands[c];
        } else {
            exageostat_b200_batch_destroy(h);
        }
    }
    if (!best) return xg_fail(XG_ERR_CUDA, "batch autotune: no tile size could be timed");
    *handle = best;
    if (ts_out) *ts_out = best_ts;
    return XG_OK;
}

