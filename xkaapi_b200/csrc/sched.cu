// Device-side ready-queue scheduler and the three execution forms of a resolved task graph.
//
// Reference behaviour replaced (XKRT, file:line): a task becomes ready when its wait counter
// reaches 0 (include/xkrt/task/task.hpp:518-551), is queued (src/sched.cc:413-455), executed
// by a device thread that launches its kernel (src/sched.cc:249-351, :469-505), and on
// completion decrements each successor's counter, queueing those that reach 0
// (src/task.cc:160-247).
//
//  * PERSISTENT: one kernel, one CTA per resident slot. CTA thread 0 takes the next queue
//    slot (atomicAdd on head) and waits, with a time limit, for a task id to be published
//    there; the CTA runs the built-in tile body; after a fence and a barrier, warp 0 decrements
//    the successors' counters with acq_rel atomics and publishes every successor that reaches
//    zero with a release store. Every queue slot is written exactly once (a task is pushed
//    once), so the queue is a plain array of ntasks slots. Tile data written inside the kernel
//    is read back with L1-bypassing loads.
//  * PLAIN: the host launches one kernel per task in spawn order (a topological order) on one
//    stream -- the reference's one-launch-per-task device path.
//  * GRAPH: the task graph becomes a CUDA graph (one kernel node per task, one edge per
//    dependency), instantiated once and replayed.
#include "common.cuh"
#include "heat.cuh"
#include "heat_bulk.cuh"
#include "internal.h"

#include <cuda.h>

#include <cmath>
#include <mutex>
#include <new>
#include <vector>

namespace xkb {

template <bool CG>
__device__ __forceinline__ double axpby1(double a, double x, double b, double y) { return __dadd_rn(__dmul_rn(a, x), __dmul_rn(b, y)); }

template <bool CG>
__device__ __forceinline__ void axpby_team(int64_t lo, int64_t hi, double a, const double * __restrict__ x,
                                           double b, double * __restrict__ y, int64_t tid, int64_t nth)
{
    if (lo >= hi) return;
    const bool same_phase = (((uintptr_t) (x + lo)) & 15) == (((uintptr_t) (y + lo)) & 15);
    int64_t head = lo;
    if (same_phase && (((uintptr_t) (y + lo)) & 15)) head = lo + 1;
    if (!same_phase) head = hi;
    if (head > hi) head = hi;
    for (int64_t i = lo + tid; i < head; i += nth)
        y[i] = axpby1<CG>(a, CG ? __ldcg(x + i) : __ldg(x + i), b, CG ? __ldcg(y + i) : y[i]);
    const int64_t nv = (hi - head) / 2;
    const double2 * xv = (const double2 *) (x + head);
    double2 * yv = (double2 *) (y + head);
    for (int64_t v = tid; v < nv; v += nth)
    {
        const double2 xx = CG ? __ldcg(xv + v) : __ldg(xv + v);
        const double2 yy = CG ? __ldcg(yv + v) : yv[v];
        yv[v] = make_double2(axpby1<CG>(a, xx.x, b, yy.x), axpby1<CG>(a, xx.y, b, yy.y));
    }
    for (int64_t i = head + 2 * nv + tid; i < hi; i += nth)
        y[i] = axpby1<CG>(a, CG ? __ldcg(x + i) : __ldg(x + i), b, CG ? __ldcg(y + i) : y[i]);
}

constexpr int SCHED_THREADS = 256;

constexpr int SCHED_BULK_NBUF = 8;       // staged columns in flight per warp (bulk tile body)
#ifndef XKB_TILE_PF
#define XKB_TILE_PF 6                    // east columns an FP32 tile strip loads ahead into registers
#endif
#ifndef XKB_F64_VEC
#define XKB_F64_VEC 4                    // rows per lane of the FP64 tile body: one warp covers 128 rows
#endif
#ifndef XKB_F64_PF
#define XKB_F64_PF 2                     // east columns the FP64 tile strip loads ahead (32 B per lane each)
#endif
#ifndef XKB_SCHED_MINB
#define XKB_SCHED_MINB 2                 // persistent CTAs resident per SM (register budget)
#endif
constexpr int SCHED_PFD_DEFAULT = 4;     // L2 prefetch distance of heat tiles in columns (3-5 measured best)
constexpr double SCHED_TIMEOUT_MAX_S = 3600.0;   // longest device wait a caller may ask for

// A device wait limit in seconds is usable when finite, positive and at most an hour.
static inline bool timeout_ok(double s) { return std::isfinite(s) && s > 0 && s <= SCHED_TIMEOUT_MAX_S; }

// Run one task with a team of `nwarps` warps; `warp` is the warp's index in the team.
__device__ __forceinline__ void run_task_team(const xkb_task_desc_t & d, int warp, int nwarps, int pfd)
{
    switch (d.kind)
    {
        case XKB_TASK_HEAT_F64: {
            const auto & h = d.u.heat;
            const bool vok = (h.ld % 2 == 0) && (h.src % 16 == 0) && (h.dst % 16 == 0);
            heat_tile_team<double, XKB_F64_VEC, XKB_F64_PF, true>((const double *) h.src, (double *) h.dst, h.ld, h.nx, h.ny,
                                               h.x0, h.x1, h.y0, h.y1, h.c, vok, pfd, warp, nwarps);
            break;
        }
        case XKB_TASK_HEAT_F32: {
            const auto & h = d.u.heat;
            const bool vok = (h.ld % 4 == 0) && (h.src % 16 == 0) && (h.dst % 16 == 0);
            // an FP32 column is half the bytes of an FP64 one: prefetch twice as many columns ahead
            heat_tile_team<float, 4, XKB_TILE_PF, true>((const float *) h.src, (float *) h.dst, h.ld, h.nx, h.ny,
                                              h.x0, h.x1, h.y0, h.y1, h.c, vok, 2 * pfd, warp, nwarps);
            break;
        }
        case XKB_TASK_AXPBY: {
            const auto & a = d.u.axpby;
            axpby_team<true>(a.lo, a.hi, a.a, (const double *) a.x, a.b, (double *) a.y,
                             (int64_t) warp * 32 + (threadIdx.x & 31), (int64_t) nwarps * 32);
            break;
        }
        default: break;   // XKB_TASK_NOOP (first-touch / placement tasks)
    }
}

__device__ __forceinline__ int atom_add_acq_rel(int * p, int v)
{
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// A run covers `ntasks` tasks numbered w * period + t (window w, task t of the window's
// `period` descriptors). A plain graph is one window (period = ntasks); a periodic graph adds
// cross-window successors (xsucc) and a wait count for tasks of later windows (npred_next).
struct SchedArgs {
    const xkb_task_desc_t * tasks;
    uint32_t ntasks;
    uint32_t period;
    const uint32_t * succ_ptr;
    const uint32_t * succ;
    const uint32_t * xsucc_ptr;    // null for a plain graph
    const uint32_t * xsucc;
    const uint32_t * npred_first;
    const uint32_t * npred_next;
    int * wc;
    int * queue;
    unsigned * ctr;            // [0] head, [1] tail, [2] status, [3] executed
    uint64_t timeout_ns;
    int pfd;                   // L2 prefetch distance of the tile bodies, in columns
};

__global__ void sched_init_kernel(SchedArgs a)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ntasks) return;
    a.queue[t] = -1;
    const uint32_t w = t / a.period, l = t - w * a.period;
    a.wc[t] = (int) (w == 0 ? a.npred_first[l] : a.npred_next[l]);
}

__global__ void sched_seed_kernel(SchedArgs a)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.ntasks) return;
    if (*(volatile unsigned *) (a.ctr + 2) != 0) return;   // a check before the run failed: nothing becomes ready
    const uint32_t w = t / a.period, l = t - w * a.period;
    if ((w == 0 ? a.npred_first[l] : a.npred_next[l]) != 0) return;
    const unsigned pos = atomicAdd(a.ctr + 1, 1u);
    a.queue[pos] = (int) t;
}

__device__ __forceinline__ void team_sync(int id, int nthreads)
{
    if (nthreads == SCHED_THREADS) __syncthreads();
    else asm volatile("bar.sync %0, %1;" :: "r"(id), "r"(nthreads) : "memory");
}

// Each CTA holds 8 / TEAM_WARPS independent TEAMS of TEAM_WARPS warps. A team's first
// thread takes the next queue slot and waits for it; the team runs the task, fences, syncs
// on its own named barrier, and its first warp releases the successors. Teams never wait for
// one another, so while one team takes or releases a task the others keep HBM busy.
//
// BULK: heat tiles whose layout allows it run the bulk-staged body (heat_bulk.cuh): each warp
// streams its strips' columns through its own ring of shared-memory slots; other tasks run the
// register body.
// Dynamic shared memory of the BULK variant with NBUF slots per warp: the slots, then the mbarriers.
constexpr size_t bulk_smem_bytes(int nbuf) { return (size_t) (SCHED_THREADS / 32) * nbuf * (BULK_SLOT_BYTES + 8); }

template <int TEAM_WARPS, bool BULK = false, int NBUF = SCHED_BULK_NBUF>
__global__ void __launch_bounds__(SCHED_THREADS, XKB_SCHED_MINB) sched_persistent_kernel(SchedArgs a)
{
    constexpr int NTEAMS = (SCHED_THREADS / 32) / TEAM_WARPS;
    constexpr int TEAM_THREADS = TEAM_WARPS * 32;
    constexpr int NWARPS = SCHED_THREADS / 32;
    __shared__ int cur[NTEAMS];
    extern __shared__ __align__(128) unsigned char bulk_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = warp / TEAM_WARPS, twarp = warp % TEAM_WARPS;
    const int bar = 1 + team;
    unsigned executed = 0;
    BulkRing<NBUF> ring;
    if constexpr (BULK)
    {
        ring.slots = bulk_smem + (size_t) warp * NBUF * BULK_SLOT_BYTES;
        ring.bars = (uint64_t *) (bulk_smem + (size_t) NWARPS * NBUF * BULK_SLOT_BYTES) + warp * NBUF;
        bulk_ring_init(ring);
    }
    for (;;)
    {
        if (twarp == 0 && lane == 0)
        {
            int t = -1;
            const unsigned slot = atomicAdd(a.ctr + 0, 1u);
            if (slot < a.ntasks)
            {
                const uint64_t t0 = xkb_globaltimer();
                uint32_t spins = 0;
                while ((t = xkb_ld_acquire(a.queue + slot)) < 0)
                {
                    if (*(volatile unsigned *) (a.ctr + 2) != 0) { t = -2; break; }   // another team gave up
                    if ((++spins & 63) == 0 && xkb_globaltimer() - t0 > a.timeout_ns)
                    {
                        atomicCAS(a.ctr + 2, 0u, (unsigned) -XKB_ETIMEDOUT);
                        t = -2;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            cur[team] = t;
        }
        team_sync(bar, TEAM_THREADS);
        const int t = cur[team];
        if (t < 0) break;
        const uint32_t w = (uint32_t) t / a.period, l = (uint32_t) t - w * a.period;
        if constexpr (BULK)
        {
            const xkb_task_desc_t & d = a.tasks[l];
            const auto & h = d.u.heat;
            // once a wait has run out anywhere, the remaining tasks are passed over quickly
            bool done = *(volatile unsigned *) (a.ctr + 2) != 0;
            if (d.kind == XKB_TASK_HEAT_F64 && bulk_ok<double, 2>((const double *) h.src, h.ld, h.nx) && h.dst % 16 == 0)
            {
                done = true;
                if (!heat_tile_team_bulk<double, 2, NBUF>((const double *) h.src, (double *) h.dst, h.ld, h.nx, h.ny, h.x0, h.x1,
                                                          h.y0, h.y1, h.c, twarp, TEAM_WARPS, ring, xkb_globaltimer() + a.timeout_ns))
                    atomicCAS(a.ctr + 2, 0u, (unsigned) -XKB_ETIMEDOUT);
            }
            else if (d.kind == XKB_TASK_HEAT_F32 && bulk_ok<float, 4>((const float *) h.src, h.ld, h.nx) && h.dst % 16 == 0)
            {
                done = true;
                if (!heat_tile_team_bulk<float, 4, NBUF>((const float *) h.src, (float *) h.dst, h.ld, h.nx, h.ny, h.x0, h.x1,
                                                         h.y0, h.y1, h.c, twarp, TEAM_WARPS, ring, xkb_globaltimer() + a.timeout_ns))
                    atomicCAS(a.ctr + 2, 0u, (unsigned) -XKB_ETIMEDOUT);
            }
            if (!done) run_task_team(d, twarp, TEAM_WARPS, a.pfd);
        }
        else
            run_task_team(a.tasks[l], twarp, TEAM_WARPS, a.pfd);
        __threadfence();
        team_sync(bar, TEAM_THREADS);
        if (twarp == 0)
        {
            const uint32_t base = w * a.period;
            const uint32_t b = a.succ_ptr[l], e = a.succ_ptr[l + 1];
            for (uint32_t i = b + lane; i < e; i += 32)
            {
                const uint32_t s = base + a.succ[i];
                if (s >= a.ntasks) continue;                 // beyond the tail of the last window
                if (atom_add_acq_rel(a.wc + s, -1) == 1)
                {
                    const unsigned pos = atomicAdd(a.ctr + 1, 1u);
                    xkb_st_release(a.queue + pos, (int) s);
                }
            }
            if (a.xsucc_ptr)
            {
                const uint32_t xb = a.xsucc_ptr[l], xe = a.xsucc_ptr[l + 1];
                for (uint32_t i = xb + lane; i < xe; i += 32)
                {
                    const uint32_t s = base + a.period + a.xsucc[i];
                    if (s >= a.ntasks) continue;
                    if (atom_add_acq_rel(a.wc + s, -1) == 1)
                    {
                        const unsigned pos = atomicAdd(a.ctr + 1, 1u);
                        xkb_st_release(a.queue + pos, (int) s);
                    }
                }
            }
            ++executed;
        }
    }
    if (twarp == 0 && lane == 0 && executed) atomicAdd(a.ctr + 3, executed);
}

// per-task kernels (PLAIN and GRAPH forms)
__global__ void __launch_bounds__(SCHED_THREADS, 2) task_kernel(xkb_task_desc_t d, int nslabs)
{
    // blockIdx.x selects a column slab of a heat tile / a chunk of an axpby range
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        xkb_task_desc_t q = d;
        const int64_t cols = (int64_t) d.u.heat.y1 - d.u.heat.y0;
        const int64_t per = (cols + nslabs - 1) / nslabs;
        q.u.heat.y0 = (int32_t) (d.u.heat.y0 + blockIdx.x * per);
        { const int64_t e = (int64_t) q.u.heat.y0 + per; q.u.heat.y1 = (int32_t) (e < d.u.heat.y1 ? e : d.u.heat.y1); }
        if (q.u.heat.y0 >= q.u.heat.y1) return;
        if (d.kind == XKB_TASK_HEAT_F64) {
            const auto & h = q.u.heat;
            const bool vok = (h.ld % 2 == 0) && (h.src % 16 == 0) && (h.dst % 16 == 0);
            heat_tile_cta<double, 2, 4, false>((const double *) h.src, (double *) h.dst, h.ld, h.nx, h.ny, h.x0, h.x1, h.y0, h.y1, h.c, vok, 8);
        } else {
            const auto & h = q.u.heat;
            const bool vok = (h.ld % 4 == 0) && (h.src % 16 == 0) && (h.dst % 16 == 0);
            heat_tile_cta<float, 4, 4, false>((const float *) h.src, (float *) h.dst, h.ld, h.nx, h.ny, h.x0, h.x1, h.y0, h.y1, h.c, vok, 8);
        }
    }
    else if (d.kind == XKB_TASK_AXPBY)
    {
        const auto & a = d.u.axpby;
        const int64_t n = a.hi - a.lo, per = ((n + nslabs - 1) / nslabs + 1) & ~(int64_t) 1;
        const int64_t lo = a.lo + blockIdx.x * per;
        const int64_t hi = (lo + per < a.hi) ? lo + per : a.hi;
        axpby_team<false>(lo, hi, a.a, (const double *) a.x, a.b, (double *) a.y, threadIdx.x, blockDim.x);
    }
}

static int task_slabs(const xkb_task_desc_t & d)
{
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        const int64_t cols = (int64_t) d.u.heat.y1 - d.u.heat.y0;
        return (int) std::max<int64_t>(1, (cols + 31) / 32);
    }
    if (d.kind == XKB_TASK_AXPBY)
    {
        const int64_t n = d.u.axpby.hi - d.u.axpby.lo;
        return (int) std::min<int64_t>(std::max<int64_t>(1, n / 4096), 1184);
    }
    return 1;
}

template <typename T>
struct Dev {
    T * p = nullptr; size_t cap = 0;
    ~Dev() { if (p) cudaFree(p); }
    int reserve(size_t n) {
        if (n <= cap) return XKB_OK;
        if (p) { cudaFree(p); p = nullptr; cap = 0; }
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        cap = n; return XKB_OK;
    }
};

} // namespace xkb

using namespace xkb;

struct xkb_sched {
    cudaStream_t stream = nullptr;
    std::vector<xkb_task_desc_t> host_tasks;  // host copy for the per-task forms (empty: device only)
    size_t ntasks = 0;                        // descriptors set
    Dev<xkb_task_desc_t> tasks;
    Dev<int> wc, queue;
    Dev<unsigned> ctr;
    Dev<unsigned long long> wsum;             // windows run without waiting: [0] first status, [1] executed
    cudaGraphExec_t gexec = nullptr;
    cudaGraph_t graph = nullptr;
    const void * graph_key = nullptr;
    int last_form = -1;
    int grid = 0;
    int team_warps = 1;                       // one warp per 128-row tile (FP64 and FP32 bodies)
    int bulk = 0;                             // 1: bulk-staged heat tile body (measured slower; opt-in)
    int pfd = SCHED_PFD_DEFAULT;              // L2 prefetch distance in columns
    uint64_t last_total = 0;                  // tasks of the last run
    cudaEvent_t ev[2] = {nullptr, nullptr};   // around the persistent kernel of the last run
    uint64_t timeout_ns = 10ull * 1000 * 1000 * 1000;
    ~xkb_sched() {
        if (ev[0]) cudaEventDestroy(ev[0]);
        if (ev[1]) cudaEventDestroy(ev[1]);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
    }
};

static int check_tasks(const xkb_task_desc_t * t, size_t n)
{
    for (size_t i = 0; i < n; ++i)
        if (!xkb_internal_task_valid(t[i]))
        {
            const uint32_t k = t[i].kind;
            if (k == XKB_TASK_HEAT_F64 || k == XKB_TASK_HEAT_F32) return xkb_set_error(XKB_EINVAL, "sched: task %zu: bad heat tile", i);
            if (k == XKB_TASK_AXPBY) return xkb_set_error(XKB_EINVAL, "sched: task %zu: bad axpby range", i);
            return xkb_set_error(XKB_EINVAL, "sched: task %zu: unknown kind %u", i, k);
        }
    return XKB_OK;
}

extern "C" int xkb_sched_create(xkb_sched_t ** out, void * stream)
{
    if (!out) return xkb_set_error(XKB_EINVAL, "sched_create: null output");
    int dev;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    xkb_sched * S = new (std::nothrow) xkb_sched();
    if (!S) return xkb_set_error(XKB_ENOMEM, "sched_create: out of host memory");
    S->stream = (cudaStream_t) stream;
    int sms = 148, per = 2;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sched_persistent_kernel<2>, SCHED_THREADS, 0);
    // (all team variants share the register budget fixed by __launch_bounds__(256, 2))
    S->grid = sms * (per > 0 ? per : 1);
    *out = S;
    return XKB_OK;
}

extern "C" int xkb_sched_destroy(xkb_sched_t * S)
{
    if (S) { cudaStreamSynchronize(S->stream); delete S; }
    return XKB_OK;
}

extern "C" int xkb_sched_set_tasks(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks)
{
    if (!S || (ntasks && !tasks)) return xkb_set_error(XKB_EINVAL, "sched_set_tasks: bad arguments");
    int rc = check_tasks(tasks, ntasks);
    if (rc) return rc;
    S->host_tasks.assign(tasks, tasks + ntasks);
    S->ntasks = ntasks;
    if ((rc = S->tasks.reserve(ntasks ? ntasks : 1))) return rc;
    if (ntasks) XKB_CUDA_TRY(cudaMemcpyAsync(S->tasks.p, tasks, ntasks * sizeof(xkb_task_desc_t), cudaMemcpyHostToDevice, S->stream));
    XKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; }
    if (S->graph) { cudaGraphDestroy(S->graph); S->graph = nullptr; }
    S->graph_key = nullptr;
    return XKB_OK;
}

// Library-internal: the descriptors go to the device only (no host copy, so only the persistent
// forms can run them); for callers that hand over millions of descriptors for one run.
int xkb_internal_sched_set_tasks_device(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks, bool checked)
{
    if (!S || (ntasks && !tasks)) return xkb_set_error(XKB_EINVAL, "sched_set_tasks: bad arguments");
    int rc = checked ? XKB_OK : check_tasks(tasks, ntasks);
    if (rc) return rc;
    S->host_tasks.clear(); S->host_tasks.shrink_to_fit();
    S->ntasks = ntasks;
    if ((rc = S->tasks.reserve(ntasks ? ntasks : 1))) return rc;
    if (ntasks) XKB_CUDA_TRY(cudaMemcpyAsync(S->tasks.p, tasks, ntasks * sizeof(xkb_task_desc_t), cudaMemcpyHostToDevice, S->stream));
    XKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
    if (S->gexec) { cudaGraphExecDestroy(S->gexec); S->gexec = nullptr; }
    if (S->graph) { cudaGraphDestroy(S->graph); S->graph = nullptr; }
    S->graph_key = nullptr;
    return XKB_OK;
}

extern "C" int xkb_sched_set_timeout(xkb_sched_t * S, double seconds)
{
    if (!S || !timeout_ok(seconds)) return xkb_set_error(XKB_EINVAL, "sched_set_timeout: the limit must be finite, above 0 and at most 3600 s");
    S->timeout_ns = (uint64_t) (seconds * 1e9);
    return XKB_OK;
}

extern "C" int xkb_sched_set_grid(xkb_sched_t * S, int ctas)
{
    if (!S || ctas <= 0) return xkb_set_error(XKB_EINVAL, "sched_set_grid: bad arguments");
    S->grid = ctas;
    return XKB_OK;
}

extern "C" int xkb_sched_set_prefetch(xkb_sched_t * S, int columns)
{
    if (!S || columns < 0 || columns > 256) return xkb_set_error(XKB_EINVAL, "sched_set_prefetch: 0..256 columns");
    S->pfd = columns;
    return XKB_OK;
}

extern "C" int xkb_sched_set_team(xkb_sched_t * S, int warps_per_task)
{
    if (!S || (warps_per_task != 1 && warps_per_task != 2 && warps_per_task != 4 && warps_per_task != 8))
        return xkb_set_error(XKB_EINVAL, "sched_set_team: warps per task must be 1, 2, 4 or 8");
    S->team_warps = warps_per_task;
    return XKB_OK;
}

extern "C" int xkb_sched_set_staging(xkb_sched_t * S, int bulk)
{
    if (!S || bulk < 0 || bulk > 1) return xkb_set_error(XKB_EINVAL, "sched_set_staging: 0 (register body) or 1 (bulk-staged body)");
    S->bulk = bulk;
    return XKB_OK;
}

static int launch_persistent(xkb_sched * S, SchedArgs & a);

template <int TEAM, int NBUF>
static int launch_bulk_n(xkb_sched * S, SchedArgs & a)
{
    const size_t smem = bulk_smem_bytes(NBUF);
    XKB_CUDA_TRY(cudaFuncSetAttribute(sched_persistent_kernel<TEAM, true, NBUF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    sched_persistent_kernel<TEAM, true, NBUF><<<S->grid, SCHED_THREADS, smem, S->stream>>>(a);
    return XKB_OK;
}

static int launch_bulk(xkb_sched * S, SchedArgs & a)
{
    switch (S->team_warps)
    {
        case 1: return launch_bulk_n<1, SCHED_BULK_NBUF>(S, a);
        case 2: return launch_bulk_n<2, SCHED_BULK_NBUF>(S, a);
        case 4: return launch_bulk_n<4, SCHED_BULK_NBUF>(S, a);
        default: return launch_bulk_n<8, SCHED_BULK_NBUF>(S, a);
    }
}

static int run_persistent(xkb_sched * S, const xkb_task_graph_t * g)
{
    const uint32_t n = (uint32_t) g->ntasks;
    int rc;
    if ((rc = S->wc.reserve(n ? n : 1)) || (rc = S->queue.reserve(n ? n : 1)) || (rc = S->ctr.reserve(4))) return rc;
    SchedArgs a;
    a.tasks = S->tasks.p; a.ntasks = n; a.period = n ? n : 1; a.succ_ptr = g->succ_ptr; a.succ = g->succ;
    a.xsucc_ptr = nullptr; a.xsucc = nullptr; a.npred_first = g->npred; a.npred_next = g->npred;
    a.wc = S->wc.p; a.queue = S->queue.p; a.ctr = S->ctr.p; a.timeout_ns = S->timeout_ns; a.pfd = S->pfd;
    return launch_persistent(S, a);
}

static int launch_persistent(xkb_sched * S, SchedArgs & a)
{
    const uint32_t n = a.ntasks;
    XKB_CUDA_TRY(cudaMemsetAsync(S->ctr.p, 0, 4 * sizeof(unsigned), S->stream));
    if (n)
    {
        sched_init_kernel<<<(n + 255) / 256, 256, 0, S->stream>>>(a);
        sched_seed_kernel<<<(n + 255) / 256, 256, 0, S->stream>>>(a);
        if (!S->ev[0]) { XKB_CUDA_TRY(cudaEventCreate(&S->ev[0])); XKB_CUDA_TRY(cudaEventCreate(&S->ev[1])); }
        XKB_CUDA_TRY(cudaEventRecord(S->ev[0], S->stream));
        if (S->bulk)
        {
            int rc = launch_bulk(S, a);
            if (rc) return rc;
        }
        else
            switch (S->team_warps)
            {
                case 1: sched_persistent_kernel<1><<<S->grid, SCHED_THREADS, 0, S->stream>>>(a); break;
                case 2: sched_persistent_kernel<2><<<S->grid, SCHED_THREADS, 0, S->stream>>>(a); break;
                case 4: sched_persistent_kernel<4><<<S->grid, SCHED_THREADS, 0, S->stream>>>(a); break;
                default: sched_persistent_kernel<8><<<S->grid, SCHED_THREADS, 0, S->stream>>>(a); break;
            }
        XKB_CUDA_TRY(cudaEventRecord(S->ev[1], S->stream));
    }
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

static int run_plain(xkb_sched * S)
{
    for (const xkb_task_desc_t & d : S->host_tasks)
    {
        if (d.kind == XKB_TASK_NOOP) continue;
        task_kernel<<<task_slabs(d), SCHED_THREADS, 0, S->stream>>>(d, task_slabs(d));
    }
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

static int build_cuda_graph(xkb_sched * S, const xkb_task_graph_t * g)
{
    const size_t n = S->host_tasks.size();
    std::vector<uint32_t> ptr(n + 1), succ(g->nedges);
    XKB_CUDA_TRY(cudaMemcpy(ptr.data(), g->succ_ptr, (n + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    if (g->nedges) XKB_CUDA_TRY(cudaMemcpy(succ.data(), g->succ, g->nedges * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    cudaGraph_t graph;
    XKB_CUDA_TRY(cudaGraphCreate(&graph, 0));
    std::vector<cudaGraphNode_t> nodes(n);
    for (size_t i = 0; i < n; ++i)
    {
        xkb_task_desc_t d = S->host_tasks[i];
        int slabs = task_slabs(d);
        void * args[2] = {&d, &slabs};
        cudaKernelNodeParams p = {};
        p.func = (void *) task_kernel;
        p.gridDim = dim3(d.kind == XKB_TASK_NOOP ? 1 : slabs);
        p.blockDim = dim3(SCHED_THREADS);
        p.kernelParams = args;
        cudaError_t e = cudaGraphAddKernelNode(&nodes[i], graph, nullptr, 0, &p);
        if (e != cudaSuccess) { cudaGraphDestroy(graph); return xkb_set_cuda_error(e); }
    }
    std::vector<cudaGraphNode_t> from, to;
    from.reserve(g->nedges); to.reserve(g->nedges);
    for (size_t t = 0; t < n; ++t)
        for (uint32_t i = ptr[t]; i < ptr[t + 1]; ++i) { from.push_back(nodes[t]); to.push_back(nodes[succ[i]]); }
    if (!from.empty())
    {
        cudaError_t e = cudaGraphAddDependencies(graph, from.data(), to.data(), from.size());
        if (e != cudaSuccess) { cudaGraphDestroy(graph); return xkb_set_cuda_error(e); }
    }
    cudaGraphExec_t exec;
    cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(graph); return xkb_set_cuda_error(e); }
    if (S->gexec) cudaGraphExecDestroy(S->gexec);
    if (S->graph) cudaGraphDestroy(S->graph);
    S->graph = graph; S->gexec = exec; S->graph_key = g->succ;
    return XKB_OK;
}

extern "C" int xkb_sched_run(xkb_sched_t * S, const xkb_task_graph_t * g, int form)
{
    if (!S || !g) return xkb_set_error(XKB_EINVAL, "sched_run: bad arguments");
    if (g->ntasks != S->ntasks)
        return xkb_set_error(XKB_EINVAL, "sched_run: graph has %llu tasks, %zu descriptors set",
                             (unsigned long long) g->ntasks, S->ntasks);
    if (form != XKB_FORM_PERSISTENT && S->host_tasks.size() != S->ntasks)
        return xkb_set_error(XKB_EINVAL, "sched_run: the descriptors were set for the persistent form only");
    S->last_form = form;
    S->last_total = g->ntasks;
    switch (form)
    {
        case XKB_FORM_PERSISTENT: return run_persistent(S, g);
        case XKB_FORM_PLAIN: return run_plain(S);
        case XKB_FORM_GRAPH:
            if (!S->gexec || S->graph_key != g->succ) { int rc = build_cuda_graph(S, g); if (rc) return rc; }
            XKB_CUDA_TRY(cudaGraphLaunch(S->gexec, S->stream));
            return XKB_OK;
        default: return xkb_set_error(XKB_EINVAL, "sched_run: unknown form %d", form);
    }
}

extern "C" int xkb_sched_run_periodic(xkb_sched_t * S, const xkb_periodic_graph_t * g, uint32_t repeats, uint32_t tail)
{
    if (!S || !g || repeats == 0 || tail == 0 || tail > g->period)
        return xkb_set_error(XKB_EINVAL, "sched_run_periodic: bad arguments");
    if (g->period != S->ntasks)
        return xkb_set_error(XKB_EINVAL, "sched_run_periodic: period %llu but %zu descriptors set",
                             (unsigned long long) g->period, S->ntasks);
    const uint64_t total = (uint64_t) (repeats - 1) * g->period + tail;
    if (total >= (1ull << 31)) return xkb_set_error(XKB_ERANGE, "sched_run_periodic: %llu tasks in one run", (unsigned long long) total);
    int rc;
    if ((rc = S->wc.reserve(total)) || (rc = S->queue.reserve(total)) || (rc = S->ctr.reserve(4))) return rc;
    SchedArgs a;
    a.tasks = S->tasks.p; a.ntasks = (uint32_t) total; a.period = (uint32_t) g->period;
    a.succ_ptr = g->succ_ptr; a.succ = g->succ; a.xsucc_ptr = g->xsucc_ptr; a.xsucc = g->xsucc;
    a.npred_first = g->npred_first; a.npred_next = g->npred_next;
    a.wc = S->wc.p; a.queue = S->queue.p; a.ctr = S->ctr.p; a.timeout_ns = S->timeout_ns; a.pfd = S->pfd;
    S->last_form = XKB_FORM_PERSISTENT;
    S->last_total = total;
    return launch_persistent(S, a);
}

// Fold one launch's status and executed count into the windows' running totals.
__global__ void window_status_kernel(const unsigned * __restrict__ ctr, unsigned long long * sum)
{
    if (threadIdx.x != 0) return;
    if (sum[0] == 0 && ctr[2] != 0) sum[0] = ctr[2];
    sum[1] += ctr[3];
}

int xkb_internal_sched_reserve(xkb_sched_t * S, size_t ntasks)
{
    if (!S) return xkb_set_error(XKB_EINVAL, "sched_reserve: null scheduler");
    int rc;
    if ((rc = S->tasks.reserve(ntasks)) || (rc = S->wc.reserve(ntasks)) || (rc = S->queue.reserve(ntasks)) || (rc = S->ctr.reserve(4)))
        return rc;
    if (!S->wsum.p)
    {
        if ((rc = S->wsum.reserve(2))) return rc;
        XKB_CUDA_TRY(cudaMemsetAsync(S->wsum.p, 0, 2 * sizeof(unsigned long long), S->stream));
    }
    return XKB_OK;
}

int xkb_internal_sched_upload_window(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks)
{
    if (!S || (ntasks && !tasks) || ntasks >= (size_t(1) << 31)) return xkb_set_error(XKB_EINVAL, "sched_upload_window: bad arguments");
    int rc;
    if (ntasks > S->tasks.cap || ntasks > S->wc.cap || ntasks > S->queue.cap)
    {
        // earlier windows may still be reading these buffers
        XKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
        const size_t c = ntasks + ntasks / 2;
        if ((rc = S->tasks.reserve(c)) || (rc = S->wc.reserve(c)) || (rc = S->queue.reserve(c))) return rc;
    }
    if (ntasks) XKB_CUDA_TRY(cudaMemcpyAsync(S->tasks.p, tasks, ntasks * sizeof(xkb_task_desc_t), cudaMemcpyHostToDevice, S->stream));
    S->host_tasks.clear();
    S->ntasks = ntasks;
    S->graph_key = nullptr;
    return XKB_OK;
}

int xkb_internal_sched_launch_window(xkb_sched_t * S, const xkb_task_graph_t * g)
{
    if (!S || !g || g->ntasks != S->ntasks) return xkb_set_error(XKB_EINVAL, "sched_launch_window: the graph and the uploaded window differ");
    int rc;
    if (!S->wsum.p)
    {
        if ((rc = S->wsum.reserve(2))) return rc;
        XKB_CUDA_TRY(cudaMemsetAsync(S->wsum.p, 0, 2 * sizeof(unsigned long long), S->stream));
    }
    const size_t ntasks = S->ntasks;
    if (ntasks == 0) return XKB_OK;
    if ((rc = S->ctr.reserve(4))) return rc;
    SchedArgs a;
    a.tasks = S->tasks.p; a.ntasks = (uint32_t) ntasks; a.period = (uint32_t) ntasks; a.succ_ptr = g->succ_ptr; a.succ = g->succ;
    a.xsucc_ptr = nullptr; a.xsucc = nullptr; a.npred_first = g->npred; a.npred_next = g->npred;
    a.wc = S->wc.p; a.queue = S->queue.p; a.ctr = S->ctr.p; a.timeout_ns = S->timeout_ns; a.pfd = S->pfd;
    if ((rc = launch_persistent(S, a))) return rc;
    window_status_kernel<<<1, 32, 0, S->stream>>>(S->ctr.p, S->wsum.p);
    XKB_CUDA_TRY(cudaGetLastError());
    S->last_form = XKB_FORM_PERSISTENT;
    S->last_total = ntasks;
    return XKB_OK;
}

int xkb_internal_sched_run_window(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks, const xkb_task_graph_t * g)
{
    if (!S || (ntasks && !tasks) || !g || g->ntasks != ntasks || ntasks >= (size_t(1) << 31))
        return xkb_set_error(XKB_EINVAL, "sched_run_window: bad arguments");
    int rc = xkb_internal_sched_upload_window(S, tasks, ntasks);
    return rc ? rc : xkb_internal_sched_launch_window(S, g);
}

int xkb_internal_sched_windows_wait(xkb_sched_t * S, uint64_t * executed)
{
    if (!S) return xkb_set_error(XKB_EINVAL, "sched_windows_wait: null scheduler");
    XKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
    unsigned long long sum[2] = {0, 0};
    if (S->wsum.p)
    {
        XKB_CUDA_TRY(cudaMemcpy(sum, S->wsum.p, sizeof(sum), cudaMemcpyDeviceToHost));
        XKB_CUDA_TRY(cudaMemset(S->wsum.p, 0, sizeof(sum)));
    }
    if (executed) *executed = sum[1];
    if (sum[0] != 0) return xkb_set_error(-(int) sum[0], "sched: a device wait ran out of time in a window run");
    return XKB_OK;
}

extern "C" int xkb_sched_wait(xkb_sched_t * S, uint64_t * executed)
{
    if (!S) return xkb_set_error(XKB_EINVAL, "sched_wait: null scheduler");
    XKB_CUDA_TRY(cudaStreamSynchronize(S->stream));
    unsigned ctr[4] = {0, 0, 0, (unsigned) S->last_total};
    if (S->ctr.p && S->last_form == XKB_FORM_PERSISTENT) XKB_CUDA_TRY(cudaMemcpy(ctr, S->ctr.p, sizeof(ctr), cudaMemcpyDeviceToHost));
    if (executed) *executed = ctr[3];
    if (ctr[2] != 0)
        return xkb_set_error(-(int) ctr[2], "sched: a device wait ran out of time (%u of %llu tasks were made ready)", ctr[1], (unsigned long long) S->last_total);
    return XKB_OK;
}

extern "C" int xkb_sched_kernel_ms(xkb_sched_t * S, double * ms)
{
    if (!S || !ms) return xkb_set_error(XKB_EINVAL, "sched_kernel_ms: bad arguments");
    *ms = 0;
    if (S->last_form != XKB_FORM_PERSISTENT || !S->ev[0]) return XKB_OK;
    float f = 0;
    XKB_CUDA_TRY(cudaEventSynchronize(S->ev[1]));
    XKB_CUDA_TRY(cudaEventElapsedTime(&f, S->ev[0], S->ev[1]));
    *ms = f;
    return XKB_OK;
}

// ------------------------------------------------------------------------------------------
// Persistent run without any allocation.
//
// Some callers cannot allocate device memory when they run a graph: a task runtime that has
// reserved most of the GPU's memory for its own allocator at start-up (XKRT reserves 90 % of
// HBM for its device memory areas), or a serving loop whose device memory is already carved
// into fixed pools, gets a failed or competing cudaMalloc; and cudaMalloc/cudaFree can
// synchronise the device in the middle of a latency-critical loop. This entry point keeps the
// scheduler's working set -- wait counters, queue slots and four counters -- in the file-scope
// array below instead, sized for at most XKB_NOALLOC_MAX_TASKS tasks (8 MiB + 256 B held by
// every GPU that loads the library, until the process exits).
static __device__ __align__(256) int g_sched_noalloc_scratch[2 * XKB_NOALLOC_MAX_TASKS + 64];   // + counters

// Counters of a no-allocation run, after the wait counters and queue: [0] head, [1] tail,
// [2] status, [3] executed, [4] the lowest task index whose descriptor failed the check.
constexpr int NOALLOC_CTRS = 8;

// Every descriptor of a no-allocation run is checked on the device with the host checks of
// xkb_sched_set_tasks before anything runs: a bad one sets the status to XKB_EINVAL, records
// the lowest such index, and the seed kernel then makes no task ready, so no tile is touched.
__global__ void noalloc_check_kernel(const xkb_task_desc_t * __restrict__ tasks, uint32_t n, unsigned * ctr)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    if (!xkb_internal_task_valid(tasks[t]))
    {
        atomicCAS(ctr + 2, 0u, (unsigned) -XKB_EINVAL);
        atomicMin(ctr + 4, t);
    }
}

// Device address of the scratch array in the current context. In host code the array's name
// only stands for it; its device address is looked up with the device current, on the first
// call made in each CUDA context (a context destroyed by cudaDeviceReset and made again gets a
// fresh lookup). The same set-up loads the kernels the run launches, so that with lazy module
// loading a later call needs no module memory either.
struct NoallocSlot { CUcontext ctx = nullptr; int * ptr = nullptr; };

static int noalloc_scratch(int ** out)
{
    static std::mutex mu;
    static NoallocSlot slots[256];
    static CUresult (*ctx_current)(CUcontext *) = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        void * f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            ctx_current = (CUresult (*)(CUcontext *)) f;
        else
            cudaGetLastError();
    });
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    if (dev < 0 || dev >= 256) return xkb_set_error(XKB_ENODEV, "sched_run_noalloc: device %d out of range", dev);
    e = cudaSetDevice(dev);                     // makes the device's primary context current (CUDA 12)
    if (e != cudaSuccess) return xkb_set_cuda_error(e);
    CUcontext ctx = nullptr;
    if (!ctx_current || ctx_current(&ctx) != CUDA_SUCCESS || !ctx)
        return xkb_set_error(XKB_ENODEV, "sched_run_noalloc: no current CUDA context on device %d", dev);
    std::lock_guard<std::mutex> lock(mu);
    NoallocSlot & sl = slots[dev];
    if (sl.ctx != ctx || !sl.ptr)
    {
        void * p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sched_noalloc_scratch);
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        cudaFuncAttributes fa;
        const void * kernels[] = {(const void *) noalloc_check_kernel, (const void *) sched_init_kernel,
                                  (const void *) sched_seed_kernel, (const void *) sched_persistent_kernel<1>,
                                  (const void *) sched_persistent_kernel<2>, (const void *) sched_persistent_kernel<4>,
                                  (const void *) sched_persistent_kernel<8>};
        for (const void * k : kernels)
            if ((e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess) return xkb_set_cuda_error(e);
        sl.ctx = ctx;
        sl.ptr = (int *) p;
    }
    *out = sl.ptr;
    return XKB_OK;
}

extern "C" int xkb_sched_run_noalloc(const xkb_task_desc_t * tasks, const xkb_task_graph_t * graph, int warps_per_task,
                                     double timeout_s, void * stream, uint64_t * executed)
{
    if (!graph || (graph->ntasks && (!tasks || !graph->succ_ptr || !graph->npred)))
        return xkb_set_error(XKB_EINVAL, "sched_run_noalloc: bad arguments");
    if (!timeout_ok(timeout_s))
        return xkb_set_error(XKB_EINVAL, "sched_run_noalloc: the time limit must be finite, above 0 and at most 3600 s");
    if (warps_per_task != 1 && warps_per_task != 2 && warps_per_task != 4 && warps_per_task != 8)
        return xkb_set_error(XKB_EINVAL, "sched_run_noalloc: warps per task must be 1, 2, 4 or 8");
    if (graph->ntasks > XKB_NOALLOC_MAX_TASKS)
        return xkb_set_error(XKB_ERANGE, "sched_run_noalloc: %llu tasks exceed the fixed capacity of %u tasks",
                             (unsigned long long) graph->ntasks, (unsigned) XKB_NOALLOC_MAX_TASKS);
    int * scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    cudaStream_t st = xkb_stream(stream);
    const uint32_t n = (uint32_t) graph->ntasks;
    SchedArgs a;
    a.tasks = tasks; a.ntasks = n; a.period = n ? n : 1; a.succ_ptr = graph->succ_ptr; a.succ = graph->succ;
    a.xsucc_ptr = nullptr; a.xsucc = nullptr; a.npred_first = graph->npred; a.npred_next = graph->npred;
    a.wc = scratch; a.queue = scratch + XKB_NOALLOC_MAX_TASKS;
    a.ctr = (unsigned *) (scratch + 2 * XKB_NOALLOC_MAX_TASKS);
    a.timeout_ns = (uint64_t) (timeout_s * 1e9);
    a.pfd = SCHED_PFD_DEFAULT;
    // the array keeps the previous call's contents: the counters are cleared here (the lowest bad
    // index to all ones), and the init kernel rewrites every wait counter and queue slot this run uses
    XKB_CUDA_TRY(cudaMemsetAsync(a.ctr, 0, 4 * sizeof(unsigned), st));
    XKB_CUDA_TRY(cudaMemsetAsync(a.ctr + 4, 0xff, (NOALLOC_CTRS - 4) * sizeof(unsigned), st));
    if (n)
    {
        int dev = 0, sms = 148, per = 2;
        XKB_CUDA_TRY(cudaGetDevice(&dev));
        XKB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        XKB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, sched_persistent_kernel<2>, SCHED_THREADS, 0));
        const unsigned grid = (unsigned) (sms * (per > 0 ? per : 1));
        noalloc_check_kernel<<<(n + 255) / 256, 256, 0, st>>>(tasks, n, a.ctr);
        sched_init_kernel<<<(n + 255) / 256, 256, 0, st>>>(a);
        sched_seed_kernel<<<(n + 255) / 256, 256, 0, st>>>(a);
        switch (warps_per_task)
        {
            case 1: sched_persistent_kernel<1><<<grid, SCHED_THREADS, 0, st>>>(a); break;
            case 2: sched_persistent_kernel<2><<<grid, SCHED_THREADS, 0, st>>>(a); break;
            case 4: sched_persistent_kernel<4><<<grid, SCHED_THREADS, 0, st>>>(a); break;
            default: sched_persistent_kernel<8><<<grid, SCHED_THREADS, 0, st>>>(a); break;
        }
        XKB_CUDA_TRY(cudaGetLastError());
    }
    unsigned ctr[NOALLOC_CTRS] = {};
    XKB_CUDA_TRY(cudaMemcpyAsync(ctr, a.ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    XKB_CUDA_TRY(cudaStreamSynchronize(st));
    if (executed) *executed = ctr[3];
    if (ctr[2] == (unsigned) -XKB_EINVAL)
        return xkb_set_error(XKB_EINVAL, "sched_run_noalloc: task %u: bad descriptor (unknown kind, bad heat tile or axpby range); nothing ran", ctr[4]);
    if (ctr[2] != 0)
        return xkb_set_error(-(int) ctr[2], "sched_run_noalloc: a device wait ran out of time (%u of %u tasks were made ready)", ctr[1], n);
    return XKB_OK;
}

// ------------------------------------------------------------------------------------------
// Device-resident serving loop: ONE persistent kernel runs the tile tasks of every admitted
// request. The host admits a request by writing its slot record (descriptors, periodic graph,
// counter and queue arrays, the grid to duplicate) and then the slot's state word; any idle team
// of the kernel then takes the slot's set-up chunks (wait counters, queue slots, second grid),
// the team that finishes the last chunk publishes the request's first ready tasks, and from then
// on teams take ready tasks from whichever slot has some -- a small request does not hold SMs it
// cannot use, and requests admitted while others run share the device at once. The team that
// executes a request's last task marks the slot done and reports the admission number to mapped
// host memory; the host copies the result out. Teams stop when the host has said no request will
// come and every slot is idle or done, on an error, or at the time limit; every wait is bounded.

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned * p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned * p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void srv_publish(const XkbSrvSlot & S, XkbSrvCtl * c, uint32_t t)
{
    const unsigned pos = atomicAdd(&c->tail, 1u);
    xkb_st_release(S.queue + pos, (int) t);
}

template <int TEAM_WARPS>
__global__ void __launch_bounds__(SCHED_THREADS, XKB_SCHED_MINB) server_kernel(XkbSrvArgs a)
{
    constexpr int NTEAMS = (SCHED_THREADS / 32) / TEAM_WARPS;
    constexpr int TEAM_THREADS = TEAM_WARPS * 32;
    __shared__ int job_kind[NTEAMS];           // 0 stop, 1 task, 2 set-up chunk, -1 nothing yet
    __shared__ int job_slot[NTEAMS];
    __shared__ int job_idx[NTEAMS];            // task id, or chunk index
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int team = warp / TEAM_WARPS, twarp = warp % TEAM_WARPS;
    const int bar = 1 + team, tthread = twarp * 32 + lane;
    const int gteam = blockIdx.x * NTEAMS + team;
    unsigned executed = 0;
    uint32_t nap = 32;
    const uint64_t t_start = xkb_globaltimer();
    for (;;)
    {
        if (tthread == 0)
        {
            int kind = -1, slot = -1, idx = -1;
            if (*(volatile unsigned *) (a.status + 2) >= 2) kind = 0;     // the host gave up: stop now
            for (int k = 0; k < a.nslots && kind < 0; ++k)
            {
                const int sl = (gteam + k) % a.nslots;
                XkbSrvCtl * c = a.ctl + sl;
                const unsigned st = ld_acquire_u32(&c->state);
                if (st == 1)
                {
                    if (*(volatile unsigned *) &c->init_next < a.slots[sl].nchunks)
                    {
                        const unsigned ch = atomicAdd(&c->init_next, 1u);
                        if (ch < a.slots[sl].nchunks) { kind = 2; slot = sl; idx = (int) ch; }
                    }
                }
                else if (st == 2 && *(volatile unsigned *) &c->head < *(volatile unsigned *) &c->tail)
                {
                    // claim the next queue position with one atomicAdd (a compare-and-swap loop on
                    // `head` serialises the teams on it); the position may be published a little
                    // later, which the wait below covers. The claim counts in `claimers` while the
                    // state is re-checked, so the team ending the request can tell when no claim
                    // on this request's counters is left.
                    atomicAdd(&c->claimers, 1u);
                    __threadfence();
                    unsigned h = 0;
                    if (ld_acquire_u32(&c->state) == 2)
                    {
                        h = atomicAdd(&c->head, 1u);
                        if (h < a.slots[sl].ntasks) { kind = 1; slot = sl; }
                    }
                    atomicSub(&c->claimers, 1u);
                    if (kind == 1)
                    {
                        // the id at that position was published (tail counts it) or is about to be
                        const int * q = a.slots[sl].queue + h;
                        const uint64_t t0 = xkb_globaltimer();
                        uint32_t spins = 0;
                        int t;
                        while ((t = xkb_ld_acquire(q)) < 0)
                        {
                            if ((++spins & 63) == 0 && xkb_globaltimer() - t0 > a.timeout_ns)
                            {
                                atomicCAS(a.status, 0u, (unsigned) -XKB_ETIMEDOUT);
                                break;
                            }
                        }
                        if (t < 0) kind = 0; else idx = t;
                    }
                }
            }
            if (kind < 0)
            {
                if (*(volatile unsigned *) a.status != 0) kind = 0;
                else if (xkb_globaltimer() - t_start > a.run_ns) { atomicCAS(a.status, 0u, (unsigned) -XKB_ETIMEDOUT); kind = 0; }
                else if (*(volatile unsigned *) (a.status + 2))
                {
                    bool busy = false;
                    for (int sl = 0; sl < a.nslots && !busy; ++sl)
                    {
                        const unsigned st = ld_acquire_u32(&a.ctl[sl].state);
                        busy = st == 1 || st == 2;
                    }
                    if (!busy) kind = 0;
                }
                if (kind < 0) { __nanosleep(nap); if (nap < 8192) nap *= 2; }
            }
            else nap = 32;
            job_kind[team] = kind; job_slot[team] = slot; job_idx[team] = idx;
        }
        team_sync(bar, TEAM_THREADS);
        const int kind = job_kind[team], sl = job_slot[team], idx = job_idx[team];
        if (kind == 0) break;
        if (kind == 2)
        {
            // set-up chunk: wait counters and empty queue slots of its tasks, and its share of the
            // second grid (a copy of the first, which the host copied in)
            const XkbSrvSlot & S = a.slots[sl];
            const uint32_t t0 = (uint32_t) idx * XKB_SRV_CHUNK, t1 = min(S.ntasks, t0 + XKB_SRV_CHUNK);
            for (uint32_t t = t0 + tthread; t < t1; t += TEAM_THREADS)
            {
                S.queue[t] = -1;
                const uint32_t w = t / S.period, l = t - w * S.period;
                S.wc[t] = (int) (w == 0 ? S.npred_first[l] : S.npred_next[l]);
            }
            const uint64_t per = ((S.copy_bytes + S.nchunks - 1) / S.nchunks + 15) & ~(uint64_t) 15;
            const uint64_t b0 = min(S.copy_bytes, (uint64_t) idx * per), b1 = min(S.copy_bytes, b0 + per);
            const uint4 * src = (const uint4 *) (S.copy_src + b0);
            uint4 * dst = (uint4 *) (S.copy_dst + b0);
            const uint64_t nv = (b1 - b0) / 16;
            uint64_t k = tthread;
            for (; k + 3 * TEAM_THREADS < nv; k += 4 * TEAM_THREADS)     // four 16-byte loads in flight per lane
            {
                const uint4 v0 = __ldcg(src + k), v1 = __ldcg(src + k + TEAM_THREADS), v2 = __ldcg(src + k + 2 * TEAM_THREADS),
                            v3 = __ldcg(src + k + 3 * TEAM_THREADS);
                dst[k] = v0; dst[k + TEAM_THREADS] = v1; dst[k + 2 * TEAM_THREADS] = v2; dst[k + 3 * TEAM_THREADS] = v3;
            }
            for (; k < nv; k += TEAM_THREADS) dst[k] = __ldcg(src + k);
            for (uint64_t r = ((b1 - b0) & ~(uint64_t) 15) + tthread; r < b1 - b0; r += TEAM_THREADS)
                S.copy_dst[b0 + r] = S.copy_src[b0 + r];
            __threadfence();
            team_sync(bar, TEAM_THREADS);
            if (tthread == 0)
            {
                XkbSrvCtl * c = a.ctl + sl;
                if (atomicAdd(&c->init_done, 1u) + 1 == S.nchunks)
                {
                    // every chunk is done: publish the tasks with no predecessor, then run
                    for (uint32_t l = 0; l < S.period && l < S.ntasks; ++l)
                        if (S.npred_first[l] == 0) srv_publish(S, c, l);
                    if (S.seed_later)
                        for (uint32_t t = S.period; t < S.ntasks; ++t)
                            if (S.npred_next[t % S.period] == 0) srv_publish(S, c, t);
                    st_release_u32(&c->state, 2u);
                }
            }
        }
        else if (kind == 1)
        {
            const XkbSrvSlot & S = a.slots[sl];
            const uint32_t t = (uint32_t) idx, w = t / S.period, l = t - w * S.period;
            run_task_team(S.tasks[l], twarp, TEAM_WARPS, S.pfd);
            __threadfence();
            team_sync(bar, TEAM_THREADS);
            if (twarp == 0)
            {
                XkbSrvCtl * c = a.ctl + sl;
                const uint32_t base = w * S.period;
                for (uint32_t i = S.succ_ptr[l] + lane; i < S.succ_ptr[l + 1]; i += 32)
                {
                    const uint32_t u = base + S.succ[i];
                    if (u < S.ntasks && atom_add_acq_rel(S.wc + u, -1) == 1) srv_publish(S, c, u);
                }
                if (S.xsucc_ptr)
                    for (uint32_t i = S.xsucc_ptr[l] + lane; i < S.xsucc_ptr[l + 1]; i += 32)
                    {
                        const uint32_t u = base + S.period + S.xsucc[i];
                        if (u < S.ntasks && atom_add_acq_rel(S.wc + u, -1) == 1) srv_publish(S, c, u);
                    }
                __syncwarp();
                if (lane == 0)
                {
                    ++executed;
                    if (atomicAdd(&c->executed, 1u) + 1 == S.ntasks)
                    {
                        st_release_u32(&c->state, 3u);
                        __threadfence();
                        // teams that saw state 2 before the store above claim past the last task
                        // and leave; wait (bounded) until none is between its check and its claim
                        const uint64_t tw = xkb_globaltimer();
                        uint32_t spins = 0;
                        while (*(volatile unsigned *) &c->claimers != 0)
                            if ((++spins & 63) == 0 && xkb_globaltimer() - tw > a.timeout_ns)
                            {
                                atomicCAS(a.status, 0u, (unsigned) -XKB_ETIMEDOUT);
                                break;
                            }
                        __threadfence_system();
                        a.host_done[sl] = S.gen;
                    }
                }
            }
        }
        team_sync(bar, TEAM_THREADS);           // job_* are rewritten only after every thread read them
    }
    if (tthread == 0 && executed) atomicAdd(a.status + 1, executed);
}

int xkb_internal_server_launch(const XkbSrvArgs & a, int grid, int warps_per_task, cudaStream_t stream)
{
    switch (warps_per_task)
    {
        case 1: server_kernel<1><<<grid, SCHED_THREADS, 0, stream>>>(a); break;
        case 2: server_kernel<2><<<grid, SCHED_THREADS, 0, stream>>>(a); break;
        case 4: server_kernel<4><<<grid, SCHED_THREADS, 0, stream>>>(a); break;
        case 8: server_kernel<8><<<grid, SCHED_THREADS, 0, stream>>>(a); break;
        default: return xkb_set_error(XKB_EINVAL, "server: warps per task must be 1, 2, 4 or 8");
    }
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}

int xkb_internal_launch_task(const xkb_task_desc_t * d, cudaStream_t stream)
{
    if (d->kind == XKB_TASK_NOOP) return XKB_OK;
    const int slabs = task_slabs(*d);
    task_kernel<<<slabs, SCHED_THREADS, 0, stream>>>(*d, slabs);
    XKB_CUDA_TRY(cudaGetLastError());
    return XKB_OK;
}
