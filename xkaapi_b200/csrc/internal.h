// Library-internal entry points shared between translation units (not exported).
#pragma once
#include <cuda_runtime.h>

#include <cstdlib>
#include <thread>

#include "../../include/xkrt_b200.h"

// Launch one task descriptor as its own kernel (the plain per-task form) on `stream`.
int xkb_internal_launch_task(const xkb_task_desc_t * d, cudaStream_t stream);
// xkb_plan_execute with host cuts (sorted addresses): no two copies whose host bytes lie on
// different sides of a cut are merged into one (each copy given must lie between two cuts).
// Host copies issued by the plan executor so far, after coalescing (traces).
uint64_t xkb_internal_issued_host_copies();
int xkb_internal_plan_execute_cut(const xkb_copy_t * copies, size_t n, void * const * alloc_ptrs, size_t nallocs,
                                  cudaStream_t stream, const uint64_t * cuts, size_t ncuts);

// Set a scheduler's descriptors on the device only (persistent forms only; no host copy).
// checked: the caller validated every descriptor with xkb_internal_task_valid.
int xkb_internal_sched_set_tasks_device(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks, bool checked);

#ifdef __CUDACC__
#define XKB_HD __host__ __device__
#else
#define XKB_HD
#endif

// The descriptor checks of xkb_sched_set_tasks: a known kind with a well-formed tile or range.
// (Heat tile bodies clip their tile to the grid's interior, so a tile beyond nx/ny is harmless
// once ld >= nx.) Also evaluated on the device by xkb_sched_run_noalloc.
static inline XKB_HD bool xkb_internal_task_valid(const xkb_task_desc_t & d)
{
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        const auto & h = d.u.heat;
        return h.src && h.dst && h.src != h.dst && h.ld >= h.nx && h.nx >= 0 && h.ny >= 0 && h.x0 <= h.x1 && h.y0 <= h.y1;
    }
    if (d.kind == XKB_TASK_AXPBY)
    {
        const auto & a = d.u.axpby;
        return a.lo >= 0 && a.lo <= a.hi && (a.hi == a.lo || (a.x && a.y));
    }
    return d.kind == XKB_TASK_NOOP;
}

// Host threads for the parallel passes of background work (resolution, coherency, descriptor
// translation): XKB_HELPERS, else the hardware threads minus four (the spawning thread, the
// worker and the page-fault helpers keep theirs), between 1 and 16.
static inline unsigned xkb_internal_helpers()
{
    if (const char * e = getenv("XKB_HELPERS")) { const int v = atoi(e); if (v > 0) return v < 64 ? (unsigned) v : 64u; }
    const unsigned hw = std::thread::hardware_concurrency();
    return hw > 5 ? (hw - 4 < 16 ? hw - 4 : 16) : 1;
}

// Reset a resolver to no tasks, keeping its device buffers for the next graph.
int xkb_internal_resolver_reset(xkb_resolver_t * R);

// A point of a resolver's edge store: the tasks added so far and where the next unique edge goes.
typedef struct xkb_edge_mark_t { size_t seg, off; uint32_t ntasks; } xkb_edge_mark_t;
int xkb_internal_resolver_edge_mark(xkb_resolver_t * R, xkb_edge_mark_t * m);
// Reserve the working memory of a batch of about nops ops up front.
int xkb_internal_resolver_prepare(xkb_resolver_t * R, size_t nops);
// Reserve the device buffers of runs of up to ntasks tasks up front.
int xkb_internal_sched_reserve(xkb_sched_t * S, size_t ntasks);
// Unique edges stored so far (no graph build).
size_t xkb_internal_resolver_nedges(const xkb_resolver_t * R);
// The window of the graph from the mark's first task to the last task added: successor CSR of
// tasks [m->ntasks, ntasks) renumbered from 0, with the edges stored since the mark whose both
// ends lie in the window (every edge into a task is stored by the batch that added the task, so
// the window keeps all edges among its tasks and drops those from earlier tasks). Device buffers
// owned by the resolver, valid until the next window (in stream order) or reset.
int xkb_internal_resolver_window_graph(xkb_resolver_t * R, const xkb_edge_mark_t * m, xkb_task_graph_t * g);

// Run tasks as one persistent launch on the scheduler's stream without waiting for it: the
// descriptors are copied in stream order (host memory may be pageable), the launch's status and
// executed count are added to the scheduler's running totals, read and cleared by
// xkb_internal_sched_windows_wait.
int xkb_internal_sched_run_window(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks, const xkb_task_graph_t * g);
// The two halves of a window run: the descriptors' copy (queued now, so that it can go ahead of
// the window's graph), then the launch on the graph of the same ntasks tasks.
int xkb_internal_sched_upload_window(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks);
int xkb_internal_sched_launch_window(xkb_sched_t * S, const xkb_task_graph_t * g);
int xkb_internal_sched_windows_wait(xkb_sched_t * S, uint64_t * executed);

// The heat update of the cells [i0, i0 + w) x [j0, j0 + h) of an nx x ny grid (interior cells
// only) on per-access replicas: src and dst point at cell (i0, j0) of theirs, each with its own
// leading dimension (xkb_diffusion_views with an explicit box).
int xkb_internal_diffusion_box(int dtype, cudaStream_t stream, const void * src, int64_t ld_src, void * dst, int64_t ld_dst,
                               int64_t i0, int64_t j0, int64_t w, int64_t h, int64_t nx, int64_t ny, double c);

// ---- device-resident serving loop (one persistent kernel for every admitted request) --------
// One admitted request, in device memory. The host writes it, then the slot's counters, then the
// slot's state word (three copies in stream order), so a team that sees the state sees the rest.
struct XkbSrvSlot {
    const xkb_task_desc_t * tasks;       // the periodic window's `period` descriptors
    const uint32_t * succ_ptr, * succ, * xsucc_ptr, * xsucc, * npred_first, * npred_next;
    int * wc;                            // ntasks wait counters
    int * queue;                         // ntasks ready-queue slots
    const uint8_t * copy_src;            // the grid the host copied in ...
    uint8_t * copy_dst;                  //   ... duplicated here by the set-up chunks (second grid)
    uint64_t copy_bytes;
    uint32_t period, ntasks;
    uint32_t nchunks;                    // set-up chunks (wait counters, queue slots, grid copy)
    uint32_t gen;                        // admission number, reported back when the request ends
    uint32_t seed_later;                 // 1: some task of a later window has no predecessor
    int32_t pfd;
};
// The slot's counters (device memory): state 0 idle, 1 admitted (set-up pending), 2 running,
// 3 done; set-up chunks claimed / finished; ready-queue head and tail; tasks executed.
// claimers: teams between their check that the slot runs (state 2) and their claim on `head`;
// the team that ends the request waits for none to be left before the host may reuse the slot.
struct XkbSrvCtl { unsigned state, init_next, init_done, head, tail, executed, claimers, pad; };
struct XkbSrvArgs {
    XkbSrvSlot * slots;
    XkbSrvCtl * ctl;
    int nslots;
    volatile unsigned * host_done;       // mapped host memory: gen of the last request each slot ended
    unsigned * status;                   // [0] first error (XKB_ETIMEDOUT), [1] tasks executed,
                                         // [2] set by the host: 1 once no request will come,
                                         //     2 to stop at once (the host gave up)
    uint64_t run_ns;                     // how long a team may run before it gives up
    uint64_t timeout_ns;                 // longest wait for one published queue slot
};
// Tasks per set-up chunk of a served request, and at most this many bytes of its grid copy.
constexpr uint32_t XKB_SRV_CHUNK = 16384;
constexpr uint64_t XKB_SRV_COPY_CHUNK = uint64_t(256) << 10;
// Launch the serving kernel (grid CTAs of 256 threads, warps_per_task 1, 2, 4 or 8).
int xkb_internal_server_launch(const XkbSrvArgs & a, int grid, int warps_per_task, cudaStream_t stream);

