/* libxkb200 -- C ABI of the B200 (sm_100a) implementation of XKRT's dataflow hot path.
 *
 * Every entry point takes plain pointers and sizes; device pointers are CUDA global
 * memory of the current device, `stream` is a cudaStream_t passed as void* (NULL = the
 * legacy default stream). Return value: XKB_OK (0) or a negative XKB_E* code; the text
 * of the last error is available from xkb_last_error(). No entry point aborts the
 * process, and none falls back to a CPU implementation: without a usable GPU they
 * return XKB_ENODEV.
 *
 * Reference interfaces replaced (XKRT, file:line within its repository) are cited on
 * each declaration.
 */
#ifndef XKRT_B200_H
#define XKRT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#  define XKB_API __attribute__((visibility("default")))
#else
#  define XKB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ---------------------------------------------------------------------- */
#define XKB_OK          0
#define XKB_EINVAL     (-22)   /* bad argument (sizes, alignment, mode bits)             */
#define XKB_ENOMEM     (-12)   /* device or host allocation failed                       */
#define XKB_ERANGE     (-34)   /* an output or scratch capacity is too small; the needed */
                               /* capacity is reported through the call's out-parameter  */
#define XKB_ETIMEDOUT  (-110)  /* a bounded device-side wait gave up (no hang, no trap)  */
#define XKB_ENODEV     (-19)   /* no CUDA device / the library cannot reach the GPU       */
#define XKB_ECUDA      (-1000) /* a CUDA runtime call failed; see xkb_last_error()       */

/* Text of the last error set on the calling thread ("" if none). */
XKB_API const char * xkb_last_error(void);

/* Library version string and the device architecture it was compiled for ("sm_100a"). */
XKB_API const char * xkb_version(void);

/* ---- access records --------------------------------------------------------------------- */
/* Access modes and types: same values as the reference's
 * include/xkrt/memory/access/mode.h:54-66 and include/xkrt/memory/access/type.h. */
#define XKB_ACCESS_MODE_R   1
#define XKB_ACCESS_MODE_W   2
#define XKB_ACCESS_MODE_RW  3
#define XKB_ACCESS_MODE_V   4
#define XKB_ACCESS_MODE_D   8
#define XKB_ACCESS_TYPE_HANDLE      0
#define XKB_ACCESS_TYPE_SEGMENT     1
#define XKB_ACCESS_TYPE_BLAS_MATRIX 2

/* One access of one task, 64 bytes, tasks in spawn order and each task's accesses in
 * declaration order (the order in which the reference's spawning thread hands them to
 * task_dependency_resolve, src/task/task.cc:285-299).
 *  matrix : addr = storage base, ld, offset_m, offset_n, m, n, sizeof_type -- the
 *           arguments of access_t's matrix constructor (include/xkrt/memory/access/access.hpp:539-574)
 *  segment: byte interval [addr, ld)  -- access_t's segment constructor (access.hpp:479-514)
 *  handle : addr = the handle (an opaque pointer naming an object, not memory) -- access_t's
 *           handle constructor; resolved like the reference's DependencyMap
 *           (include/xkrt/memory/access/handle/dependency-map.hpp)
 *  reserved: bits 8-15 = the access's concurrency (xkrt_access_concurrency_t: 0 or 1 sequential,
 *           2 commutative, 4 concurrent); bits 0-7 are ignored by the resolver. The resolver
 *           takes sequential and commutative accesses (ordered alike, as in the reference); a
 *           stream with concurrent handle accesses goes through xkb_handle_map_expand first. */
typedef struct xkb_access_rec_t {
    uint32_t task;
    uint8_t  type;
    uint8_t  mode;
    uint16_t reserved;
    uint64_t addr;
    uint64_t ld;
    uint64_t offset_m;
    uint64_t offset_n;
    uint64_t m;
    uint64_t n;
    uint64_t sizeof_type;
} xkb_access_rec_t;

/* ---- dependency resolution ------------------------------------------------------------- */
/* A resolver keeps, per dependency domain, the last writer and the readers since that write
 * of every elementary cell, in HBM, so tasks can be added in batches (spawn order continues
 * across batches). It computes the same dependency edges as the reference's domains:
 * KBLASDependencyTree per (ld, sizeof) and IntervalDependencyTree, driven by
 * task_dependency_resolve (src/task/task.cc:203-299; include/xkrt/memory/access/blas/dependency-tree.hpp:228-426;
 * include/xkrt/memory/access/interval/dependency-tree.hpp:225-360), as the set of unique
 * (predecessor task, successor task) pairs. No task completes while resolving, so no edge is
 * dropped for a completed predecessor. */
typedef struct xkb_resolver xkb_resolver_t;

/* Successor graph in device memory (owned by the resolver, valid until its next call). */
typedef struct xkb_task_graph_t {
    uint64_t ntasks;
    uint64_t nedges;
    const uint32_t * succ_ptr;   /* [ntasks+1] CSR offsets into succ                           */
    const uint32_t * succ;       /* [nedges] successor task ids, ascending within each task     */
    const uint32_t * npred;      /* [ntasks] number of unique predecessors = initial wait count */
} xkb_task_graph_t;

/* Create a resolver working on `stream` (device = current device). Replaces the per-thread
 * implicit task's dependency domains (include/xkrt/task/task.hpp task_dom_info_t;
 * include/xkrt/thread/thread.h:159-196). */
XKB_API int xkb_resolver_create(xkb_resolver_t ** resolver, void * stream);
XKB_API int xkb_resolver_destroy(xkb_resolver_t * resolver);
/* Forget every task, edge and domain (the next add starts a new graph at task 0) but keep the
 * device and page-locked working buffers, so the next graph resolves without allocating them
 * again -- what a runtime does between waits (the reference drops its dependency domains with the
 * implicit task's, src/memory/invalidate.cc:103-121). */
XKB_API int xkb_resolver_reset(xkb_resolver_t * resolver);

/* Resolve a batch of host-resident access records (tasks dense, in spawn order, the first
 * one numbered like the number of tasks added so far). Replaces, for each task of the batch,
 * thread_t::resolve (include/xkrt/thread/thread.h:264-271) -> task_dependency_resolve
 * (src/task/task.cc:285-299). */
XKB_API int xkb_resolver_add(xkb_resolver_t * resolver, const xkb_access_rec_t * accesses, size_t naccesses);

/* Concurrent-mode handle accesses (ACCESS_CONCURRENCY_CONCURRENT), ordered as the reference's
 * DependencyMap orders them (include/xkrt/memory/access/handle/dependency-map.hpp:157-297): a
 * concurrent write depends on the last sequential write only, the next sequential access waits
 * for all the concurrent writes, and where the reference inserts an extra empty writer task
 * (insert_empty_write, :93-137) the expanded stream has one. xkb_handle_map_expand rewrites
 * records (tasks dense, in spawn order, continuing across calls like xkb_resolver_add) into a
 * stream the resolver takes: each extra task is a task of its own, numbered just before the task
 * whose access needed it (one handle access, mode VW), later tasks renumbered after it (task id
 * + extra tasks so far), and each concurrent write of a handle becomes a read of it. `out` needs
 * naccesses + (handle accesses) records at most (XKB_ERANGE if `cap` is smaller); *nout
 * receives the count. XKB_EINVAL for a concurrent access to a segment or matrix (the reference
 * asserts these sequential or commutative, access.hpp:500-502), and for the two forms whose
 * reference order no point-wise state expresses: a task listing a handle again after an access
 * that needs an extra writer, and a concurrent read-only access while concurrent writes of
 * earlier tasks are pending. After an error the map holds the state of the tasks before the
 * failing one. */
typedef struct xkb_handle_map xkb_handle_map_t;
XKB_API int xkb_handle_map_create(xkb_handle_map_t ** map);
XKB_API int xkb_handle_map_destroy(xkb_handle_map_t * map);
XKB_API int xkb_handle_map_expand(xkb_handle_map_t * map, const xkb_access_rec_t * in, size_t naccesses,
                                  xkb_access_rec_t * out, size_t cap, size_t * nout);

/* Build (if needed) and return the successor CSR of every task added so far. */
XKB_API int xkb_resolver_graph(xkb_resolver_t * resolver, xkb_task_graph_t * graph);

/* Copy the unique (pred, succ) pairs, sorted by pred then succ, to host memory as uint32
 * pairs. *nedges receives the count; XKB_ERANGE if cap_pairs is smaller. */
XKB_API int xkb_resolver_edges(xkb_resolver_t * resolver, uint32_t * pairs, size_t cap_pairs, size_t * nedges);

/* A periodic graph: the same window of `period` tasks repeated, task t of window w+1
 * depending on tasks of window w only through the `x` (cross-window) edges -- e.g. the
 * heat-diffusion graph with a window of two Jacobi steps (the grids swap back every two steps).
 * Device arrays, owned by the resolver that built them. */
typedef struct xkb_periodic_graph_t {
    uint64_t period;
    const uint32_t * succ_ptr;     /* [period+1] successors inside the same window              */
    const uint32_t * succ;
    const uint32_t * xsucc_ptr;    /* [period+1] successors in the NEXT window (ids in that window) */
    const uint32_t * xsucc;
    const uint32_t * npred_first;  /* [period] wait count of a task of the first window          */
    const uint32_t * npred_next;   /* [period] wait count of a task of every later window        */
} xkb_periodic_graph_t;

/* Extract the periodic form of a resolver holding exactly three windows of `period` tasks:
 * checks that window 1 repeats window 0 (its own and its incoming edges, shifted) and that no
 * edge skips a window; XKB_EINVAL if the graph is not periodic that way. */
XKB_API int xkb_resolver_periodic(xkb_resolver_t * resolver, uint64_t period, xkb_periodic_graph_t * out);

/* Counters: tasks added, unique edges, device+host time of the last batch in ms. */
XKB_API int xkb_resolver_stats(xkb_resolver_t * resolver, uint64_t * ntasks, uint64_t * nedges, double * last_batch_ms);
/* Where the last batch's time went: building the per-domain op lists (host), coordinate
 * compression (new boundaries found on the device, merged on the host), state refinement and
 * mapping of the ops to cells, and the whole batch (host and device). */
XKB_API int xkb_resolver_timing(xkb_resolver_t * resolver, double * ops_ms, double * compress_ms, double * batch_ms);

/* ---- coherency and transfer planning (1 host + 1 GPU) ------------------------------------ */
/* A planner decides, for each access fetched to the GPU (device 1) or back to the host
 * (device 0), which device allocation holds it and which copies make it coherent -- the
 * decisions of the reference's coherency controller, KBLASMemoryTree::fetch
 * (include/xkrt/memory/access/blas/memory-tree.hpp:1805-1874; fetch_list_to_device :1738-1802,
 * fetch_list_to_host :1185-1215), with every fetch's copies completed before the next fetch.
 * Device addresses are reported as (allocation ordinal, byte offset); host addresses as raw
 * byte addresses. A block needing a 9th allocation view returns XKB_ERANGE where the reference
 * aborts (MEMORY_REPLICATE_ALLOCATION_VIEWS_MAX, memory-tree.hpp:91,1364-1365). */
typedef struct xkb_planner xkb_planner_t;

#define XKB_COPY_H2D 0
#define XKB_COPY_D2H 1
#define XKB_COPY_D2D 2

typedef struct xkb_copy_t {
    int64_t task, access, kind;            /* issuing access; XKB_COPY_*                        */
    int64_t src_dev, src_alloc, src_off, src_ld;
    int64_t dst_dev, dst_alloc, dst_off, dst_ld;
    int64_t m, n, sizeof_type;             /* m x n elements (segments: m bytes, n = 1, size 1) */
} xkb_copy_t;

typedef struct xkb_view_t { int64_t alloc, off, ld; } xkb_view_t;   /* an access's device view */

XKB_API int xkb_planner_create(xkb_planner_t ** planner);
XKB_API int xkb_planner_destroy(xkb_planner_t * planner);
/* Fetch one access (record of task `access->task`, index `access_index` in that task) to
 * `device`; appends its copies; *view receives the device view the task body uses. */
XKB_API int xkb_planner_fetch(xkb_planner_t * planner, const xkb_access_rec_t * access, uint32_t access_index,
                              int device, xkb_view_t * view);
/* Fetch every access of a stream in order to `device`; views[i] (optional) for access i. */
XKB_API int xkb_planner_plan(xkb_planner_t * planner, const xkb_access_rec_t * accesses, size_t n, int device,
                             xkb_view_t * views);
/* Copies planned so far (*n = count; out may be NULL to query); take != 0 clears the list. */
XKB_API int xkb_planner_copies(xkb_planner_t * planner, xkb_copy_t * out, size_t cap, size_t * n, int take);
/* Byte size of every device allocation made so far, in allocation order. */
XKB_API int xkb_planner_allocations(xkb_planner_t * planner, uint64_t * sizes, size_t cap, size_t * n);

/* Device budget of a planner in the reference's mode (before its first fetch): every device
 * allocation gets an offset in one region of `bytes` bytes, handed out best fit (the reference's
 * area allocator, src/driver/device.cc:185-280; 256-byte rounding). When an allocation does not
 * fit, allocations the task being fetched does not use are evicted, oldest first: each block
 * loses its view on them, and a block whose only coherent copy was such a view is first copied
 * back to the host (a D2H record of the fetch that needed the room). The reference evicts only
 * blocks coherent elsewhere (memory-tree.hpp:1221-1324) and aborts when that is not enough;
 * XKB_ENOMEM here when the task's own allocations leave no room. */
XKB_API int xkb_planner_set_device_budget(xkb_planner_t * planner, uint64_t bytes);
/* Offset of each allocation in the budget, in allocation order, and whether it is still live
 * (either array may be NULL). An evicted allocation keeps its offset: the copies planned by the
 * fetch that evicted it read it before the room is reused (run each fetch's copies before the
 * next fetch). */
XKB_API int xkb_planner_allocation_offsets(xkb_planner_t * planner, int64_t * offsets, uint8_t * live, size_t cap, size_t * n);
/* Host fetches of a planner in the reference's mode copy from the largest allocation's view of a
 * block, as the reference does (memory-tree.hpp:1110-1160), even when that view is not coherent:
 * the host then receives stale data. on != 0: copy from the largest COHERENT view instead (what
 * the C API's reference mode does, so that host memory is right after xkrt_task_wait). */
XKB_API int xkb_planner_set_writeback_coherent(xkb_planner_t * planner, int on);
/* Allocations evicted and blocks written back to the host by evictions so far. */
XKB_API int xkb_planner_eviction_stats(xkb_planner_t * planner, uint64_t * evicted, uint64_t * written_back);

/* Registration-overflow protection of the reference's default build (XKRT_MEMORY_REGISTER_-
 * OVERFLOW_PROTECTION with protect_registered_memory_overflow on): host memory [ptr, ptr + size)
 * got registered / unregistered. The range is rounded out to pages; register takes the pieces not
 * registered yet, unregister every registered interval the range meets; each is inserted into
 * every (ld, sizeof) frame (and into frames made later, while registered) as its 1-3 rects, so no
 * block and no copy straddles a registration boundary (memory-tree.hpp:2184-2240,
 * src/memory/register.cc:89-262). The blocks' state is unchanged. Reference mode only.
 * Divergence: where a registration meets two or more registered intervals, the reference walks
 * them in tree order (its IntervalSet::find is not sorted, an assert of its debug build says
 * they should be); this planner walks them in address order. */
XKB_API int xkb_planner_register(xkb_planner_t * planner, uint64_t ptr, uint64_t size);
XKB_API int xkb_planner_unregister(xkb_planner_t * planner, uint64_t ptr, uint64_t size);

/* Forget every device copy: the host's copy of every block is the only coherent one again and
 * the next fetch of a block copies it from the host (the reference's runtime_t::reset drops the
 * coherency controllers and the device memory, src/memory/invalidate.cc:66-133). Reference mode:
 * the allocations are forgotten too (the next one is allocation 0 again, at offset 0 of a
 * budget); resident mode: the regions and their mirrors stay. Blocks whose only copy is on the
 * device are lost, as in the reference: write them back first (xkb_planner_flush_to_host in
 * resident mode). XKB_EINVAL while planned copies have not been taken. */
XKB_API int xkb_planner_invalidate(xkb_planner_t * planner);

/* Resident mode (the B200 layout): every host region registered with xkb_planner_add_region
 * has ONE device mirror with the host layout (allocation ordinal = region index, byte offset =
 * offset in the region). A fetch to the GPU copies (H2D) only the blocks of the access the
 * mirror lacks; a fetch to the host copies back (D2H) only blocks the host lacks; a write makes
 * the writer's copy the only coherent one. Blocks are the same canonical partition as above. */
XKB_API int xkb_planner_create_resident(xkb_planner_t ** planner);
XKB_API int xkb_planner_add_region(xkb_planner_t * planner, uint64_t host_base, uint64_t size, int32_t * region);
/* Resident mode: the regions inside [host_base, host_base + size) (none may cross its ends) are
 * replaced by one region covering it, with a new allocation ordinal: what registering memory
 * that overlaps registered memory does (the union becomes one region). The blocks keep their
 * coherency states; the caller moves the old mirrors' bytes into the new mirror. */
XKB_API int xkb_planner_replace_regions(xkb_planner_t * planner, uint64_t host_base, uint64_t size, int32_t * region);
/* Resident mode: make the host coherent again for every block whose only coherent copy is on
 * the GPU -- what fetching every record device tasks wrote back to the host does, without the
 * records (one walk over the partition). Blocks that follow one another in a slab and in the
 * same region are copied together (one D2H record per run, task and access -1); the blocks
 * become coherent on both sides. Replaces the write-back fetches of memory_coherent_async
 * (src/memory/coherent.cc:137-231) over the whole registered memory. */
XKB_API int xkb_planner_flush_to_host(xkb_planner_t * planner);

/* Run planned copies in order on `stream`: H2D and D2H with cudaMemcpy2DAsync, the D2D copies
 * of each access as one gather kernel (one CTA per copy). alloc_ptrs[k] is the device
 * memory backing allocation ordinal k (at least xkb_planner_allocations' size). Host addresses
 * in the records must be valid host memory (pinned memory makes the copies asynchronous).
 * Replaces the copy commands the reference queues per planned copy (runtime_t::copy,
 * src/memory/copy.cc:65-105, executed by src/driver/driver_cu.cc:616-767). */
XKB_API int xkb_plan_execute(const xkb_copy_t * copies, size_t n, void * const * alloc_ptrs, size_t nallocs, void * stream);

/* The reference tile body's contract on per-access replicas (diffusion_cuda,
 * examples/heat-diffusion-2d/src/kernels/diffusion.cu:130-154): src and dst are the replicas'
 * device views re-based to the tile origin as the example's launcher does
 * (examples/heat-diffusion-2d/src/main.cc:214-219), each with its own leading dimension;
 * nx, ny, c and the storage type are run-time arguments instead of compile-time constants. */
XKB_API int xkb_diffusion_views(int dtype, void * stream, const void * src, int64_t ld_src, void * dst, int64_t ld_dst,
                                int64_t tile_x, int64_t tile_y, int64_t tsx, int64_t tsy, int64_t nx, int64_t ny, double c);

/* ---- tasks and the device scheduler ------------------------------------------------------ */
/* Built-in task bodies the device scheduler can run inline (the reference runs them as
 * per-task kernel launches through a format's launcher, include/xkrt/driver/kernel-launcher.h:44-51). */
#define XKB_TASK_NOOP      0   /* placement / first-touch task with no body (src/memory/distribute.cc:86-170) */
#define XKB_TASK_HEAT_F64  1   /* heat tile, FP64 grids                                      */
#define XKB_TASK_HEAT_F32  2   /* heat tile, FP32 storage with FP64 arithmetic               */
#define XKB_TASK_AXPBY     3   /* y[lo:hi] = a*x[lo:hi] + b*y[lo:hi], FP64                    */

/* 64-byte task descriptor. heat: whole grids src/dst (device pointers, column-major, ld),
 * nx x ny, the tile's rows [x0,x1) x cols [y0,y1) (only interior cells are written), c.
 * axpby: device vectors x, y, element range [lo, hi), scalars a, b. */
typedef struct xkb_task_desc_t {
    uint32_t kind;
    uint32_t flags;
    union {
        struct { uint64_t src, dst; int64_t ld; int32_t nx, ny, x0, x1, y0, y1; double c; } heat;
        struct { uint64_t x, y; int64_t lo, hi; double a, b; } axpby;
        uint8_t raw[56];
    } u;
} xkb_task_desc_t;

/* Execution forms of a resolved task graph. */
#define XKB_FORM_PERSISTENT 0  /* one persistent kernel, device ready queue, inline task bodies   */
#define XKB_FORM_PLAIN      1  /* one kernel launch per task in spawn order (the reference's path) */
#define XKB_FORM_GRAPH      2  /* CUDA graph: one kernel node per task, one edge per dependency    */

typedef struct xkb_sched xkb_sched_t;

/* Scheduler bound to `stream`. Replaces the device threads' ready queues and launch loop
 * (src/sched.cc:249-351, :413-505) and completion/successor release (src/task.cc:160-247). */
XKB_API int xkb_sched_create(xkb_sched_t ** sched, void * stream);
XKB_API int xkb_sched_destroy(xkb_sched_t * sched);
/* Host array of task descriptors, in spawn order (task i of the graph = tasks[i]); copied. */
XKB_API int xkb_sched_set_tasks(xkb_sched_t * sched, const xkb_task_desc_t * tasks, size_t ntasks);
/* Longest time a persistent CTA waits for its next queue slot before it gives up and reports
 * XKB_ETIMEDOUT (default 10 s; finite, above 0 and at most 3600 s, else XKB_EINVAL). */
XKB_API int xkb_sched_set_timeout(xkb_sched_t * sched, double seconds);
/* CTAs of the persistent kernel (default: SMs x resident CTAs per SM). */
XKB_API int xkb_sched_set_grid(xkb_sched_t * sched, int ctas);
/* Heat tile body of the persistent kernel: 0 (default) = register body (16-byte vector loads
 * into registers, PF columns ahead, bulk L2 prefetch further ahead); 1 = bulk-staged body (per
 * warp, source columns stream into a ring of 8 shared-memory slots by asynchronous bulk copies,
 * cp.async.bulk with mbarrier completion, halo rows included). Same results either way; on the
 * 16384^2 FP64 graph the register body moves 4.8 TB/s and the bulk-staged one 3.2 TB/s. Tiles
 * whose rows are not 16-byte aligned always use the register body. */
XKB_API int xkb_sched_set_staging(xkb_sched_t * sched, int bulk);
/* Warps that execute one task in the persistent kernel (1, 2, 4 or 8; default 2): each CTA
 * of 8 warps runs 8 / warps_per_task tasks at a time, each team taking and releasing tasks on
 * its own. */
XKB_API int xkb_sched_set_team(xkb_sched_t * sched, int warps_per_task);
/* Distance, in columns, of the L2 bulk prefetch ahead of a heat tile's sweep (0 = off; default 4). */
XKB_API int xkb_sched_set_prefetch(xkb_sched_t * sched, int columns);
/* Enqueue one execution of the whole graph on the scheduler's stream (asynchronous). */
XKB_API int xkb_sched_run(xkb_sched_t * sched, const xkb_task_graph_t * graph, int form);
/* Wait for the stream; *executed = tasks the persistent kernel ran. Returns XKB_ETIMEDOUT if
 * a device wait ran out of time (the kernel returned; the context stays usable). */
XKB_API int xkb_sched_wait(xkb_sched_t * sched, uint64_t * executed);
/* Device time of the last run's persistent kernel (CUDA events on the scheduler's stream). */
XKB_API int xkb_sched_kernel_ms(xkb_sched_t * sched, double * ms);

/* Run `repeats` windows of a periodic graph in ONE persistent launch (the last window only up
 * to its first `tail` tasks, 1 <= tail <= period); the descriptors set with
 * xkb_sched_set_tasks are the window's `period` tasks. Task t of window w runs
 * tasks[t] -- the window's data must be valid for every repetition (for heat: an even number
 * of steps per window, so the grids are back in place). */
XKB_API int xkb_sched_run_periodic(xkb_sched_t * sched, const xkb_periodic_graph_t * graph, uint32_t repeats,
                                   uint32_t tail);

/* Persistent run of a graph that allocates nothing. This entry point has no counterpart in the
 * reference. It is for callers that cannot allocate device memory at the time they run a graph:
 * a runtime that reserved most of the GPU's memory for its own allocator at start-up (XKRT
 * reserves 90 % of HBM), a serving loop whose memory is already split into fixed pools, or a
 * latency-critical loop where cudaMalloc/cudaFree would synchronise the device. The wait
 * counters and queue live in one fixed array of the library (8 MiB + 256 B on every GPU that
 * loads it, held until the process exits), so a graph may have at most XKB_NOALLOC_MAX_TASKS
 * tasks; larger graphs get XKB_ERANGE. `tasks` is a DEVICE array of descriptors, `graph` the
 * resolver's device CSR. The call waits for the run to finish and returns XKB_ETIMEDOUT if a
 * device wait gave up after timeout_s seconds (finite, above 0, at most 3600 s); *executed
 * (optional) = tasks run.
 *
 * Set-up: the array and the kernels are device memory that the CUDA driver creates when the
 * library's module is first used on a device (modules load lazily), and the first call in each
 * CUDA context looks up the array's device address. Make one call with an empty graph
 * (ntasks = 0, tasks may be null) on each device before reserving device memory for other uses
 * and before any stream capture: it loads the module, the array and the kernels, so later
 * calls need no device memory at all.
 *
 * Descriptors are checked on the device before anything runs (the checks of
 * xkb_sched_set_tasks): a bad one returns XKB_EINVAL and no task runs. The successor CSR is
 * trusted: successor ids at or beyond ntasks are skipped, but wrong wait counts make the run
 * wait until timeout_s and return XKB_ETIMEDOUT. Every call shares the array: calls whose runs
 * overlap on the GPU (other streams, other host threads) race and must be serialised by the
 * caller. */
#define XKB_NOALLOC_MAX_TASKS (1u << 20)
XKB_API int xkb_sched_run_noalloc(const xkb_task_desc_t * tasks, const xkb_task_graph_t * graph, int warps_per_task,
                                  double timeout_s, void * stream, uint64_t * executed);

/* ---- serving: continuous admission of heat graphs under an HBM budget ------------------ */
typedef struct xkb_server xkb_server_t;

typedef struct xkb_server_cfg_t {
    uint64_t budget_bytes;   /* device memory the server reserves once and carves grids from    */
    int slots;               /* requests in flight at most (one stream each), 1..64              */
    int ctas_per_graph;      /* CTAs of each request's persistent kernel (0 = SMs x resident)    */
    double max_seconds;      /* xkb_server_run gives up (XKB_ETIMEDOUT) after this long (0: 600) */
} xkb_server_cfg_t;

/* One heat-diffusion request: nx x ny grid, ts x ts tiles, `steps` Jacobi steps, f32 = 1 for
 * FP32 storage, coefficient c; arrival_s is when it arrives (seconds after xkb_server_run
 * starts, non-decreasing). input (optional, host memory of nx*ny elements of the storage type;
 * page-locked memory makes its copy asynchronous) is the initial grid, copied in when the
 * request is admitted; without it the server builds the grid from `seed` (U[0,1) interior from
 * splitmix64 of seed * 0x100000001b3 + cell index, boundary 0). result (optional, host memory
 * of nx*ny elements) receives the final grid. start_s / finish_s are filled in: admission time,
 * and the time the host saw the result in `result` (or the run end). */
typedef struct xkb_request_t {
    double arrival_s;
    int64_t nx, ny, ts;
    int32_t steps, f32;
    uint64_t seed;
    double c;
    void * result;
    const void * input;
    double start_s, finish_s;
} xkb_request_t;

/* The serving loop of the path: requests are admitted in arrival order as soon as a slot is
 * free and their memory fits in the budget (best-fit allocation with split/merge, as the
 * reference's device allocator, src/driver/device.cc:49-280). ONE persistent kernel, launched
 * for the whole trace, runs the tile tasks of every admitted request: the host copies a request's
 * input grid in and writes its slot record; the kernel's idle teams set the request up (wait
 * counters, queue, second grid) and then take ready tasks from whichever request has some; the
 * host copies each result out as its last task ends. The graph of every request shape is
 * resolved (two-step windows, periodic form) before the loop starts. XKB_SERVE_MODE=launch in
 * the environment runs each request as its own persistent launch on its slot's stream instead. */
XKB_API int xkb_server_create(xkb_server_t ** server, const xkb_server_cfg_t * cfg);
XKB_API int xkb_server_destroy(xkb_server_t * server);
/* Serve a whole arrival trace; returns when every request has completed. */
XKB_API int xkb_server_run(xkb_server_t * server, xkb_request_t * requests, size_t n);

/* ---- heat-diffusion-2d tile body ------------------------------------------------------- */
/* Storage types for the stencil. XKB_F64: double storage and arithmetic. XKB_F32: float
 * storage, every cell update computed in double and rounded once to float on store. */
#define XKB_F64 0
#define XKB_F32 1

/* One Jacobi step of the 5-point heat stencil on the tile task (tile_x, tile_y) of an
 * nx x ny column-major grid (cell (i,j) at G[j*ld + i]):
 *   D(i,j) = S(i,j) + c*( (S(i+1,j) - 2S(i,j) + S(i-1,j)) + (S(i,j+1) - 2S(i,j) + S(i,j-1)) )
 * for the cells of rows [tile_x*tsx, tile_x*tsx+tsx) x cols [tile_y*tsy, tile_y*tsy+tsy)
 * that are interior (0 < i < nx-1, 0 < j < ny-1); boundary cells are never written.
 * src/dst are the WHOLE grids, resident on the device (this library keeps one replica per
 * grid in the host layout instead of one compact replica per access).
 * Replaces the tile body diffusion_cuda() of examples/heat-diffusion-2d/src/kernels/diffusion.cu:130-154
 * (c = ALPHA*DT/(DX*DY) with DX = DY = 1, examples/heat-diffusion-2d/src/main.cc:408-421). */
XKB_API int xkb_heat_tile(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                  int64_t tile_x, int64_t tile_y, int64_t tsx, int64_t tsy, double c, void * stream);

/* One whole Jacobi step (every interior cell of the grid) in one launch: the fused form of
 * all tile tasks of one step of examples/heat-diffusion-2d/src/main.cc:569-581 (update()). */
XKB_API int xkb_heat_step(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                  double c, void * stream);

/* Launch shape of the whole-step stencil kernel (chosen by xkb_heat_autotune or by hand).
 *   pf               east columns each lane loads before using any (2, 4 or 8)
 *   min_blocks       CTAs per SM the register budget is sized for (1, 2 or 4; pf 8 allows 1-2)
 *   ctas_per_sm      grid size = SMs x ctas_per_sm (the CTAs then stride over strips)
 *   l2_prefetch_cols distance, in columns, of the bulk L2 prefetch ahead of the sweep (0 = off)
 *   cols_per_strip   columns one warp sweeps per strip */
typedef struct xkb_heat_cfg_t {
    int pf;
    int min_blocks;
    int ctas_per_sm;
    int l2_prefetch_cols;
    int cols_per_strip;
} xkb_heat_cfg_t;

/* xkb_heat_step with an explicit launch shape (NULL = the library default). */
XKB_API int xkb_heat_step_cfg(int dtype, const void * src, void * dst, int64_t ld, int64_t nx, int64_t ny,
                              double c, const xkb_heat_cfg_t * cfg, void * stream);

/* FP64 checks of one Jacobi step's result, whatever the storage type (a precision mode keeps its
 * checks in FP64): into the DEVICE array out[4] -- out[0] the largest |dst| on the grid boundary
 * (0 for the Dirichlet-0 condition, which no task writes), out[1] the sum of dst^2 over the
 * interior (its square root is the grid's L2 norm), out[2] the residual of the step: the largest
 * |dst - (src + c*lap(src))| over the interior with src promoted to double and the update in the
 * reference's order (0 for FP64 grids; the storage rounding for FP32 ones), out[3] the largest
 * interior |dst|. No counterpart in the reference, whose example checks its grid by exporting it
 * (examples/heat-diffusion-2d/src/main.cc:115-163). Asynchronous on `stream`. */
XKB_API int xkb_heat_norms(int dtype, const void * src, const void * dst, int64_t ld, int64_t nx, int64_t ny, double c,
                           double * out, void * stream);

/* ---- axpby tile body -------------------------------------------------------------------- */
/* y[i] = a*x[i] + b*y[i] for i in [0, n), FP64, computed as (a*x) + (b*y) with no fused
 * multiply-add. No reference kernel exists; nearest reference task body is the byte-wise
 * z = x + y of examples/task-axpby.cc:43-52. */
XKB_API int xkb_axpby(int64_t n, double a, const double * x, double b, double * y, void * stream);

#ifdef __cplusplus
}
#endif
#endif /* XKRT_B200_H */
