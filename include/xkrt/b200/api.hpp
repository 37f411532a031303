/* The XKRT C++ source API on libxkb200: one header that defines what the reference's headers
 * <xkrt/runtime.h>, <xkrt/task/task.hpp>, <xkrt/task/format.h>, <xkrt/thread/thread.h>,
 * <xkrt/memory/access/access.hpp> and their neighbours give a program that builds its own
 * tasks, so that such a program recompiles unchanged against this include tree (each of those
 * paths is a small header here that includes this one).
 *
 * Kept from the reference (names, argument meaning, semantics):
 *  - runtime_t: init/deinit, task formats (create/put/set/get), task_commit, task_wait,
 *    task_complete, task_detachable_incr/decr, task_enqueue and its static forms,
 *    task_instanciate / task_spawn with std::function bodies and access setters,
 *    task_kernel_launch<synchronous> and the task_detachable_kernel_launch alias, host
 *    memory, registration, distribute_async and memory_coherent_async
 *    (include/xkrt/runtime.h:232-277, 400-504, 676-905, 1244-1311);
 *  - the task layout contract: task_t, task_dep_info_t, task_det_info_t, task_dev_info_t,
 *    task_compute_size, TASK_DEP_INFO / DET_INFO / DEV_INFO / DOM_INFO / MOL_INFO, TASK_ACCESSES,
 *    TASK_ARGS, TASK_SIZE -- blocks in the reference's order: task, dep, det, dev, dom, mol,
 *    accesses, args (include/xkrt/task/task.hpp:73-446); every block is padded to 8 bytes so the
 *    accesses behind them are aligned;
 *  - access_t with the reference's constructors for handles, segments (interval and
 *    pointer + count), BLAS matrices (with and without offsets), copies of another access and
 *    null accesses, its host_view and the device_view a body reads
 *    (include/xkrt/memory/access/access.hpp:452-665);
 *  - thread_t::get_tls / allocate_task / deallocate_all_tasks / resolve / commit
 *    (include/xkrt/thread/thread.h:254-284).
 * Bodies are called as f(runtime, device, task) (src/task.cc:336); a CUDA-target body launches
 * its kernels through runtime->task_kernel_launch, whose launcher receives a queue_cu_t whose
 * cu.handle.high is the stream to launch on (include/xkrt/driver/driver-cu.h).
 *
 * Execution: committed tasks join the C API runtime's current batch: dependencies are resolved
 * on the GPU, each task's data is made coherent where it runs, and the batch runs at task_wait
 * as a dataflow graph on a team of host threads (one CUDA stream each). Differences: a
 * moldable task's split condition is not consulted (it runs whole); thread_t::commit's enqueue
 * callback is not called (ready tasks always go to the library's scheduler); spawning from a
 * task body during task_wait is refused, as in the C API. */
#ifndef XKRT_B200_CXX_API_HPP
#define XKRT_B200_CXX_API_HPP

#include <atomic>
#include <cassert>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <new>

#include "../../xkrt_capi.h"
#include "../namespace.h"
#include "../support.h"
#include "../logger/logger.h"
#include "../logger/metric.h"
#include "../memory/access/blas/matrix.h"
#include "../utils/min-max.h"

/* ---- bridge into libxkb200 (C ABI; defined in xkaapi_b200/csrc/xkrt_capi.cc) -------------- */
extern "C" {
/* Bind a C++ runtime object to its C API runtime: bodies of C++ tasks receive cxx_runtime. */
XKB_API void   xkb_cxx_bind(xkrt_runtime_t * runtime, void * cxx_runtime);
/* Commit a task built with this header (task_t *): its accesses (dep_info->ac of them when the
 * task is DEPENDENT) order it after earlier tasks; it runs at the next wait. */
XKB_API void   xkb_cxx_commit(xkrt_runtime_t * runtime, void * task);
/* Detachable counter of a committed task: +1 (incr), -1 (decr; completes at 0), 0 (complete). */
XKB_API void   xkb_cxx_detachable(xkrt_runtime_t * runtime, void * task, int delta);
/* Inside a CUDA-target body: call launcher(cxx runtime, device, task, queue_cu_t *, NULL, 0). */
XKB_API void   xkb_cxx_kernel_launch(xkrt_runtime_t * runtime, void * device, void * task, int synchronous,
                                     xkrt_kernel_launcher_t launcher);
/* Task memory of the calling thread: 64-byte aligned, kept until released (never freed one by one). */
XKB_API void * xkb_cxx_allocate_task(size_t size);
XKB_API void   xkb_cxx_release_tasks(void);
}

XKRT_NAMESPACE_BEGIN

struct runtime_t;
struct thread_t;
struct team_t;
class access_t;

typedef xkrt_task_wait_counter_type_t   task_wait_counter_type_t;
typedef std::atomic<uint32_t>           task_wait_counter_t;
typedef xkrt_task_access_counter_type_t task_access_counter_t;
typedef xkrt_task_flags_t               task_flags_t;
typedef xkrt_task_flag_bitfield_t       task_flag_bitfield_t;
typedef xkrt_device_driver_id_t         device_driver_id_t;
typedef xkrt_device_global_id_t         device_global_id_t;
typedef xkrt_device_global_id_bitfield_t device_global_id_bitfield_t;
typedef xkrt_driver_type_t              driver_type_t;
typedef xkrt_driver_type_bitfield_t     driver_type_bitfield_t;
typedef xkrt_access_concurrency_t       access_concurrency_t;
typedef xkrt_access_mode_t              access_mode_t;
typedef xkrt_access_scope_t             access_scope_t;
typedef xkrt_access_type_t              access_type_t;
typedef xkrt_matrix_storage_t           matrix_storage_t;
typedef xkrt_task_format_id_t           task_format_id_t;
typedef xkrt_task_format_func_t         task_format_func_t;
typedef xkrt_task_format_target_t       task_format_target_t;
typedef xkrt_queue_type_t               queue_type_t;
typedef xkrt_queue_command_list_counter_t queue_command_list_counter_t;
typedef xkrt_kernel_launcher_t          kernel_launcher_t;
typedef xkrt_driver_module_t            driver_module_t;
typedef xkrt_driver_module_fn_t         driver_module_fn_t;

typedef enum task_state_t : uint8_t {
    TASK_STATE_ALLOCATED = 0, TASK_STATE_READY = 1, TASK_STATE_DATA_FETCHING = 2, TASK_STATE_DATA_FETCHED = 3,
    TASK_STATE_EXECUTING = 4, TASK_STATE_COMPLETED = 5, TASK_STATE_DEALLOCATED = 6, TASK_STATE_MAX = 7
} task_state_t;

/* A device as bodies see it: global id 0 is the host, 1 the GPU. */
struct device_t { int global_id; };

/* ---- tasks -------------------------------------------------------------------------------- */
constexpr uint32_t TASK_MAGIC = 0x786b7274u;   /* marks a task_t built with this header */

typedef struct task_t {
    task_t * parent;
    std::atomic<uint32_t> cc;                  /* uncompleted children */
    struct { uint32_t lock; task_state_t value; } state;
    task_format_id_t fmtid;
    task_flag_bitfield_t flags;
    uint32_t magic;
    uint64_t impl;                             /* the runtime's handle of the committed task */
#if XKRT_SUPPORT_DEBUG
    char label[128];
#endif
    task_t(task_format_id_t fmtid, task_flag_bitfield_t flags)
        : parent(nullptr), cc(0), state{0, TASK_STATE_ALLOCATED}, fmtid(fmtid), flags(flags), magic(TASK_MAGIC), impl(~0ull)
    {
#if XKRT_SUPPORT_DEBUG
        strncpy(this->label, "(unamed)", sizeof(this->label));
#endif
    }
} task_t;

/* dependency info: wait counter (1 until committed) and the number of accesses */
typedef struct alignas(8) task_dep_info_t {
    task_wait_counter_t wc;
    task_access_counter_t ac;
    task_dep_info_t(task_access_counter_t ac) : wc(1), ac(ac) {}
} task_dep_info_t;

/* detachable counter: the task completes when its body returned and the counter is back to 0 */
typedef struct alignas(8) task_det_info_t {
    task_wait_counter_t wc;
    task_det_info_t() : task_det_info_t(0) {}
    task_det_info_t(task_wait_counter_type_t value) : wc(value) {}
} task_det_info_t;

/* device info: the targeted device (UNSPECIFIED_DEVICE_GLOBAL_ID: the scheduler decides), the
 * access whose owner should run it (one GPU here: any owner is that GPU), the elected device */
typedef struct alignas(8) task_dev_info_t {
    device_global_id_t targeted_device_id;
    task_access_counter_t ocr_access_index;
    device_global_id_t elected_device_id;
    task_dev_info_t(device_global_id_t target, task_access_counter_t ocr)
        : targeted_device_id(target), ocr_access_index(ocr), elected_device_id(UNSPECIFIED_DEVICE_GLOBAL_ID) {}
} task_dev_info_t;

/* dependency domain of a task whose children spawn (the runtime keeps domains itself) */
typedef struct alignas(8) task_dom_info_t { void * domain; task_dom_info_t() : domain(nullptr) {} } task_dom_info_t;

/* moldability info (the split condition is kept but not consulted) */
typedef struct alignas(8) task_mol_info_t {
    const std::function<bool(task_t *, access_t *)> & split_condition;
    const size_t args_size;
    task_mol_info_t(const std::function<bool(task_t *, access_t *)> & split_condition, const size_t args_size = 0)
        : split_condition(split_condition), args_size(args_size) {}
} task_mol_info_t;

/* An invalid flag combination (DOMAIN with DEVICE) in a constant expression is a compile error. */
inline size_t task_flags_invalid(task_flag_bitfield_t flags)
{
    fprintf(stderr, "[xkrt] invalid task flag combination %u\n", (unsigned) flags);
    abort();
}

static constexpr size_t task_get_extra_size(const task_flag_bitfield_t flags)
{
    return ((flags & TASK_FLAG_DOMAIN) && (flags & TASK_FLAG_DEVICE)) ? task_flags_invalid(flags) :
           ((flags & TASK_FLAG_DEPENDENT)  ? sizeof(task_dep_info_t) : 0) +
           ((flags & TASK_FLAG_DETACHABLE) ? sizeof(task_det_info_t) : 0) +
           ((flags & TASK_FLAG_DEVICE)     ? sizeof(task_dev_info_t) : 0) +
           ((flags & TASK_FLAG_DOMAIN)     ? sizeof(task_dom_info_t) : 0) +
           ((flags & TASK_FLAG_MOLDABLE)   ? sizeof(task_mol_info_t) : 0);
}

/* ---- accesses ----------------------------------------------------------------------------- */
typedef uintptr_t INTERVAL_TYPE_T;

/* half-open interval [a, b) */
class Interval {
public:
    INTERVAL_TYPE_T a, b;
    Interval() : a(0), b(0) {}
    Interval(INTERVAL_TYPE_T a, INTERVAL_TYPE_T b) : a(a), b(b) {}
    bool is_empty() const { return b <= a; }
    bool intersects(const Interval & o) const { return a < o.b && o.a < b; }
    bool includes(const Interval & o) const { return a <= o.a && o.b <= b; }
    INTERVAL_TYPE_T length() const { return b > a ? b - a : 0; }
};

/* the host memory an access names: a column-major sub-matrix (a segment is m bytes with
 * ld = SIZE_MAX, a handle one byte) */
typedef struct memory_view_t {
    matrix_storage_t storage;
    uintptr_t addr;
    size_t ld, offset_m, offset_n, m, n, sizeof_type;
    memory_view_t(matrix_storage_t storage, uintptr_t addr, size_t ld, size_t offset_m, size_t offset_n, size_t m, size_t n,
                  size_t s)
        : storage(storage), addr(addr), ld(ld), offset_m(offset_m), offset_n(offset_n), m(m), n(n), sizeof_type(s) {}
    memory_view_t(matrix_storage_t storage, const void * addr, size_t ld, size_t offset_m, size_t offset_n, size_t m, size_t n,
                  size_t s)
        : memory_view_t(storage, (uintptr_t) addr, ld, offset_m, offset_n, m, n, s) {}
    /* address of the first element */
    uintptr_t begin_addr() const { return addr + (offset_n * ld + offset_m) * sizeof_type; }
} memory_view_t;

/* where a body finds the access's data: the address of its first element and the leading
 * dimension (in elements) on the device the body runs on */
typedef struct memory_replica_view_t {
    uintptr_t addr;
    size_t ld;
    memory_replica_view_t() : addr(0), ld(0) {}
    memory_replica_view_t(uintptr_t addr, size_t ld) : addr(addr), ld(ld) {}
} memory_replica_view_t;

typedef enum access_state_t : uint8_t { ACCESS_STATE_INIT, ACCESS_STATE_FETCHING, ACCESS_STATE_FETCHED } access_state_t;

class access_t {
public:
    access_state_t state;
    access_mode_t mode;
    access_concurrency_t concurrency;
    access_scope_t scope;
    access_type_t type;
    task_t * task;
    memory_view_t host_view;
    memory_replica_view_t device_view;      /* filled in before the body runs */

    /* handle */
    access_t(task_t * task, const void * addr, access_mode_t mode,
             access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL, access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : state(ACCESS_STATE_INIT), mode(mode), concurrency(concurrency), scope(scope), type(ACCESS_TYPE_HANDLE), task(task),
          host_view(MATRIX_COLMAJOR, addr, 1, 0, 0, 1, 1, 1), device_view() {}

    /* segment [a, b) */
    access_t(task_t * task, const uintptr_t a, const uintptr_t b, access_mode_t mode,
             access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL, access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : state(ACCESS_STATE_INIT), mode(mode), concurrency(concurrency), scope(scope), type(ACCESS_TYPE_SEGMENT), task(task),
          host_view(MATRIX_COLMAJOR, a, SIZE_MAX, 0, 0, (size_t) (b - a), 1, 1), device_view()
    {
        assert(a < b);
    }

    /* segment of n elements of sizeof_type bytes from ptr */
    access_t(task_t * task, const void * ptr, const size_t n, const size_t sizeof_type, access_mode_t mode,
             access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL, access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : access_t(task, ((uintptr_t) ptr), ((uintptr_t) ptr) + n * sizeof_type, mode, concurrency, scope) {}

    /* BLAS matrix: the m x n block at (offset_m, offset_n) of a column-major matrix of leading
     * dimension ld and element size s */
    access_t(task_t * task, const matrix_storage_t & storage, const void * addr, const size_t ld, const size_t offset_m,
             const size_t offset_n, const size_t m, const size_t n, const size_t s, access_mode_t mode,
             access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL, access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : state(ACCESS_STATE_INIT), mode(mode), concurrency(concurrency), scope(scope), type(ACCESS_TYPE_BLAS_MATRIX),
          task(task), host_view(storage, addr, ld, offset_m, offset_n, m, n, s), device_view()
    {
        assert(storage == MATRIX_COLMAJOR);
    }

    /* BLAS matrix from its first element */
    access_t(task_t * task, const matrix_storage_t & storage, const void * addr, const size_t ld, const size_t m, const size_t n,
             const size_t s, access_mode_t mode, access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL,
             access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : access_t(task, storage, addr, ld, 0, 0, m, n, s, mode, concurrency, scope) {}

    /* the memory of another access, in another mode */
    access_t(task_t * task, const access_t * other, access_mode_t mode,
             access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL, access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : access_t(task, other->host_view.storage, (const void *) other->host_view.addr, other->host_view.ld,
                   other->host_view.offset_m, other->host_view.offset_n, other->host_view.m, other->host_view.n,
                   other->host_view.sizeof_type, mode, concurrency, scope) {}

    /* null access: orders nothing, moves nothing */
    access_t(task_t * task, access_mode_t mode, access_concurrency_t concurrency = ACCESS_CONCURRENCY_SEQUENTIAL,
             access_scope_t scope = ACCESS_SCOPE_NONUNIFIED)
        : state(ACCESS_STATE_INIT), mode(mode), concurrency(concurrency), scope(scope), type(ACCESS_TYPE_NULL), task(task),
          host_view(MATRIX_COLMAJOR, (uintptr_t) 0, 0, 0, 0, 0, 0, 0), device_view() {}
};

/* ---- task layout ---------------------------------------------------------------------------- */
/* bytes of a task with these flags and ac accesses, without its arguments */
static constexpr inline size_t task_compute_size(const task_flag_bitfield_t flags, const task_access_counter_t ac)
{
    return sizeof(task_t) + task_get_extra_size(flags) + ac * sizeof(access_t);
}

static inline task_dep_info_t * TASK_DEP_INFO(const task_t * task)
{
    assert(task->flags & TASK_FLAG_DEPENDENT);
    return (task_dep_info_t *) (task + 1);
}

static inline task_det_info_t * TASK_DET_INFO(const task_t * task)
{
    assert(task->flags & TASK_FLAG_DETACHABLE);
    return (task_det_info_t *) ((char *) (task + 1) + ((task->flags & TASK_FLAG_DEPENDENT) ? sizeof(task_dep_info_t) : 0));
}

static inline task_dev_info_t * TASK_DEV_INFO(const task_t * task)
{
    assert((task->flags & TASK_FLAG_DEVICE) && !(task->flags & TASK_FLAG_DOMAIN));
    return (task_dev_info_t *) ((char *) (task + 1) + task_get_extra_size(task->flags & (TASK_FLAG_DEPENDENT | TASK_FLAG_DETACHABLE)));
}

static inline task_dom_info_t * TASK_DOM_INFO(const task_t * task)
{
    assert((task->flags & TASK_FLAG_DOMAIN) && !(task->flags & TASK_FLAG_DEVICE));
    return (task_dom_info_t *) ((char *) (task + 1) + task_get_extra_size(task->flags & (TASK_FLAG_DEPENDENT | TASK_FLAG_DETACHABLE)));
}

static inline task_mol_info_t * TASK_MOL_INFO(const task_t * task)
{
    assert(task->flags & TASK_FLAG_MOLDABLE);
    return (task_mol_info_t *) ((char *) (task + 1) +
                                task_get_extra_size(task->flags & (TASK_FLAG_DEPENDENT | TASK_FLAG_DETACHABLE | TASK_FLAG_DEVICE | TASK_FLAG_DOMAIN)));
}

/* tells the runtime to requeue this task after its body returns */
#define TASK_MUST_REQUEUE(T) do { (T)->flags |= TASK_FLAG_REQUEUE; } while (0)

static constexpr size_t TASK_ACCESSES_OFFSET(const task_flag_bitfield_t flags)
{
    return sizeof(task_t) + task_get_extra_size(flags & ~TASK_FLAG_REQUEUE);
}

static inline access_t * TASK_ACCESSES(const task_t * task, const task_flag_bitfield_t flags)
{
    return (access_t *) (((char *) task) + TASK_ACCESSES_OFFSET(flags));
}

static inline access_t * TASK_ACCESSES(const task_t * task) { return TASK_ACCESSES(task, task->flags); }

static inline void * TASK_ARGS(const task_t * task, const size_t task_size) { return (void *) (((char *) task) + task_size); }

static inline size_t TASK_SIZE(const task_t * task)
{
    const size_t ac = (task->flags & TASK_FLAG_DEPENDENT) ? TASK_DEP_INFO(task)->ac : 0;
    return TASK_ACCESSES_OFFSET(task->flags) + ac * sizeof(access_t);
}

static inline void * TASK_ARGS(const task_t * task) { return TASK_ARGS(task, TASK_SIZE(task)); }

/* ---- formats -------------------------------------------------------------------------------- */
typedef xkrt_task_format_target_t (*task_format_suggest_t)(void * task);

typedef struct xkrt_task_format_t {
    xkrt_task_format_func_t f[XKRT_TASK_FORMAT_TARGET_MAX];
    char label[32];
    xkrt_task_format_target_t (*suggest)(void * task);
} task_format_t;

#define XKRT_TASK_FORMAT_TARGET_NO_SUGGEST XKRT_TASK_FORMAT_TARGET_MAX

/* ---- threads -------------------------------------------------------------------------------- */
runtime_t * runtime_current();

struct thread_t {
    int tid = 0;
    task_t * current_task = nullptr;
    thread_t * prev = nullptr;

    /* the calling thread's object */
    static thread_t * get_tls()
    {
        static thread_local thread_t self;
        return &self;
    }

    /* task memory (64-byte aligned), kept until deallocate_all_tasks or the runtime's deinit */
    task_t * allocate_task(const size_t size) { return (task_t *) xkb_cxx_allocate_task(size); }
    void deallocate_all_tasks(void) { xkb_cxx_release_tasks(); }

    /* the reference inserts the accesses into the dependency trees here; this runtime resolves
     * every committed task's accesses on the GPU when the batch is handed over */
    inline void resolve(access_t * accesses, task_access_counter_t AC)
    {
        assert(AC > 0);
        assert(accesses);
        (void) accesses; (void) AC;
    }

    /* commit a task; the ready callback F is the reference's queue hand-off (unused: ready tasks
     * go to the library's scheduler). One overload per callback shape the reference's runtime
     * passes (runtime_t::task_enqueue, task_thread_enqueue, task_team_enqueue), so an overloaded
     * name resolves as it does there, and a template for any other callback. */
    inline void commit(task_t * task, void (*F)(runtime_t *, task_t *), runtime_t * runtime);
    inline void commit(task_t * task, void (*F)(runtime_t *, thread_t *, task_t *), runtime_t * runtime, thread_t * thread);
    inline void commit(task_t * task, void (*F)(runtime_t *, team_t *, task_t *), runtime_t * runtime, team_t * team);
    template <typename FN, typename... Args>
    inline void commit(task_t * task, FN F, Args... args);
};

/* ---- runtime -------------------------------------------------------------------------------- */
typedef enum distribution_type_t {
    XKRT_DISTRIBUTION_TYPE_CYCLIC1D,
    XKRT_DISTRIBUTION_TYPE_CYCLIC2D,
    XKRT_DISTRIBUTION_TYPE_CYCLIC2DBLOCK,
    XKRT_DISTRIBUTION_TYPE_MAX
} distribution_type_t;

struct runtime_t {
    xkrt_runtime_t * capi = nullptr;
    struct { struct { unsigned int n = 0; } devices; } drivers;
    struct { task_format_id_t host_capture = 0; } formats;
    task_format_t format_table[256];

    typedef std::function<void(runtime_t *, device_t *, task_t *)> task_routine_t;
    typedef std::function<void(task_t *, access_t *)> task_accesses_setter_t;

    int init(void);
    int deinit(void);
    void reset(void) { if (capi) xkrt_reset(capi); }

    /* formats */
    task_format_id_t task_format_create(const task_format_t * format)
    {
        const task_format_id_t id = task_format_put(format->label);
        if (!id) return 0;
        for (int t = 0; t < XKRT_TASK_FORMAT_TARGET_MAX; ++t)
            if (format->f[t]) task_format_set(id, (task_format_target_t) t, format->f[t]);
        format_table[id].suggest = format->suggest;
        return id;
    }
    task_format_id_t task_format_put(const char * label)
    {
        const task_format_id_t id = xkrt_task_format_put(capi, label);
        if (id)
        {
            memset(&format_table[id], 0, sizeof(task_format_t));
            snprintf(format_table[id].label, sizeof(format_table[id].label), "%s", label ? label : "");
        }
        return id;
    }
    int task_format_set(task_format_id_t fmtid, task_format_target_t target, task_format_func_t func)
    {
        const int rc = xkrt_task_format_set(capi, fmtid, target, func);
        if (rc == 0) format_table[fmtid].f[target] = func;
        return rc;
    }
    task_format_t * task_format_get(task_format_id_t fmtid) { return fmtid ? &format_table[fmtid] : nullptr; }

    /* tasking */
    void task_commit(task_t * task) { xkb_cxx_commit(capi, task); }
    void task_detachable_decr(task_t * task) { xkb_cxx_detachable(capi, task, -1); }
    void task_detachable_incr(task_t * task) { xkb_cxx_detachable(capi, task, +1); }
    void task_complete(task_t * task) { xkb_cxx_detachable(capi, task, 0); }
    void task_wait(void) { xkrt_task_wait(capi); }
    void task_enqueue(task_t * task) { xkb_cxx_commit(capi, task); }
    static inline void task_enqueue(runtime_t * runtime, task_t * task) { runtime->task_enqueue(task); }
    void task_thread_enqueue(thread_t *, task_t * task) { task_enqueue(task); }
    static inline void task_thread_enqueue(runtime_t * runtime, thread_t * thread, task_t * task)
    {
        runtime->task_thread_enqueue(thread, task);
    }
    void task_team_enqueue(team_t *, task_t * task) { task_enqueue(task); }
    static inline void task_team_enqueue(runtime_t * runtime, team_t * team, task_t * task) { runtime->task_team_enqueue(team, task); }

    /* a task of format fmtid whose args are a copy of args, with naccesses accesses set by
     * set_accesses and resolved */
    template <task_flag_bitfield_t flags>
    inline task_t * task_instanciate(const task_format_id_t fmtid, const void * args, const size_t args_size,
                                     const task_accesses_setter_t & set_accesses, const task_access_counter_t naccesses)
    {
        assert(naccesses > 0);
        assert(set_accesses);
        thread_t * tls = thread_t::get_tls();
        const size_t task_size = task_compute_size(flags, naccesses);
        task_t * task = tls->allocate_task(task_size + args_size);
        new (task) task_t(fmtid, flags);
        new (TASK_DEP_INFO(task)) task_dep_info_t(naccesses);
        if (args_size) memcpy(TASK_ARGS(task, task_size), args, args_size);
        access_t * accesses = TASK_ACCESSES(task, flags);
        set_accesses(task, accesses);
        tls->resolve(accesses, naccesses);
        return task;
    }

    template <task_flag_bitfield_t flags, size_t args_size>
    inline task_t * task_instanciate(const task_format_id_t fmtid, const task_accesses_setter_t & set_accesses,
                                     const task_access_counter_t naccesses)
    {
        thread_t * tls = thread_t::get_tls();
        const size_t task_size = task_compute_size(flags, naccesses);
        task_t * task = tls->allocate_task(task_size + args_size);
        new (task) task_t(fmtid, flags);
        new (TASK_DEP_INFO(task)) task_dep_info_t(naccesses);
        access_t * accesses = TASK_ACCESSES(task, flags);
        set_accesses(task, accesses);
        tls->resolve(accesses, naccesses);
        return task;
    }

    /* a host task whose body is the function f (copied into the task's args) */
    template <task_access_counter_t ac, bool has_set_accesses, bool has_split_condition>
    inline task_t * task_instanciate(const std::function<void(runtime_t *, device_t *, task_t *)> & f,
                                     const task_accesses_setter_t & set_accesses,
                                     const std::function<bool(task_t *, access_t *)> & split_condition)
    {
        static_assert(ac == 0 || has_set_accesses, "accesses need a setter");
        static_assert(!has_split_condition || ac > 0, "a task without accesses cannot split");
        constexpr task_flag_bitfield_t depflag = ac ? TASK_FLAG_DEPENDENT : TASK_FLAG_ZERO;
        constexpr task_flag_bitfield_t molflag = has_split_condition ? TASK_FLAG_MOLDABLE : TASK_FLAG_ZERO;
        constexpr task_flag_bitfield_t flags = depflag | molflag;
        constexpr size_t task_size = task_compute_size(flags, ac);
        thread_t * tls = thread_t::get_tls();
        task_t * task = tls->allocate_task(task_size + sizeof(task_routine_t));
        new (task) task_t(formats.host_capture, flags);
        new (TASK_ARGS(task, task_size)) task_routine_t(f);
        if constexpr (ac > 0)
        {
            new (TASK_DEP_INFO(task)) task_dep_info_t(ac);
            access_t * accesses = TASK_ACCESSES(task, flags);
            set_accesses(task, accesses);
            tls->resolve(accesses, ac);
        }
        if constexpr (has_split_condition) new (TASK_MOL_INFO(task)) task_mol_info_t(split_condition, sizeof(task_routine_t));
        return task;
    }

    template <task_access_counter_t ac, bool has_set_accesses, bool has_split_condition>
    inline void task_spawn(const task_accesses_setter_t & set_accesses,
                           const std::function<bool(task_t *, access_t *)> & split_condition,
                           const std::function<void(runtime_t *, device_t *, task_t *)> & f)
    {
        task_t * task = this->task_instanciate<ac, has_set_accesses, has_split_condition>(f, set_accesses, split_condition);
        thread_t::get_tls()->commit(task, task_enqueue, this);
    }

    template <task_access_counter_t ac>
    inline void task_spawn(const task_accesses_setter_t & set_accesses,
                           const std::function<bool(task_t *, access_t *)> & split_condition,
                           const std::function<void(runtime_t *, device_t *, task_t *)> & f)
    {
        this->task_spawn<ac, true, true>(set_accesses, split_condition, f);
    }

    template <task_access_counter_t ac>
    inline void task_spawn(const task_accesses_setter_t & set_accesses, const std::function<void(runtime_t *, device_t *, task_t *)> & f)
    {
        this->task_spawn<ac, true, false>(set_accesses, nullptr, f);
    }

    inline void task_spawn(const std::function<void(runtime_t *, device_t *, task_t *)> & f)
    {
        this->task_spawn<0, false, false>(nullptr, nullptr, f);
    }

    /* kernel launch from a CUDA-target body: the launcher gets the queue of the thread running
     * the body; the task completes once its kernels did */
    template <bool synchronous>
    void task_kernel_launch(device_t * device, task_t * task, kernel_launcher_t launcher)
    {
        xkb_cxx_kernel_launch(capi, device, task, synchronous ? 1 : 0, launcher);
    }
    void task_detachable_kernel_launch(device_t * device, task_t * task, kernel_launcher_t launcher)
    {
        task_kernel_launch<false>(device, task, launcher);
    }

    /* memory */
    void * memory_host_allocate(const device_global_id_t device_global_id, const size_t size)
    {
        return xkrt_memory_host_allocate(capi, device_global_id, size);
    }
    void memory_host_deallocate(const device_global_id_t device_global_id, void * mem, const size_t size)
    {
        xkrt_memory_host_deallocate(capi, device_global_id, mem, size);
    }
    void * memory_unified_allocate(const device_global_id_t device_global_id, const size_t size)
    {
        return xkrt_memory_unified_allocate(capi, device_global_id, size);
    }
    void memory_unified_deallocate(const device_global_id_t device_global_id, void * mem, const size_t size)
    {
        xkrt_memory_unified_deallocate(capi, device_global_id, mem, size);
    }
    int memory_register(void * ptr, size_t size) { return xkrt_memory_register(capi, ptr, size); }
    int memory_unregister(void * ptr, size_t size) { return xkrt_memory_unregister(capi, ptr, size); }
    int memory_register_async(void * ptr, size_t size) { return xkrt_memory_register_async(capi, ptr, size); }
    int memory_unregister_async(void * ptr, size_t size) { return xkrt_memory_unregister_async(capi, ptr, size); }

    /* placement: one empty task with a read access per tile (halo hx, hy) on the device the
     * distribution gives it (src/memory/distribute.cc:86-170); one GPU receives every tile */
    void distribute_async(distribution_type_t type, matrix_storage_t storage, void * ptr, size_t ld, size_t m, size_t n, size_t mb,
                          size_t nb, size_t sizeof_type, size_t hx, size_t hy);
    void distribute_async(distribution_type_t type, void * ptr, size_t size, size_t nb, size_t h);

    /* an empty task with a read access on the memory, run on the device: the device (the host
     * for HOST_DEVICE_GLOBAL_ID) holds a coherent copy afterwards (src/memory/coherent.cc:100-231) */
    void memory_coherent_async(device_global_id_t device_global_id, void * ptr, size_t size);
    void memory_coherent_async(device_global_id_t device_global_id, matrix_storage_t storage, void * ptr, size_t ld, size_t m,
                               size_t n, size_t sizeof_type);

    unsigned int get_ndevices(void) { return xkrt_get_ndevices(capi); }

private:
    void spawn_read_task(device_global_id_t device, const access_t & proto);
};

/* the runtime initialised last (the one thread_t::commit hands tasks to) */
inline std::atomic<runtime_t *> & runtime_current_slot()
{
    static std::atomic<runtime_t *> cur{nullptr};
    return cur;
}
inline runtime_t * runtime_current() { return runtime_current_slot().load(std::memory_order_acquire); }

inline void thread_t::commit(task_t * task, void (*F)(runtime_t *, task_t *), runtime_t * runtime)
{
    (void) F;
    runtime->task_commit(task);
}

inline void thread_t::commit(task_t * task, void (*F)(runtime_t *, thread_t *, task_t *), runtime_t * runtime, thread_t * thread)
{
    (void) F; (void) thread;
    runtime->task_commit(task);
}

inline void thread_t::commit(task_t * task, void (*F)(runtime_t *, team_t *, task_t *), runtime_t * runtime, team_t * team)
{
    (void) F; (void) team;
    runtime->task_commit(task);
}

template <typename FN, typename... Args>
inline void thread_t::commit(task_t * task, FN F, Args... args)
{
    (void) F;
    ((void) args, ...);
    runtime_t * rt = runtime_current();
    assert(rt);
    if (rt) rt->task_commit(task);
}

/* body of the std::function tasks (formats.host_capture) */
static inline void runtime_host_capture_body(runtime_t * runtime, device_t * device, task_t * task)
{
    runtime_t::task_routine_t * f = (runtime_t::task_routine_t *) TASK_ARGS(task);
    (*f)(runtime, device, task);
    std::destroy_at(f);
}

inline int runtime_t::init(void)
{
    const int rc = xkrt_init(&capi);
    if (rc) return rc;
    drivers.devices.n = xkrt_get_ndevices(capi);
    xkb_cxx_bind(capi, this);
    memset(format_table, 0, sizeof(format_table));
    task_format_t capture;
    memset(&capture, 0, sizeof(capture));
    capture.f[XKRT_TASK_FORMAT_TARGET_HOST] = (task_format_func_t) runtime_host_capture_body;
    snprintf(capture.label, sizeof(capture.label), "host-capture");
    formats.host_capture = task_format_create(&capture);
    runtime_current_slot().store(this, std::memory_order_release);
    return 0;
}

inline int runtime_t::deinit(void)
{
    if (!capi) return 0;
    xkrt_task_wait(capi);
    const int rc = xkrt_deinit(capi);
    capi = nullptr;
    xkb_cxx_release_tasks();
    runtime_t * self = this;
    runtime_current_slot().compare_exchange_strong(self, nullptr);
    return rc;
}

inline void runtime_t::spawn_read_task(device_global_id_t device, const access_t & proto)
{
    constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT | TASK_FLAG_DEVICE;
    constexpr size_t task_size = task_compute_size(flags, 1);
    task_t * task = thread_t::get_tls()->allocate_task(task_size);
    new (task) task_t(XKRT_TASK_FORMAT_NULL, device == HOST_DEVICE_GLOBAL_ID ? (task_flag_bitfield_t) TASK_FLAG_DEPENDENT : flags);
    new (TASK_DEP_INFO(task)) task_dep_info_t(1);
    if (device != HOST_DEVICE_GLOBAL_ID) new (TASK_DEV_INFO(task)) task_dev_info_t(device, 0);
    access_t * a = TASK_ACCESSES(task);
    new (a) access_t(proto);
    a->task = task;
    task_commit(task);
}

inline void runtime_t::distribute_async(distribution_type_t type, matrix_storage_t storage, void * ptr, size_t ld, size_t m,
                                        size_t n, size_t mb, size_t nb, size_t sizeof_type, size_t hx, size_t hy)
{
    (void) type;
    if (!mb || !nb) return;
    const device_global_id_t gpu = drivers.devices.n > 1 ? 1 : HOST_DEVICE_GLOBAL_ID;
    for (size_t tx = 0; tx < (m + mb - 1) / mb; ++tx)
        for (size_t ty = 0; ty < (n + nb - 1) / nb; ++ty)
        {
            const size_t x0 = tx * mb > hx ? tx * mb - hx : 0, y0 = ty * nb > hy ? ty * nb - hy : 0;
            const size_t x1 = (tx + 1) * mb + hx < m ? (tx + 1) * mb + hx : m, y1 = (ty + 1) * nb + hy < n ? (ty + 1) * nb + hy : n;
            spawn_read_task(gpu, access_t(nullptr, storage, ptr, ld, x0, y0, x1 - x0, y1 - y0, sizeof_type, ACCESS_MODE_R));
        }
}

inline void runtime_t::distribute_async(distribution_type_t type, void * ptr, size_t size, size_t nb, size_t h)
{
    (void) type;
    if (!nb) return;
    const device_global_id_t gpu = drivers.devices.n > 1 ? 1 : HOST_DEVICE_GLOBAL_ID;
    for (size_t b = 0; b < size; b += nb)
    {
        const size_t lo = b > h ? b - h : 0, hi = b + nb + h < size ? b + nb + h : size;
        spawn_read_task(gpu, access_t(nullptr, (uintptr_t) ptr + lo, (uintptr_t) ptr + hi, ACCESS_MODE_R));
    }
}

inline void runtime_t::memory_coherent_async(device_global_id_t device_global_id, void * ptr, size_t size)
{
    if (size) spawn_read_task(device_global_id, access_t(nullptr, (uintptr_t) ptr, (uintptr_t) ptr + size, ACCESS_MODE_R));
}

inline void runtime_t::memory_coherent_async(device_global_id_t device_global_id, matrix_storage_t storage, void * ptr, size_t ld,
                                             size_t m, size_t n, size_t sizeof_type)
{
    if (m && n) spawn_read_task(device_global_id, access_t(nullptr, storage, ptr, ld, 0, 0, m, n, sizeof_type, ACCESS_MODE_R));
}

XKRT_NAMESPACE_END

#endif /* XKRT_B200_CXX_API_HPP */
