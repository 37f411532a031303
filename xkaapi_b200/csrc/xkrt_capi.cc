// The XKRT C API (task spawn, accesses, formats, wait) over libxkb200.
//
// Reference behaviour kept (api/c/src/xkrt.cc, src/task.cc, src/task/task.cc):
//  * tasks get dependencies from their accesses in spawn order (LINK all, then PUT all); a task
//    runs once every predecessor ran; format bodies are called as f(runtime, device, task) and
//    team/func spawns as func(runtime, device, task, user_data) (xkrt.cc:540-642);
//  * formats are numbered from 1 (XKRT_TASK_FORMAT_NULL = 0) and hold one function per target.
// B200 design: spawns are buffered until xkrt_task_wait; the batch's dependencies are resolved
// on the GPU; data coherency uses the resident planner (one device mirror per registered host
// region, copies only for blocks the executing side lacks); a batch of built-in device bodies
// runs as one persistent-scheduler launch, any other batch as a dataflow graph on a team of host
// threads. Host memory is coherent again when xkrt_task_wait returns.
#include "capi_objects.h"
#include "common.cuh"
#include "handles.h"
#include "internal.h"
#include "pool.h"
#include "../../include/xkrt_capi.h"
#include "../../include/xkrt/b200/api.hpp"
#include "../../include/xkrt/driver/driver-cu.h"

#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <mutex>
#include <memory>
#include <new>
#include <thread>
#include <string>
#include <vector>

struct xkb_runtime;

// Accesses per resolver batch: the resolver's working set grows with the batch, and batches of
// about a million accesses keep it small while amortising each batch's fixed costs.
constexpr size_t RESOLVE_CHUNK = size_t(1) << 20;

namespace {

struct Format {
    bool used = false;
    std::string label;
    xkrt_task_format_func_t f[XKRT_TASK_FORMAT_TARGET_MAX] = {};
    int builtin = -1;                     // XKB_TASK_* for built-in device bodies
};

// A spawned task. Tasks, their arguments, accesses and replica pointers live in the runtime's
// pools (one mapping per pool, not one allocation per task); the pools only grow during spawns,
// so their addresses are stable while bodies run.
struct Task {
    ::xkb_runtime * rt = nullptr;
    uint8_t fmtid = 0, flags = 0;
    xkrt_device_global_id_t device = 0;
    uint32_t nargs = 0, nacc = 0;
    size_t args_off = 0, acc_off = 0;
    xkrt_task_func_t func = nullptr;      // team / plain function spawns
    void * user_data = nullptr;           // their argument; without func: the task_t of a task built
                                          // with the C++ source API (null otherwise)
    int detach = 0;                       // references (atomic builtins): the running body's, plus each
                                          // xkrt_task_detachable_incr; the task completes at 0
};
static_assert(sizeof(Task) == 64, "a spawned task record is one cache line");

// The task_t of a task built with the C++ source API, or null.
static inline void * cxx_of(const Task & T) { return T.func ? nullptr : T.user_data; }

struct Region { uint64_t size; void * mirror; bool pinned_by_us; int32_t id; bool unified; };

// Drop one reference of a task; true when it was the last one (the task completes now).
// A task already at 0 (completed by xkrt_task_complete) stays there.
static bool task_unref(Task & T)
{
    int v = __atomic_load_n(&T.detach, __ATOMIC_ACQUIRE);
    while (v > 0)
        if (__atomic_compare_exchange_n(&T.detach, &v, v - 1, false, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE)) return v == 1;
    return false;
}

using xkb_capi::Device;
using xkb_capi::Driver;
using xkb_capi::Queue;

thread_local Task * g_current = nullptr;  // task whose body runs on this thread (xkrt_task_current)
thread_local cudaStream_t g_stream = nullptr;   // the stream of the worker running a CUDA body

// Records that name the same bytes in the same mode: fetching them again to the same device is a
// no-op (a device fetch never invalidates the device's copy of other data), so batches whose
// fetches all go one way fetch each distinct record once. The set grows with the number of
// DISTINCT records (a few per tile for a stencil), so it stays in cache however long the batch.
class RecordSet {
public:
    RecordSet() : slot_(1024, UINT32_MAX) {}
    // true if r (task id ignored) was not in the set; it is now
    bool insert(const xkb_access_rec_t * recs, uint32_t i)
    {
        if (2 * (used_ + 1) > slot_.size()) rehash(recs);
        const size_t mask = slot_.size() - 1;
        size_t h = key_hash(recs[i]) & mask;
        while (slot_[h] != UINT32_MAX)
        {
            if (same(recs[slot_[h]], recs[i])) return false;
            h = (h + 1) & mask;
        }
        slot_[h] = i;
        ++used_;
        return true;
    }
    // whether a record equal to recs[i] is in the set (read only: callable from several threads)
    bool contains(const xkb_access_rec_t * recs, uint32_t i) const
    {
        const size_t mask = slot_.size() - 1;
        size_t h = key_hash(recs[i]) & mask;
        while (slot_[h] != UINT32_MAX)
        {
            if (same(recs[slot_[h]], recs[i])) return true;
            h = (h + 1) & mask;
        }
        return false;
    }
    void reset() { slot_.assign(1024, UINT32_MAX); used_ = 0; }
    static uint64_t key_hash(const xkb_access_rec_t & r)
    {
        uint64_t h = ((uint64_t) r.type << 8) | r.mode;
        for (uint64_t v : {r.addr, r.ld, r.offset_m, r.offset_n, r.m, r.n, r.sizeof_type}) h = mix(h, v);
        return h * 0xff51afd7ed558ccdull;
    }
private:
    void rehash(const xkb_access_rec_t * recs)
    {
        std::vector<uint32_t> old(2 * slot_.size(), UINT32_MAX);
        old.swap(slot_);
        const size_t mask = slot_.size() - 1;
        for (uint32_t i : old)
            if (i != UINT32_MAX)
            {
                size_t h = key_hash(recs[i]) & mask;
                while (slot_[h] != UINT32_MAX) h = (h + 1) & mask;
                slot_[h] = i;
            }
    }
    static uint64_t mix(uint64_t h, uint64_t v) { h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2); return h; }
    static bool same(const xkb_access_rec_t & a, const xkb_access_rec_t & b)
    {
        return a.type == b.type && a.mode == b.mode && a.addr == b.addr && a.ld == b.ld && a.offset_m == b.offset_m &&
               a.offset_n == b.offset_n && a.m == b.m && a.n == b.n && a.sizeof_type == b.sizeof_type;
    }
    std::vector<uint32_t> slot_;
    size_t used_ = 0;
};

} // namespace

static void task_completed(::xkb_runtime * R, Task & T);

struct xkb_runtime {
    Format formats[256];
    int next_fmtid = 1;
    xkb::PoolArray<Task> pending;                     // bodies get Task *
    xkb::PoolArray<uint8_t> args_pool;                // argument bytes, 16-byte aligned per task
    xkb::PoolArray<xkrt_access_t> acc_pool;
    xkb::PoolArray<void *> replica_pool;              // sized to acc_pool at wait
    xkb::PoolArray<xkb_access_rec_t> recs;            // one record per access, same index (wait)
    std::atomic<bool> in_wait{false};
    // background resolution: with fixed pools, a worker thread resolves chunks of spawned tasks
    // on the GPU while the program keeps spawning (the reference resolves at spawn time too)
    bool bg = false;
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    size_t handed = 0, handed_acc = 0;                // tasks / accesses handed to the worker
    std::deque<std::pair<size_t, size_t>> hand_q;     // ends (tasks, accesses) of the hand-overs not yet claimed
    size_t claimed = 0, done = 0;                     // tasks the worker took / finished
    bool stop = false;
    int bg_rc = XKB_OK;
    std::string bg_err;                               // the worker's error text
    int device = 0;
    size_t chunk = 0;                                 // accesses per resolver batch
    xkb_resolver_t * res = nullptr;                   // resolver of the batch being spawned
    bool res_stale = false;                           // res still holds the previous batch
    // page prefaulting of the spawn pools: a helper thread keeps the pages the next spawns will
    // fill backed, so the spawning thread does not take the page faults
    std::thread prefaulter[3];                        // one per pool: tasks, argument bytes, accesses
    std::atomic<size_t> pf_want{0};                   // spawned tasks the pools should be ready for
    std::atomic<bool> pf_stop{false};
    // dataflow execution of non-fused batches: a team of host threads, one CUDA stream each;
    // the planner (coherency decisions and their copies) is used by one task at a time
    std::vector<cudaStream_t> wstreams;
    std::mutex plan_mu;
    // page-locked prefix of the args pool (the descriptor upload of fused batches reads it; one
    // registration per growth, and an upload never spans two of them)
    size_t args_pinned = 0;
    std::vector<std::pair<void *, size_t>> pinned_ranges;
    std::map<uint64_t, uint64_t> user_pinned;         // page-locked pieces of registered memory: start -> end
    std::atomic<bool> args_dense{true};               // every task's args: one descriptor, back to back
    // streaming: while the program spawns, the worker hands each resolved window of a batch made
    // only of built-in device tasks to the GPU (coherency, descriptors, one persistent launch)
    size_t streamed = 0;                              // tasks [0, streamed) are on the GPU
    bool stream_ok = true;                            // the batch can still be streamed
    bool stream_on = true;                            // XKB_STREAM=0 turns streaming off
    xkb_edge_mark_t rest_mark{};                      // edge mark at task `streamed` once streaming stopped
    RecordSet dset;                                   // distinct records of the batch made coherent so far
    xkb_handles::Map hmap;                            // handle states of the batch (concurrent-mode accesses)
    std::vector<xkb_handles::Access> hacc;            //   a spawn's handle accesses
    std::vector<uint64_t> hextra;                     //   handles that get an extra writer task before it
    std::vector<uint32_t> dfirst;                     //   their first occurrences, in record order
    uint64_t cur_h2d = 0, cur_d2h = 0, cur_h2d_bytes = 0, cur_d2h_bytes = 0;   // copies of the batch in progress
    uint64_t cur_d2d = 0;                             // device-to-device copies (reference mode)
    uint64_t copy_calls = 0;                          // run_copies calls that issued copies (under plan_mu)
    // page-locked descriptor slots of streamed windows (a slot is reused once its copy is done)
    struct DescSlot { xkb_task_desc_t * p = nullptr; size_t cap = 0; cudaEvent_t ev = nullptr; } dslot[2];
    int dslot_next = 0;
    bool preplanned = false;                          // the batch's accesses were made coherent up front
    std::atomic<struct Dataflow *> df{nullptr};       // the batch being executed (detached completion)
    uint64_t last_base = 0, last_end = 0;             // region of the last mirror lookup
    uint8_t * last_mirror = nullptr;
    std::map<uint64_t, Region> regions;               // host base -> region
    xkb_planner_t * planner = nullptr;
    xkb_sched_t * sched = nullptr;
    cudaStream_t stream = nullptr;
    bool gpu = false;
    std::atomic<int> status{XKB_OK};                 // first failure recorded (any thread)
    uint64_t last_tasks = 0, last_edges = 0, last_h2d = 0, last_d2h = 0, last_h2d_bytes = 0, last_d2h_bytes = 0;
    int last_fused = 0;
    double last_ms[4] = {0, 0, 0, 0};                 // resolve, coherency + launch prep, run, write-back
    int dummy_team = 0;
    Device devices[2] = {{0}, {1}};                   // the host, the GPU
    Driver drivers[2] = {{XKRT_DRIVER_TYPE_HOST, -1, &devices[0]}, {XKRT_DRIVER_TYPE_CUDA, 0, &devices[1]}};
    xkrt_task_format_id_t fmt_file[2] = {0, 0};       // file read / write tasks
    bool any_unified = false;
    // XKB_PLANNER=reference: the reference's coherency decisions (per-access device allocations,
    // H2D / D2D / D2H as its memory tree plans them) on the tasks run one at a time in spawn order
    bool ref_mode = false;
    std::vector<void *> allocs;                       //   device memory of each planner allocation
    uint64_t budget = 0;                              //   XKB_DEVICE_BUDGET: one region the allocations share,
    uint8_t * budget_base = nullptr;                  //   evicting old ones when a new one does not fit
    FILE * plan_record = nullptr;                     // XKB_PLAN_RECORD: every executed copy record
    // registration-overflow protection (reference mode; XKAAPI_MEMORY_REGISTER_PROTECT_OVERFLOW=0
    // turns it off, as in the reference): (un)registrations, applied to the planner before the
    // fetches of the task spawned next after the call, in spawn order
    bool protect_overflow = true;
    struct RegEvent { size_t before; bool reg; uint64_t ptr, size; };
    std::vector<RegEvent> reg_events;
    size_t reg_next = 0;
    void * cxx_rt = nullptr;                          // the C++ runtime_t bodies of C++ tasks receive
    bool cxx_task_first = false;                      // XKB_CXX_HOST_BODY=task: host bodies of C++ tasks get the task first
};

static xkb_runtime * RT(xkrt_runtime_t * r) { return (xkb_runtime *) r; }

// Records the runtime's first failure (xkb_runtime_status; xkrt_deinit returns it). With
// XKB_TRACE_ERRORS set, the failure's text is printed on stderr when it is recorded -- programs
// written for the reference only see the status.
static void fail(xkb_runtime * R, int rc)
{
    int ok = XKB_OK;
    if (R && rc != XKB_OK && R->status.compare_exchange_strong(ok, rc) && getenv("XKB_TRACE_ERRORS"))
        fprintf(stderr, "[xkrt] error %d: %s\n", rc, xkb_last_error());
}

// The prefault helpers (one per spawn pool): while the program spawns, they fault in the pages
// of the next PREFAULT_AHEAD tasks (argument bytes and two accesses per task assumed; more only
// means later faults), so that spawning itself takes no page faults. Nothing is populated before
// the first spawns, and pages stay backed for the next batch.
constexpr size_t PREFAULT_AHEAD = size_t(1) << 20;

static void prefault_loop(xkb_runtime * R, int pool)
{
    const size_t per_task = pool == 0 ? sizeof(Task) : pool == 1 ? 80 : 2 * sizeof(xkrt_access_t);
    constexpr size_t STEP = size_t(8) << 20;
    size_t done = 0;
    while (!R->pf_stop.load(std::memory_order_relaxed))
    {
        const size_t want = R->pf_want.load(std::memory_order_relaxed) * per_task;
        if (want <= done)
        {
            std::this_thread::sleep_for(std::chrono::microseconds(200));
            continue;
        }
        const size_t to = std::min(want, done + STEP);
        const size_t got = pool == 0 ? R->pending.populate(done, to) : pool == 1 ? R->args_pool.populate(done, to)
                                                                          : R->acc_pool.populate(done, to);
        if (got <= done) { std::this_thread::sleep_for(std::chrono::microseconds(200)); continue; }   // reservation full
        done = got;
    }
}

// File I/O task body (src/file/readwrite.cc:60-90 submits the same read or write as an io_uring
// command): pread / pwrite of the task's slice of the buffer at the same offset of the file.
struct FileArgs { int fd; int write; size_t offset; void * buffer; size_t size; };

static void file_body(xkrt_runtime_t * runtime, xkrt_device_t * device, xkrt_task_t * task)
{
    (void) device;
    FileArgs a;
    memcpy(&a, xkrt_task_args(task), sizeof(a));
    size_t done = 0;
    while (done < a.size)
    {
        char * p = (char *) a.buffer + done;
        const ssize_t k = a.write ? pwrite(a.fd, p, a.size - done, (off_t) (a.offset + done))
                                  : pread(a.fd, p, a.size - done, (off_t) (a.offset + done));
        if (k < 0 && errno == EINTR) continue;
        if (k <= 0)
        {
            fail(RT(runtime), xkb_set_error(XKB_EINVAL, "file %s: %zu of %zu bytes at offset %zu (%s)", a.write ? "write" : "read", done,
                                             a.size, a.offset, k < 0 ? strerror(errno) : "end of file"));
            return;
        }
        done += (size_t) k;
    }
}

static void register_file_formats(xkb_runtime * R)
{
    for (int w = 0; w < 2; ++w)
    {
        const int id = R->next_fmtid++;
        R->formats[id].used = true;
        R->formats[id].label = w ? "file_write_async" : "file_read_async";
        R->formats[id].f[XKRT_TASK_FORMAT_TARGET_HOST] = (xkrt_task_format_func_t) file_body;
        R->fmt_file[w] = (xkrt_task_format_id_t) id;
    }
}

extern "C" int xkrt_init(xkrt_runtime_t ** out)
{
    if (!out) return xkb_set_error(XKB_EINVAL, "xkrt_init: null output");
    xkb_runtime * R = new (std::nothrow) xkb_runtime();
    if (!R) return xkb_set_error(XKB_ENOMEM, "xkrt_init: out of host memory");
    int n = 0;
    R->gpu = cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
    if (R->gpu) cudaGetDevice(&R->device);
    R->drivers[1].ordinal = R->device;
    R->chunk = RESOLVE_CHUNK;
    if (const char * e = getenv("XKB_STREAM")) R->stream_on = atoi(e) != 0;
    if (const char * e = getenv("XKB_CXX_HOST_BODY")) R->cxx_task_first = strcmp(e, "task") == 0;
    if (const char * e = getenv("XKB_PLANNER")) R->ref_mode = strcmp(e, "reference") == 0;
    if (R->ref_mode) R->stream_on = false;
    if (const char * e = getenv("XKB_DEVICE_BUDGET"))
    {
        char * end = nullptr;
        double v = strtod(e, &end);
        if (end && (*end == 'k' || *end == 'K')) v *= 1024.0;
        else if (end && (*end == 'm' || *end == 'M')) v *= 1024.0 * 1024.0;
        else if (end && (*end == 'g' || *end == 'G')) v *= 1024.0 * 1024.0 * 1024.0;
        R->budget = v > 0 ? (uint64_t) v : 0;
    }
    if (const char * e = getenv("XKB_PLAN_RECORD")) R->plan_record = fopen(e, "wb");
    if (const char * e = getenv("XKAAPI_MEMORY_REGISTER_PROTECT_OVERFLOW")) R->protect_overflow = atoi(e) != 0;
    if (const char * c = getenv("XKB_RESOLVE_CHUNK"))      // smaller batches (tests, memory-tight hosts)
        R->chunk = std::max<size_t>(16, strtoull(c, nullptr, 10));
    // fixed pools (address space only; pages are backed when touched) let a worker thread read
    // spawned tasks while spawning continues; without them resolution waits for xkrt_task_wait
    {
        constexpr size_t MAXT = size_t(1) << 28, MAXA = size_t(1) << 29;
        const bool fixed = R->pending.reserve_fixed(MAXT) && R->args_pool.reserve_fixed(MAXT * 64) &&
                           R->acc_pool.reserve_fixed(MAXA) && R->recs.reserve_fixed(MAXA) && R->replica_pool.reserve_fixed(MAXA);
        if (!fixed) { R->pending.release(); R->args_pool.release(); R->acc_pool.release(); R->recs.release(); R->replica_pool.release(); }
        R->bg = R->gpu && fixed;
        if (const char * e = getenv("XKB_BACKGROUND")) if (atoi(e) == 0) R->bg = false;   // resolution at the wait
    }
    if (R->pending.fixed())
    {
        R->pf_want = 0;                            // nothing is populated before the first spawns
        for (int k = 0; k < 3; ++k) R->prefaulter[k] = std::thread(prefault_loop, R, k);
    }
    register_file_formats(R);
    int rc = R->ref_mode ? xkb_planner_create(&R->planner) : xkb_planner_create_resident(&R->planner);
    // the reference's write-back may copy a stale view to the host; the runtime copies coherent data
    if (rc == XKB_OK && R->ref_mode) rc = xkb_planner_set_writeback_coherent(R->planner, 1);
    if (rc == XKB_OK && R->ref_mode && R->budget)
    {
        if ((rc = xkb_planner_set_device_budget(R->planner, R->budget)) == XKB_OK && R->gpu &&
            cudaMalloc((void **) &R->budget_base, R->budget) != cudaSuccess)
            rc = xkb_set_error(XKB_ENOMEM, "xkrt_init: device budget of %llu bytes", (unsigned long long) R->budget);
    }
    if (rc == XKB_OK && R->gpu)
    {
        if (cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_init: stream");
        else rc = xkb_sched_create(&R->sched, R->stream);
    }
    if (rc == XKB_OK && R->bg)
    {
        // the working memory of one background batch (about R->chunk accesses: twice as many
        // resolver ops, up to half as many tasks), reserved here rather than while the program spawns
        if ((rc = xkb_resolver_create(&R->res, R->stream)) == XKB_OK) rc = xkb_internal_resolver_prepare(R->res, 2 * R->chunk);
        if (rc == XKB_OK) rc = xkb_internal_sched_reserve(R->sched, R->chunk / 2 + R->chunk / 8 + 64);
        for (auto & d : R->dslot)
        {
            if (rc != XKB_OK) break;
            const size_t c = R->chunk / 2 + R->chunk / 8 + 64;
            if (cudaHostAlloc((void **) &d.p, c * sizeof(xkb_task_desc_t), cudaHostAllocDefault) != cudaSuccess)
                rc = xkb_set_error(XKB_ENOMEM, "xkrt_init: page-locked descriptor slots");
            else d.cap = c;
        }
    }
    if (rc)
    {
        R->pf_stop = true;
        for (auto & th : R->prefaulter) if (th.joinable()) th.join();
        if (R->res) xkb_resolver_destroy(R->res);
        if (R->sched) xkb_sched_destroy(R->sched);
        for (auto & d : R->dslot) if (d.p) cudaFreeHost(d.p);
        if (R->stream) cudaStreamDestroy(R->stream);
        if (R->planner) xkb_planner_destroy(R->planner);
        delete R;
        return rc;
    }
    *out = (xkrt_runtime_t *) R;
    return XKB_OK;
}

extern "C" int xkrt_deinit(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return xkb_set_error(XKB_EINVAL, "xkrt_deinit: null runtime");
    if (!R->pending.empty()) xkrt_task_wait(runtime);
    if (R->worker.joinable())
    {
        { std::lock_guard<std::mutex> lk(R->mu); R->stop = true; }
        R->cv.notify_all();
        R->worker.join();
    }
    if (R->res) { xkb_resolver_destroy(R->res); R->res = nullptr; }
    R->pf_stop = true;
    for (auto & th : R->prefaulter) if (th.joinable()) th.join();
    if (R->stream) cudaStreamSynchronize(R->stream);
    for (auto & kv : R->regions)
    {
        if (kv.second.unified) { cudaFree(kv.second.mirror); continue; }
        if (kv.second.mirror) cudaFree(kv.second.mirror);
        if (kv.second.pinned_by_us) cudaFreeHost((void *) kv.first);
    }
    for (cudaStream_t w : R->wstreams) cudaStreamDestroy(w);
    for (auto & r : R->pinned_ranges) cudaHostUnregister(r.first);
    for (auto & r : R->user_pinned) cudaHostUnregister((void *) r.first);
    for (auto & d : R->dslot) { if (d.ev) cudaEventDestroy(d.ev); if (d.p) cudaFreeHost(d.p); }
    if (R->sched) xkb_sched_destroy(R->sched);
    if (R->planner) xkb_planner_destroy(R->planner);
    if (R->budget_base) cudaFree(R->budget_base);
    else for (void * p : R->allocs) if (p) cudaFree(p);
    if (R->plan_record) fclose(R->plan_record);
    if (R->stream) cudaStreamDestroy(R->stream);
    const int st = R->status;
    delete R;
    return st;
}

static void bg_finish(xkb_runtime * R);
static void bg_wait_done(xkb_runtime * R);
static int apply_registrations(xkb_runtime * R, size_t upto);

extern "C" void xkrt_reset(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return;
    if (R->worker.joinable()) bg_wait_done(R);
    if (R->streamed && R->sched) xkb_internal_sched_windows_wait(R->sched, nullptr);   // windows already on the GPU finish
    bg_finish(R);
    R->pending.clear(); R->args_pool.clear(); R->acc_pool.clear(); R->replica_pool.clear(); R->recs.clear();
    R->args_dense = true;
    R->cur_h2d = R->cur_d2h = R->cur_h2d_bytes = R->cur_d2h_bytes = 0;
    // the coherency state goes too (src/memory/invalidate.cc:66-133 drops the memory controllers
    // and the device memory): the next task fetches every block from the host again. Each wait
    // left the host coherent, so the host holds everything completed tasks wrote.
    if (R->planner)
    {
        if (R->ref_mode) apply_registrations(R, SIZE_MAX);             // registrations outlive the reset
        size_t n = 0;                                                   // copies planned for dropped tasks
        if (xkb_planner_copies(R->planner, nullptr, 0, &n, 0) == XKB_OK && n)
        {
            std::vector<xkb_copy_t> drop(n);
            xkb_planner_copies(R->planner, drop.data(), n, &n, 1);
        }
        if (xkb_planner_invalidate(R->planner) != XKB_OK) fail(R, XKB_EINVAL);
    }
    if (R->ref_mode)
    {
        if (R->gpu) cudaStreamSynchronize(R->stream);
        if (!R->budget_base) for (void * p : R->allocs) if (p) cudaFree(p);
        R->allocs.clear();
    }
}

// Registering memory that overlaps registered memory (the reference's assisted registration,
// src/memory/register.cc:121-166, registers only the pages not registered yet): the union of the
// range and the regions it meets becomes one region, so an access over the union has one mirror.
// The old mirrors' bytes move into the new one; the blocks keep their coherency states.
static int merge_regions(xkb_runtime * R, const std::vector<uint64_t> & over, uint64_t lo, uint64_t hi, bool unified)
{
    if (over.size() == 1)
    {
        const Region & g = R->regions[over[0]];
        if (over[0] == lo && g.size == hi - lo) return XKB_OK;     // inside one region already
    }
    for (uint64_t k : over)
    {
        const Region & g = R->regions[k];
        if (unified || g.unified || g.pinned_by_us)
            return xkb_set_error(XKB_EINVAL, "memory registration: the range overlaps memory the runtime allocated");
    }
    if (!R->pending.empty())
        return xkb_set_error(XKB_EINVAL, "memory registration: the range overlaps registered memory while %zu spawned tasks "
                                         "wait; register it before spawning them or after xkrt_task_wait", R->pending.size());
    int32_t id = -1;
    if (!R->ref_mode)
    {
        const int rc = xkb_planner_replace_regions(R->planner, lo, hi - lo, &id);
        if (rc) return rc;
    }
    void * mirror = nullptr;
    if (R->gpu && !R->ref_mode)
    {
        cudaError_t e = cudaMalloc(&mirror, hi - lo);
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        for (uint64_t k : over)
        {
            const Region & g = R->regions[k];
            if (g.mirror && (e = cudaMemcpyAsync((uint8_t *) mirror + (k - lo), g.mirror, g.size, cudaMemcpyDeviceToDevice,
                                                 R->stream)) != cudaSuccess)
                return xkb_set_cuda_error(e);
        }
        if ((e = cudaStreamSynchronize(R->stream)) != cudaSuccess) return xkb_set_cuda_error(e);
        for (uint64_t k : over) if (R->regions[k].mirror) cudaFree(R->regions[k].mirror);
    }
    for (uint64_t k : over) R->regions.erase(k);
    R->regions[lo] = Region{hi - lo, mirror, false, id, false};
    R->last_base = R->last_end = 0; R->last_mirror = nullptr;     // the lookup hint may name a freed mirror
    return XKB_OK;
}

static int add_region(xkb_runtime * R, void * ptr, size_t size, bool pinned, bool unified = false)
{
    std::lock_guard<std::mutex> lk(R->plan_mu);       // the worker may be streaming a window
    {
        const uint64_t b = (uint64_t) ptr, e = b + size;
        uint64_t lo = b, hi = e;
        std::vector<uint64_t> over;
        auto it = R->regions.upper_bound(b);
        if (it != R->regions.begin()) { auto p = std::prev(it); if (p->first + p->second.size > b) it = p; }
        for (; it != R->regions.end() && it->first < e; ++it)
        {
            over.push_back(it->first);
            lo = std::min(lo, it->first); hi = std::max(hi, it->first + it->second.size);
        }
        if (!over.empty()) return merge_regions(R, over, lo, hi, unified);
    }
    int32_t id = -1;
    int rc = R->ref_mode ? XKB_OK : xkb_planner_add_region(R->planner, (uint64_t) ptr, size, &id);
    if (rc) return rc;
    void * mirror = unified ? ptr : nullptr;          // unified memory: the device uses it in place
    if (R->gpu && !unified && !R->ref_mode)           // reference mode: per-access allocations instead
    {
        cudaError_t e = cudaMalloc(&mirror, size);
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
    }
    R->regions[(uint64_t) ptr] = Region{size, mirror, pinned, id, unified};
    R->any_unified = R->any_unified || unified;
    return XKB_OK;
}

// Reference mode: the registration reaches the planner before the fetches of the next task
// spawned (the tasks spawned before it were fetched first under the canonical schedule).
static void note_registration(xkb_runtime * R, bool reg, void * ptr, size_t size)
{
    if (!R->ref_mode || !R->protect_overflow || !size) return;
    std::lock_guard<std::mutex> lk(R->plan_mu);
    R->reg_events.push_back({R->pending.size(), reg, (uint64_t) ptr, (uint64_t) size});
}

// Registrations noted before task `upto` (every one with upto = SIZE_MAX) into the planner.
static int apply_registrations(xkb_runtime * R, size_t upto)
{
    int rc = XKB_OK;
    while (rc == XKB_OK && R->reg_next < R->reg_events.size() && R->reg_events[R->reg_next].before <= upto)
    {
        const auto & e = R->reg_events[R->reg_next++];
        rc = e.reg ? xkb_planner_register(R->planner, e.ptr, e.size) : xkb_planner_unregister(R->planner, e.ptr, e.size);
    }
    if (R->reg_next == R->reg_events.size()) { R->reg_events.clear(); R->reg_next = 0; }
    return rc;
}

extern "C" int xkrt_memory_register(xkrt_runtime_t * runtime, void * ptr, size_t size)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !ptr || !size) return xkb_set_error(XKB_EINVAL, "xkrt_memory_register: bad arguments");
    if (R->gpu)
    {
        // page-lock the range (faster copies): the pages of [ptr, ptr + size) and of every locked
        // piece they meet or touch become ONE locked piece -- the driver refuses a range sharing a
        // page with a locked one. Tasks in flight may be copying from the pieces met, so then
        // only a range that meets none is locked. Copies never run across a piece's end
        // (run_copies splits them), so partly locked memory is safe either way.
        std::lock_guard<std::mutex> lk(R->plan_mu);
        static const uint64_t page = (uint64_t) sysconf(_SC_PAGESIZE);
        const uint64_t b = (uint64_t) ptr, e = b + size;
        uint64_t lo = b - b % page, hi = (e + page - 1) / page * page;
        std::vector<uint64_t> meet;
        auto it = R->user_pinned.upper_bound(lo);
        if (it != R->user_pinned.begin() && std::prev(it)->second >= lo) it = std::prev(it);
        for (; it != R->user_pinned.end() && it->first <= hi; ++it)
        {
            meet.push_back(it->first);
            lo = std::min(lo, it->first); hi = std::max(hi, it->second);
        }
        const bool covered = meet.size() == 1 && meet[0] <= b - b % page && R->user_pinned[meet[0]] >= e;
        if (!covered && (meet.empty() || R->pending.empty()))
        {
            for (uint64_t m : meet) { cudaHostUnregister((void *) m); R->user_pinned.erase(m); }
            if (cudaHostRegister((void *) lo, hi - lo, cudaHostRegisterDefault) == cudaSuccess) R->user_pinned[lo] = hi;
            cudaGetLastError();
        }
    }
    note_registration(R, true, ptr, size);
    return add_region(R, ptr, size, false);
}

extern "C" int xkrt_memory_unregister(xkrt_runtime_t * runtime, void * ptr, size_t size)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !ptr) return xkb_set_error(XKB_EINVAL, "xkrt_memory_unregister: bad arguments");
    if (R->gpu)
    {
        // unlock the page-locked pieces inside the range (the mirror stays until xkrt_deinit)
        std::lock_guard<std::mutex> lk(R->plan_mu);
        static const uint64_t page = (uint64_t) sysconf(_SC_PAGESIZE);
        const uint64_t b = (uint64_t) ptr - (uint64_t) ptr % page, e = ((uint64_t) ptr + size + page - 1) / page * page;
        for (auto it = R->user_pinned.lower_bound(b); it != R->user_pinned.end() && it->second <= e;)
        {
            cudaHostUnregister((void *) it->first);
            cudaGetLastError();
            it = R->user_pinned.erase(it);
        }
    }
    note_registration(R, false, ptr, size);
    return XKB_OK;
}

extern "C" void * xkrt_memory_host_allocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, size_t size)
{
    xkb_runtime * R = RT(runtime);
    (void) device;
    if (!R || !size) return nullptr;
    void * p = nullptr;
    if (R->gpu) { if (cudaMallocHost(&p, size) != cudaSuccess) { fail(R, XKB_ENOMEM); return nullptr; } }
    else { p = aligned_alloc(4096, (size + 4095) & ~(size_t) 4095); if (!p) { fail(R, XKB_ENOMEM); return nullptr; } }
    int rc = add_region(R, p, size, R->gpu);
    if (rc) { fail(R, rc); return nullptr; }
    return p;
}

extern "C" void xkrt_memory_host_deallocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, void * ptr, size_t size)
{
    (void) runtime; (void) device; (void) ptr; (void) size;   // released by xkrt_deinit
}

extern "C" unsigned int xkrt_get_ndevices(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    return R ? (R->gpu ? 2u : 1u) : 0u;
}

extern "C" unsigned int xkrt_get_ndevices_max(xkrt_runtime_t * runtime)
{
    return xkrt_get_ndevices(runtime);           // one host and (at most) one GPU
}

extern "C" int xkrt_memory_register_async(xkrt_runtime_t * runtime, void * ptr, size_t size)
{
    return xkrt_memory_register(runtime, ptr, size);
}

extern "C" int xkrt_memory_unregister_async(xkrt_runtime_t * runtime, void * ptr, size_t size)
{
    return xkrt_memory_unregister(runtime, ptr, size);
}

extern "C" void * xkrt_memory_unified_allocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, size_t size)
{
    xkb_runtime * R = RT(runtime);
    (void) device;
    if (!R || !size) return nullptr;
    if (!R->gpu) { fail(R, xkb_set_error(XKB_ENODEV, "xkrt_memory_unified_allocate: no GPU")); return nullptr; }
    void * p = nullptr;
    if (cudaMallocManaged(&p, size) != cudaSuccess) { cudaGetLastError(); fail(R, XKB_ENOMEM); return nullptr; }
    int rc = add_region(R, p, size, false, true);
    if (rc) { cudaFree(p); fail(R, rc); return nullptr; }
    return p;
}

extern "C" void xkrt_memory_unified_deallocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, void * ptr, size_t size)
{
    (void) runtime; (void) device; (void) ptr; (void) size;   // released by xkrt_deinit
}

extern "C" xkrt_driver_t * xkrt_driver_get(xkrt_runtime_t * runtime, xkrt_driver_type_t type)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return nullptr;
    if (type == XKRT_DRIVER_TYPE_HOST) return (xkrt_driver_t *) &R->drivers[0];
    if (type == XKRT_DRIVER_TYPE_CUDA && R->gpu) return (xkrt_driver_t *) &R->drivers[1];
    return nullptr;
}

extern "C" xkrt_device_t * xkrt_device_get(xkrt_runtime_t * runtime, xkrt_device_global_id_t device)
{
    xkb_runtime * R = RT(runtime);
    if (!R || device >= xkrt_get_ndevices(runtime)) return nullptr;
    return (xkrt_device_t *) &R->devices[device];
}

extern "C" xkrt_driver_t * xkrt_device_driver_get(xkrt_runtime_t * runtime, xkrt_device_t * device)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !device) return nullptr;
    return (xkrt_driver_t *) &R->drivers[((Device *) device)->global_id == 0 ? 0 : 1];
}

extern "C" xkrt_device_driver_id_t xkrt_device_driver_id_get(xkrt_runtime_t * runtime, xkrt_device_t * device)
{
    (void) runtime; (void) device;
    return 0;                                    // the first (only) device of its driver
}

extern "C" xkrt_task_t * xkrt_task_current(xkrt_runtime_t * runtime)
{
    (void) runtime;
    return (xkrt_task_t *) g_current;
}

extern "C" void xkrt_task_detachable_incr(xkrt_runtime_t * runtime, xkrt_task_t * task)
{
    (void) runtime;
    if (task) __atomic_add_fetch(&((Task *) task)->detach, 1, __ATOMIC_ACQ_REL);
}

// Any thread may drop the reference that completes a task; its successors are released then
// (src/task.cc:260-270, __task_detachable_decr).
extern "C" void xkrt_task_detachable_decr(xkrt_runtime_t * runtime, xkrt_task_t * task)
{
    (void) runtime;
    if (task && task_unref(*(Task *) task)) task_completed(((Task *) task)->rt, *(Task *) task);
}

// Complete a task now, whatever references it still holds (src/task.cc:405-412).
extern "C" void xkrt_task_complete(xkrt_runtime_t * runtime, xkrt_task_t * task)
{
    (void) runtime;
    if (task && __atomic_exchange_n(&((Task *) task)->detach, 0, __ATOMIC_ACQ_REL) > 0) task_completed(((Task *) task)->rt, *(Task *) task);
}

// Tasks of the spawn calls are committed when spawned; a task built by hand with the C++ source
// API (include/xkrt/task/task.hpp) is committed here (api/c/src/xkrt.cc:278-285). Anything else
// records XKB_EINVAL.
extern "C" void xkrt_task_commit(xkrt_runtime_t * runtime, xkrt_task_t * task)
{
    if (task && ((const xkrt::task_t *) task)->magic == xkrt::TASK_MAGIC) { xkb_cxx_commit(runtime, task); return; }
    fail(RT(runtime), xkb_set_error(XKB_EINVAL, "xkrt_task_commit: not a task built with the C++ source API (spawned tasks are committed when spawned)"));
}

// The reference pushes an already ready task to a queue; here a hand-built task is committed (its
// accesses still order it after earlier tasks, which a ready task has no pending ones of).
extern "C" void xkrt_task_enqueue(xkrt_runtime_t * runtime, xkrt_task_t * task)
{
    if (task && ((const xkrt::task_t *) task)->magic == xkrt::TASK_MAGIC) { xkb_cxx_commit(runtime, task); return; }
    fail(RT(runtime), xkb_set_error(XKB_EINVAL, "xkrt_task_enqueue: tasks are scheduled by xkrt_task_wait"));
}

static void logger(const char * level, const char * msg) { fprintf(stderr, "[xkrt] %s: %s\n", level, msg ? msg : ""); }
extern "C" void xkrt_logger_info (const char * msg) { logger("info", msg); }
extern "C" void xkrt_logger_debug(const char * msg) { logger("debug", msg); }
extern "C" void xkrt_logger_warn (const char * msg) { logger("warn", msg); }
extern "C" void xkrt_logger_error(const char * msg) { logger("error", msg); }
extern "C" void xkrt_logger_fatal(const char * msg) { logger("fatal", msg); abort(); }   // the reference's contract

extern "C" xkrt_task_format_id_t xkrt_task_format_put(xkrt_runtime_t * runtime, const char * label)
{
    xkb_runtime * R = RT(runtime);
    if (!R || R->next_fmtid >= 256) { fail(R, XKB_ERANGE); return XKRT_TASK_FORMAT_NULL; }
    const int id = R->next_fmtid++;
    R->formats[id].used = true;
    R->formats[id].label = label ? label : "";
    return (xkrt_task_format_id_t) id;
}

extern "C" int xkrt_task_format_set(xkrt_runtime_t * runtime, xkrt_task_format_id_t fmtid, xkrt_task_format_target_t target,
                                    xkrt_task_format_func_t func)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !R->formats[fmtid].used || target < 0 || target >= XKRT_TASK_FORMAT_TARGET_MAX)
        return xkb_set_error(XKB_EINVAL, "xkrt_task_format_set: bad format or target");
    R->formats[fmtid].f[target] = func;
    return XKB_OK;
}

extern "C" xkrt_task_format_id_t xkb_task_format_builtin(xkrt_runtime_t * runtime, int kind)
{
    xkb_runtime * R = RT(runtime);
    if (!R || (kind != XKB_TASK_HEAT_F64 && kind != XKB_TASK_HEAT_F32 && kind != XKB_TASK_AXPBY)) { fail(R, XKB_EINVAL); return 0; }
    xkrt_task_format_id_t id = xkrt_task_format_put(runtime, "builtin");
    if (id) R->formats[id].builtin = kind;
    return id;
}

extern "C" int xkb_runtime_status(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return XKB_EINVAL;
    return R->status.exchange(XKB_OK);
}

extern "C" void * xkb_runtime_stream(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return nullptr;
    return (void *) (g_stream ? g_stream : R->stream);      // inside a CUDA body: its worker's stream
}

extern "C" int xkb_runtime_last_wait(xkrt_runtime_t * runtime, uint64_t * tasks, uint64_t * edges, uint64_t * h2d,
                                     uint64_t * d2h, int * fused)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return xkb_set_error(XKB_EINVAL, "xkb_runtime_last_wait: null runtime");
    if (tasks) *tasks = R->last_tasks;
    if (edges) *edges = R->last_edges;
    if (h2d) *h2d = R->last_h2d;
    if (d2h) *d2h = R->last_d2h;
    if (fused) *fused = R->last_fused;
    return XKB_OK;
}

// ---- spawn -----------------------------------------------------------------------------------

static void bg_hand_over(xkb_runtime * R, bool final);

static inline void copy64(void * dst, const void * src)
{
    struct B64 { unsigned char b[64]; };
    *(B64 *) dst = *(const B64 *) src;
}

static void spawn_task(xkb_runtime * R, xkrt_device_global_id_t device, xkrt_task_flag_bitfield_t flags, xkrt_task_format_id_t fmtid,
                       const void * args, size_t args_size, const xkrt_access_t * acc, size_t nacc, xkrt_task_func_t func, void * ud,
                       void * cxx = nullptr, int detach0 = 0);

// cxx: the task_t of a C++ task (its body receives it); detach0: the detachable counter's
// initial value (the task completes once its body returned and the counter is back to 0)
static void spawn(xkb_runtime * R, xkrt_device_global_id_t device, xkrt_task_flag_bitfield_t flags, xkrt_task_format_id_t fmtid,
                  const void * args, size_t args_size, const xkrt_access_t * acc, size_t nacc, xkrt_task_func_t func, void * ud,
                  void * cxx = nullptr, int detach0 = 0)
{
    if (!R) return;
    if (nacc && !acc) { fail(R, xkb_set_error(XKB_EINVAL, "spawn: null accesses")); return; }
    bool handles = false;
    for (size_t i = 0; i < nacc; ++i)
    {
        if (acc[i].type == ACCESS_TYPE_HANDLE) handles = true;
        else if (acc[i].concurrency == ACCESS_CONCURRENCY_CONCURRENT)    // asserted away in access.hpp:500-502
        { fail(R, xkb_set_error(XKB_EINVAL, "spawn: concurrent mode applies to handle accesses only")); return; }
    }
    if (args_size && !args) { fail(R, xkb_set_error(XKB_EINVAL, "spawn: null arguments")); return; }
    if (R->in_wait) { fail(R, xkb_set_error(XKB_EINVAL, "spawn: spawning from a task body during xkrt_task_wait is not supported")); return; }
    if (handles)
    {
        // the handle map's extra empty writer tasks go first, each with one sequential VW access
        // of its handle (dependency-map.hpp:93-137)
        R->hacc.clear(); R->hextra.clear();
        for (size_t i = 0; i < nacc; ++i)
            if (acc[i].type == ACCESS_TYPE_HANDLE)
                R->hacc.push_back({(uint64_t) (uintptr_t) acc[i].region.handle.addr, (uint8_t) acc[i].mode, (int) acc[i].concurrency});
        const char * why = "";
        if (R->hmap.task(R->hacc.data(), R->hacc.size(), false, R->hextra, &why))
        { fail(R, xkb_set_error(XKB_EINVAL, "spawn: %s", why)); return; }
        for (uint64_t h : R->hextra)
        {
            xkrt_access_t e;
            memset(&e, 0, sizeof(e));
            e.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; e.mode = ACCESS_MODE_VW; e.scope = ACCESS_SCOPE_NONUNIFIED;
            e.type = ACCESS_TYPE_HANDLE; e.region.handle.addr = (void *) (uintptr_t) h;
            spawn_task(R, HOST_DEVICE_GLOBAL_ID, 0, XKRT_TASK_FORMAT_NULL, nullptr, 0, &e, 1, nullptr, nullptr);
        }
    }
    spawn_task(R, device, flags, fmtid, args, args_size, acc, nacc, func, ud, cxx, detach0);
}

// Append one task to the batch (arguments already checked).
static void spawn_task(xkb_runtime * R, xkrt_device_global_id_t device, xkrt_task_flag_bitfield_t flags, xkrt_task_format_id_t fmtid,
                       const void * args, size_t args_size, const xkrt_access_t * acc, size_t nacc, xkrt_task_func_t func, void * ud,
                       void * cxx, int detach0)
{
    Task t;
    t.rt = R; t.fmtid = fmtid; t.flags = flags; t.device = device;
    t.detach = detach0;
    t.nargs = (uint32_t) args_size; t.nacc = (uint32_t) nacc;
    t.args_off = (R->args_pool.size() + 15) & ~(size_t) 15;
    t.acc_off = R->acc_pool.size();
    t.func = func; t.user_data = cxx ? cxx : ud;       // C++ tasks have no func
    
    const size_t args_end = args_size ? t.args_off + args_size : R->args_pool.size();
    if (!R->args_pool.resize(args_end) || !R->acc_pool.resize(t.acc_off + nacc) || !R->pending.push_back(t))
    {
        fail(R, xkb_set_error(XKB_ENOMEM, "spawn: out of host memory"));
        return;
    }
    for (size_t k = 0; k < nacc; ++k) R->acc_pool[t.acc_off + k] = acc[k];
    if (cxx)
    {
        ((xkrt::task_t *) cxx)->impl = R->pending.size() - 1;
        ((xkrt::task_t *) cxx)->state.value = xkrt::TASK_STATE_READY;
    }
    if (args_size == sizeof(xkb_task_desc_t)) copy64(R->args_pool.data() + t.args_off, args);   // a descriptor: fixed-size copy
    else if (args_size) memcpy(R->args_pool.data() + t.args_off, args, args_size);
    const size_t nt = R->pending.size();
    if (args_size != sizeof(xkb_task_desc_t) || t.args_off != (nt - 1) * sizeof(xkb_task_desc_t)) R->args_dense = false;
    if ((nt & 4095) == 0 && R->prefaulter[0].joinable()) R->pf_want.store(nt + PREFAULT_AHEAD, std::memory_order_relaxed);
    // hand over once a batch's worth of accesses is spawned (the same test as bg_hand_over's,
    // inlined: the spawn loop runs it every time)
    if (R->bg && R->acc_pool.size() - R->handed_acc >= (R->handed ? R->chunk : std::max<size_t>(16, R->chunk / 32)))
        bg_hand_over(R, false);
}

extern "C" void xkrt_task_spawn_generic(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                        const xkrt_task_flag_bitfield_t flags, const xkrt_task_format_id_t fmtid,
                                        const void * args, const size_t args_size, const xkrt_access_t * accesses,
                                        const xkrt_task_access_counter_type_t naccesses,
                                        const xkrt_task_access_counter_type_t ocr_access,
                                        const xkrt_task_wait_counter_type_t detachable_counter_initial)
{
    // one GPU: every owner of the ocr access is that GPU, so the placement hint changes nothing
    (void) ocr_access;
    spawn(RT(runtime), device_global_id, flags, fmtid, args, args_size, accesses, naccesses, nullptr, nullptr, nullptr,
          (flags & TASK_FLAG_DETACHABLE) ? (int) detachable_counter_initial : 0);
}

extern "C" void xkrt_task_spawn_with_format(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                            const xkrt_task_format_id_t fmtid, const void * args, const size_t args_size)
{
    spawn(RT(runtime), device_global_id, device_global_id ? TASK_FLAG_DEVICE : 0, fmtid, args, args_size, nullptr, 0, nullptr, nullptr);
}

extern "C" void xkrt_task_spawn_with_format_with_accesses(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                                          const xkrt_task_format_id_t fmtid, const void * args,
                                                          const size_t args_size, const xkrt_access_t * accesses,
                                                          const int naccesses)
{
    spawn(RT(runtime), device_global_id, (device_global_id ? TASK_FLAG_DEVICE : 0) | TASK_FLAG_DEPENDENT, fmtid, args,
          args_size, accesses, naccesses > 0 ? (size_t) naccesses : 0, nullptr, nullptr);
}

extern "C" void xkrt_task_spawn(xkrt_runtime_t * runtime, xkrt_task_func_t func, void * user_data)
{
    spawn(RT(runtime), HOST_DEVICE_GLOBAL_ID, 0, 0, nullptr, 0, nullptr, 0, func, user_data);
}

extern "C" xkrt_team_t * xkrt_team_driver_device_get(xkrt_runtime_t * runtime, xkrt_driver_type_t type,
                                                     xkrt_device_driver_id_t device_driver_id)
{
    xkb_runtime * R = RT(runtime);
    (void) device_driver_id;
    if (!R || type != XKRT_DRIVER_TYPE_HOST) return nullptr;
    return (xkrt_team_t *) &R->dummy_team;
}

extern "C" void xkrt_team_task_spawn(xkrt_runtime_t * runtime, xkrt_team_t * team, xkrt_task_func_t func, void * user_data)
{
    (void) team;
    spawn(RT(runtime), HOST_DEVICE_GLOBAL_ID, 0, 0, nullptr, 0, nullptr, 0, func, user_data);
}

extern "C" void xkrt_team_task_spawn_with_accesses(xkrt_runtime_t * runtime, xkrt_team_t * team, xkrt_task_func_t func,
                                                   void * user_data, const xkrt_access_t * accesses, const int naccesses)
{
    (void) team;
    spawn(RT(runtime), HOST_DEVICE_GLOBAL_ID, TASK_FLAG_DEPENDENT, 0, nullptr, 0, accesses, naccesses > 0 ? (size_t) naccesses : 0,
          func, user_data);
}

extern "C" xkrt_team_t * xkrt_team_driver_get(xkrt_runtime_t * runtime, xkrt_driver_type_t type)
{
    return xkrt_team_driver_device_get(runtime, type, 0);
}

extern "C" xkrt_team_t * xkrt_team_driver_get_any(xkrt_runtime_t * runtime, xkrt_driver_type_bitfield_t types)
{
    return (types & (1u << XKRT_DRIVER_TYPE_HOST)) ? xkrt_team_driver_device_get(runtime, XKRT_DRIVER_TYPE_HOST, 0) : nullptr;
}

// Spawn n tasks over [buffer, buffer + size), split as the reference's runtime_t::foreach does
// (include/xkrt/runtime.h:333-352: n = min(n, size) chunks of size / n bytes, the last one takes
// the rest), each reading or writing its slice of the file (src/file/readwrite.cc:104-170). The
// reference declares a virtual write (VW) on the slice, which orders the tasks but moves no data;
// here a read declares W and a write RW: the same dependencies (W and RW order exactly like VW),
// and the buffer is also coherent on the host when the body runs and owned by it after a read.
static int file_async(xkrt_runtime_t * runtime, int fd, void * buffer, size_t size, unsigned int n, int write)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !buffer || fd < 0 || n == 0) return xkb_set_error(XKB_EINVAL, "xkrt_file_%s_async: bad arguments", write ? "write" : "read");
    if (size == 0) return XKB_OK;
    if (size < n) n = (unsigned) size;
    const size_t chunk = size / n;
    const uintptr_t p = (uintptr_t) buffer;
    for (unsigned i = 0; i < n; ++i)
    {
        const uintptr_t a = p + i * chunk, b = i == n - 1 ? p + size : p + (i + 1) * chunk;
        FileArgs f{fd, write, (size_t) (a - p), (void *) a, (size_t) (b - a)};
        xkrt_access_t acc;
        memset(&acc, 0, sizeof(acc));
        acc.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; acc.mode = write ? ACCESS_MODE_RW : ACCESS_MODE_W;
        acc.scope = ACCESS_SCOPE_NONUNIFIED; acc.type = ACCESS_TYPE_SEGMENT;
        acc.region.segment.a = (void *) a; acc.region.segment.b = (void *) b;
        xkrt_task_spawn_with_format_with_accesses(runtime, HOST_DEVICE_GLOBAL_ID, R->fmt_file[write], &f, sizeof(f), &acc, 1);
    }
    return XKB_OK;
}

extern "C" int xkrt_file_read_async(xkrt_runtime_t * runtime, int fd, void * buffer, size_t n, unsigned int nchunks)
{
    return file_async(runtime, fd, buffer, n, nchunks, 0);
}

extern "C" int xkrt_file_write_async(xkrt_runtime_t * runtime, int fd, void * buffer, size_t n, unsigned int nchunks)
{
    return file_async(runtime, fd, buffer, n, nchunks, 1);
}

extern "C" void * xkrt_memory_device_allocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, size_t size)
{
    xkb_runtime * R = RT(runtime);
    if (!R || device > 1 || (device == 1 && !R->gpu)) { fail(R, xkb_set_error(XKB_EINVAL, "xkrt_memory_device_allocate: no device %d", (int) device)); return nullptr; }
    void * p = xkrt_driver_memory_device_allocate((xkrt_driver_t *) &R->drivers[device], 0, size, 0);
    if (!p) fail(R, XKB_ENOMEM);
    return p;
}

extern "C" void xkrt_memory_device_deallocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, void * chunk)
{
    xkb_runtime * R = RT(runtime);
    if (!R || device > 1) { fail(R, XKB_EINVAL); return; }
    xkrt_driver_memory_device_deallocate((xkrt_driver_t *) &R->drivers[device], 0, chunk, 0, 0);
}

// The launcher gets the queue of the host thread running the CUDA body (its stream); the task's
// kernels are complete when the body's task completes (src/sched.cc:469-505 records an event on
// the kernel queue and completes the task from its callback).
extern "C" void xkrt_task_kernel_launch(xkrt_runtime_t * runtime, xkrt_device_t * device, xkrt_task_t * task, int synchronous,
                                        xkrt_kernel_launcher_t launcher)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !launcher) { fail(R, xkb_set_error(XKB_EINVAL, "xkrt_task_kernel_launch: no runtime or launcher")); return; }
    if (!g_stream) { fail(R, xkb_set_error(XKB_EINVAL, "xkrt_task_kernel_launch: called outside a CUDA task body")); return; }
    Queue q{XKRT_DRIVER_TYPE_CUDA, XKRT_QUEUE_TYPE_KERN, R->device, g_stream, false, 0, nullptr};
    launcher(runtime, device, task, &q, nullptr, 0);
    if (synchronous && cudaStreamSynchronize(g_stream) != cudaSuccess) fail(R, xkb_set_cuda_error(cudaGetLastError()));
}

extern "C" int xkrt_device_kernel_launch(xkrt_runtime_t * runtime, xkrt_device_t * device, xkrt_queue_t * queue,
                                         xkrt_queue_command_list_counter_t idx, const xkrt_driver_module_fn_t * fn,
                                         const unsigned int gx, const unsigned int gy, const unsigned int gz, const unsigned int bx,
                                         const unsigned int by, const unsigned int bz, const unsigned int shared_memory_bytes,
                                         void * args, const size_t args_size)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !device || ((Device *) device)->global_id != 1 || !R->gpu)
        return xkb_set_error(XKB_EINVAL, "xkrt_device_kernel_launch: kernels run on the GPU device");
    return xkrt_driver_kernel_launch((xkrt_driver_t *) &R->drivers[1], queue, idx, fn, gx, gy, gz, bx, by, bz, shared_memory_bytes,
                                     args, args_size);
}

// ---- task accessors --------------------------------------------------------------------------

extern "C" void * xkrt_task_args(xkrt_task_t * task)
{
    Task * t = (Task *) task;
    return t && t->nargs ? t->rt->args_pool.data() + t->args_off : nullptr;
}
extern "C" xkrt_access_t * xkrt_task_accesses(xkrt_task_t * task)
{
    Task * t = (Task *) task;
    return t && t->nacc ? t->rt->acc_pool.data() + t->acc_off : nullptr;
}
extern "C" xkrt_access_t * xkrt_task_access(xkrt_task_t * task, xkrt_task_access_counter_type_t i)
{
    Task * t = (Task *) task;
    return t && i < t->nacc ? t->rt->acc_pool.data() + t->acc_off + i : nullptr;
}
extern "C" void * xkrt_task_access_replica(xkrt_task_t * task, xkrt_task_access_counter_type_t i)
{
    Task * t = (Task *) task;
    return t && i < t->nacc && t->acc_off + i < t->rt->replica_pool.size() ? t->rt->replica_pool[t->acc_off + i] : nullptr;
}

// ---- wait --------------------------------------------------------------------------------------

static bool to_rec(const xkrt_access_t & a, uint32_t task, xkb_access_rec_t & r)
{
    memset(&r, 0, sizeof(r));
    r.task = task;
    r.mode = (uint8_t) a.mode;
    if (a.type == ACCESS_TYPE_HANDLE)
    {
        // a concurrent write of a handle is resolved as a read of it (handles.h)
        r.mode = xkb_handles::resolve_mode(r.mode, (int) a.concurrency);
        r.type = XKB_ACCESS_TYPE_HANDLE; r.addr = (uint64_t) a.region.handle.addr;
        return r.addr != ~0ull;
    }
    if (a.type == ACCESS_TYPE_SEGMENT)
    {
        r.type = XKB_ACCESS_TYPE_SEGMENT; r.addr = (uint64_t) a.region.segment.a; r.ld = (uint64_t) a.region.segment.b;
        return r.ld > r.addr;
    }
    if (a.type == ACCESS_TYPE_BLAS_MATRIX)
    {
        const auto & m = a.region.matrix;
        r.type = XKB_ACCESS_TYPE_BLAS_MATRIX; r.addr = (uint64_t) m.addr; r.ld = m.ld; r.offset_m = m.offset_m;
        r.offset_n = m.offset_n; r.m = m.m; r.n = m.n; r.sizeof_type = m.sizeof_type;
        return m.storage == MATRIX_COLMAJOR && m.m && m.n;
    }
    return false;
}

static bool is_device(const xkb_runtime * R, const Task & t)
{
    const Format & f = R->formats[t.fmtid];
    // a device task with no format (XKRT_TASK_FORMAT_NULL) places its data on the device and runs nothing
    return (t.flags & TASK_FLAG_DEVICE) && t.device != HOST_DEVICE_GLOBAL_ID &&
           (f.builtin >= 0 || f.f[XKRT_TASK_FORMAT_TARGET_CUDA] || t.fmtid == XKRT_TASK_FORMAT_NULL);
}

// Last region a lookup hit (consecutive lookups mostly hit the same one).
struct RegionHint { uint64_t base = 0, end = 0; uint8_t * mirror = nullptr; };

static void * mirror_lookup(const xkb_runtime * R, uint64_t host, RegionHint & h)
{
    if (host >= h.base && host < h.end) return h.mirror + (host - h.base);
    auto it = R->regions.upper_bound(host);
    if (it == R->regions.begin()) return nullptr;
    --it;
    if (host >= it->first + it->second.size || !it->second.mirror) return nullptr;
    h.base = it->first; h.end = it->first + it->second.size; h.mirror = (uint8_t *) it->second.mirror;
    return (uint8_t *) it->second.mirror + (host - it->first);
}

// First byte an access record touches.
static uint64_t rec_begin(const xkb_access_rec_t & r)
{
    return r.type == XKB_ACCESS_TYPE_SEGMENT ? r.addr : r.addr + (r.offset_n * r.ld + r.offset_m) * r.sizeof_type;
}

// Is the record's memory unified (used in place by the device, never copied)?
static bool in_unified(const xkb_runtime * R, const xkb_access_rec_t & r)
{
    if (!R->any_unified || r.type == XKB_ACCESS_TYPE_HANDLE) return false;
    const uint64_t b = rec_begin(r);
    auto it = R->regions.upper_bound(b);
    if (it == R->regions.begin()) return false;
    --it;
    return it->second.unified && b < it->first + it->second.size;
}

static void * mirror_of(xkb_runtime * R, uint64_t host)
{
    RegionHint h{R->last_base, R->last_end, R->last_mirror};
    void * p = mirror_lookup(R, host, h);
    R->last_base = h.base; R->last_end = h.end; R->last_mirror = h.mirror;
    return p;
}

// Reference mode: device memory for every allocation the planner made since the last call.
static int ensure_allocs(xkb_runtime * R)
{
    if (R->budget_base)
    {
        // every allocation lives at its offset in the budget (evicted ones keep theirs until reused)
        size_t n = 0;
        int rc = xkb_planner_allocation_offsets(R->planner, nullptr, nullptr, 0, &n);
        if (rc || n <= R->allocs.size()) return rc;
        std::vector<int64_t> off(n);
        if ((rc = xkb_planner_allocation_offsets(R->planner, off.data(), nullptr, n, &n))) return rc;
        while (R->allocs.size() < n) R->allocs.push_back(R->budget_base + off[R->allocs.size()]);
        return XKB_OK;
    }
    size_t n = 0;
    int rc = xkb_planner_allocations(R->planner, nullptr, 0, &n);
    if (rc || n <= R->allocs.size()) return rc;
    std::vector<uint64_t> sizes(n);
    if ((rc = xkb_planner_allocations(R->planner, sizes.data(), n, &n))) return rc;
    while (R->allocs.size() < n)
    {
        void * p = nullptr;
        const cudaError_t e = cudaMalloc(&p, std::max<uint64_t>(sizes[R->allocs.size()], 16));
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
        R->allocs.push_back(p);
    }
    return XKB_OK;
}

// A host copy whose host bytes run across an end of a page-locked piece of registered memory
// (locked and pageable memory, or two pieces, in one copy: the driver refuses it) becomes one
// copy per column, each cut at those ends -- what the reference's registration-overflow
// protection does by splitting its partition (memory-tree.hpp:2184-2240).
static void split_at_locked_ends(const xkb_runtime * R, std::vector<xkb_copy_t> & c)
{
    if (R->user_pinned.empty()) return;
    auto cuts_inside = [&](uint64_t lo, uint64_t hi, std::vector<uint64_t> * out) {
        bool any = false;
        auto it = R->user_pinned.upper_bound(lo);
        if (it != R->user_pinned.begin()) --it;
        for (; it != R->user_pinned.end() && it->first < hi; ++it)
            for (uint64_t x : {it->first, it->second})
                if (lo < x && x < hi) { any = true; if (out) out->push_back(x); }
        return any;
    };
    std::vector<xkb_copy_t> out;
    bool changed = false;
    for (const xkb_copy_t & k : c)
    {
        if (k.kind == XKB_COPY_D2D) { out.push_back(k); continue; }
        const bool h2d = k.kind == XKB_COPY_H2D;
        const uint64_t hbase = (uint64_t) (h2d ? k.src_off : k.dst_off);
        const int64_t row = k.m * k.sizeof_type;
        const int64_t hld = (h2d ? k.src_ld : k.dst_ld) * k.sizeof_type, dld = (h2d ? k.dst_ld : k.src_ld) * k.sizeof_type;
        const uint64_t span = (uint64_t) ((k.n - 1) * hld + row);
        if (!cuts_inside(hbase, hbase + span, nullptr)) { out.push_back(k); continue; }
        changed = true;
        const int64_t dbase = h2d ? k.dst_off : k.src_off;
        for (int64_t j = 0; j < k.n; ++j)
        {
            const uint64_t h0 = hbase + (uint64_t) (j * hld);
            std::vector<uint64_t> cut;
            cuts_inside(h0, h0 + (uint64_t) row, &cut);
            std::sort(cut.begin(), cut.end());
            uint64_t a = h0;
            cut.push_back(h0 + (uint64_t) row);
            for (uint64_t x : cut)
            {
                xkb_copy_t q = k;
                q.m = (int64_t) (x - a); q.n = 1; q.sizeof_type = 1; q.src_ld = q.dst_ld = 0;
                const int64_t d = dbase + j * dld + (int64_t) (a - h0);
                if (h2d) { q.src_off = (int64_t) a; q.dst_off = d; } else { q.dst_off = (int64_t) a; q.src_off = d; }
                out.push_back(q);
                a = x;
            }
        }
    }
    if (changed) c.swap(out);
}

static int run_copies(xkb_runtime * R, cudaStream_t stream)
{
    size_t n = 0;
    int rc = xkb_planner_copies(R->planner, nullptr, 0, &n, 0);
    if (rc || !n) return rc;
    std::vector<xkb_copy_t> c(n);
    if ((rc = xkb_planner_copies(R->planner, c.data(), n, &n, 1))) return rc;
    ++R->copy_calls;
    if (R->plan_record) fwrite(c.data(), sizeof(xkb_copy_t), n, R->plan_record);      // the planner's records
    split_at_locked_ends(R, c);
    n = c.size();
    std::vector<uint64_t> cuts;                       // locked-piece ends: copies are not merged across them
    for (auto & kv : R->user_pinned) { cuts.push_back(kv.first); cuts.push_back(kv.second); }
    if (R->ref_mode)
    {
        if ((rc = ensure_allocs(R))) return rc;
        for (const xkb_copy_t & k : c)
        {
            (k.kind == XKB_COPY_H2D ? R->cur_h2d : k.kind == XKB_COPY_D2H ? R->cur_d2h : R->cur_d2d) += 1;
            if (k.kind != XKB_COPY_D2D)
                (k.kind == XKB_COPY_H2D ? R->cur_h2d_bytes : R->cur_d2h_bytes) += (uint64_t) (k.m * k.n * k.sizeof_type);
        }
        return xkb_internal_plan_execute_cut(c.data(), n, R->allocs.data(), R->allocs.size(), stream, cuts.data(), cuts.size());
    }
    int32_t maxid = -1;                               // ids of merged-away regions are not reused
    for (auto & kv : R->regions) maxid = std::max(maxid, kv.second.id);
    std::vector<void *> ptrs((size_t) (maxid + 1), nullptr);
    for (auto & kv : R->regions) if (kv.second.id >= 0) ptrs[kv.second.id] = kv.second.mirror;
    for (const xkb_copy_t & k : c)
    {
        (k.kind == XKB_COPY_H2D ? R->cur_h2d : R->cur_d2h) += 1;
        (k.kind == XKB_COPY_H2D ? R->cur_h2d_bytes : R->cur_d2h_bytes) += (uint64_t) (k.m * k.n * k.sizeof_type);
    }
    return xkb_internal_plan_execute_cut(c.data(), n, ptrs.data(), ptrs.size(), stream, cuts.data(), cuts.size());
}

// Point a built-in descriptor's host addresses at the device mirrors.
// false when a pointer lies outside every registered region (no error text: callable from
// several threads at once)
// The mirror of host bytes [host, host + bytes), or null unless one region holds all of them (a
// body indexes its grid or vector from the translated base, so every byte it may touch must be
// in that region's mirror).
static void * mirror_range(const xkb_runtime * R, uint64_t host, uint64_t bytes, RegionHint & h)
{
    uint8_t * m = (uint8_t *) mirror_lookup(R, host, h);
    return m && bytes <= h.end - host ? m : nullptr;
}

static bool translate_hint(const xkb_runtime * R, xkb_task_desc_t & d, RegionHint & h)
{
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        // the whole grid: the tile's strips may read any row of its columns and their neighbours
        const auto & g = d.u.heat;
        if (g.nx <= 0 || g.ny <= 0 || g.ld < g.nx) return false;
        const uint64_t esz = d.kind == XKB_TASK_HEAT_F64 ? 8 : 4;
        const uint64_t bytes = ((uint64_t) (g.ny - 1) * (uint64_t) g.ld + (uint64_t) g.nx) * esz;
        void * s = mirror_range(R, g.src, bytes, h), * t = mirror_range(R, g.dst, bytes, h);
        if (!s || !t) return false;
        d.u.heat.src = (uint64_t) s; d.u.heat.dst = (uint64_t) t;
    }
    else if (d.kind == XKB_TASK_AXPBY)
    {
        const auto & v = d.u.axpby;
        if (v.lo < 0 || v.hi < v.lo) return false;
        const uint64_t off = (uint64_t) v.lo * 8, bytes = (uint64_t) (v.hi - v.lo) * 8;
        // x and y are the vectors' bases; the task touches elements [lo, hi) of each
        void * x = mirror_range(R, v.x + off, bytes, h), * y = mirror_range(R, v.y + off, bytes, h);
        if (!x || !y) return false;
        d.u.axpby.x = (uint64_t) x - off; d.u.axpby.y = (uint64_t) y - off;
    }
    return true;
}

static int translate(xkb_runtime * R, xkb_task_desc_t & d)
{
    RegionHint h{R->last_base, R->last_end, R->last_mirror};
    if (!translate_hint(R, d, h)) return xkb_set_error(XKB_EINVAL, "task %s outside every registered region",
                                                       d.kind == XKB_TASK_AXPBY ? "vector" : "grid");
    return XKB_OK;
}

constexpr uint8_t REC_NONE = 0xff;                     // record type of an untracked access

// fn(begin, end) over [0, n) in contiguous chunks on up to 16 host threads (inline when small)
template <typename F>
static void parallel_chunks(size_t n, F fn)
{
    const size_t nth = std::min<size_t>(xkb_internal_helpers(), n / 65536);
    if (nth < 2) { fn(0, n); return; }
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nth; ++k) pool.emplace_back(fn, n * k / nth, n * (k + 1) / nth);
    fn(0, n / nth);
    for (auto & th : pool) th.join();
}

// Indices of the first occurrence of every distinct record among those `keep` accepts, in
// record order. Chunks of records are scanned on host threads, each keeping its own first
// occurrences; merging the chunks' lists in chunk order keeps the global first occurrences.
template <typename Keep>
static std::vector<uint32_t> distinct_records(const xkb_access_rec_t * recs, size_t n, Keep keep)
{
    const size_t nth = std::max<size_t>(1, std::min<size_t>(xkb_internal_helpers(), n / 65536));
    std::vector<std::vector<uint32_t>> firsts(nth);
    auto scan = [&](size_t k) {
        RecordSet seen;
        for (size_t i = n * k / nth; i < n * (k + 1) / nth; ++i)
            if (keep(i) && seen.insert(recs, (uint32_t) i)) firsts[k].push_back((uint32_t) i);
    };
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nth; ++k) pool.emplace_back(scan, k);
    scan(0);
    for (auto & th : pool) th.join();
    if (nth == 1) return std::move(firsts[0]);
    std::vector<uint32_t> out;
    RecordSet seen;
    for (auto & f : firsts)
        for (uint32_t i : f)
            if (seen.insert(recs, i)) out.push_back(i);
    return out;
}

// The records of accesses [a0, a1) that carry data to make coherent on the device (not handles,
// not unified memory) and were not seen before in this batch: their first occurrences are added
// to R->dfirst in record order; returns where they start there. Host threads scan chunks of the
// range, each skipping what the batch's set already holds and keeping its own first occurrences;
// adding the chunks' lists in chunk order keeps the first occurrences.
static size_t add_distinct(xkb_runtime * R, size_t a0, size_t a1)
{
    const xkb_access_rec_t * recs = R->recs.data();
    const size_t start = R->dfirst.size(), n = a1 - a0;
    const size_t nth = std::max<size_t>(1, std::min<size_t>(xkb_internal_helpers(), n / 65536));
    std::vector<std::vector<uint32_t>> firsts(nth);
    const RecordSet & known = R->dset;
    auto scan = [&](size_t k) {
        RecordSet seen;
        for (size_t i = a0 + n * k / nth; i < a0 + n * (k + 1) / nth; ++i)
            if (recs[i].type != REC_NONE && recs[i].type != XKB_ACCESS_TYPE_HANDLE && !known.contains(recs, (uint32_t) i) &&
                !in_unified(R, recs[i]) && seen.insert(recs, (uint32_t) i))
                firsts[k].push_back((uint32_t) i);
    };
    std::vector<std::thread> pool;
    for (size_t k = 1; k < nth; ++k) pool.emplace_back(scan, k);
    scan(0);
    for (auto & th : pool) th.join();
    pool.clear();
    size_t total = 0;
    for (auto & f : firsts) total += f.size();
    if (nth == 1 || total < 65536)
    {
        for (auto & f : firsts)
            for (uint32_t i : f)
                if (R->dset.insert(recs, i)) R->dfirst.push_back(i);
        return start;
    }
    // many candidates (a first window): the threads split the keys by hash, each keeping the
    // first occurrence of its keys (lists in chunk order); sorted by index, the winners are the
    // first occurrences in record order
    std::vector<std::vector<uint32_t>> part(nth);
    auto merge = [&](size_t j) {
        RecordSet mine;
        for (auto & f : firsts)
            for (uint32_t i : f)
                if ((RecordSet::key_hash(recs[i]) >> 40) % nth == j && mine.insert(recs, i)) part[j].push_back(i);
    };
    for (size_t k = 1; k < nth; ++k) pool.emplace_back(merge, k);
    merge(0);
    for (auto & th : pool) th.join();
    std::vector<uint32_t> win;
    for (auto & q : part) win.insert(win.end(), q.begin(), q.end());
    std::sort(win.begin(), win.end());
    for (uint32_t i : win) { R->dset.insert(recs, i); R->dfirst.push_back(i); }
    return start;
}

static double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Trace clock: milliseconds since the process's first trace line.
static double trace_clock_ms()
{
    static const auto epoch = std::chrono::steady_clock::now();
    return ms_since(epoch);
}

// Device array owned by the runtime (freed when replaced or at deinit).
struct DevArray {
    void * p = nullptr;
    size_t bytes = 0;
    ~DevArray() { if (p) cudaFree(p); }
    int put(const void * host, size_t n)
    {
        if (n > bytes)
        {
            if (p) { cudaFree(p); p = nullptr; bytes = 0; }
            if (cudaMalloc(&p, n) != cudaSuccess) { cudaGetLastError(); return xkb_set_error(XKB_ENOMEM, "xkrt_task_wait: device allocation"); }
            bytes = n;
        }
        if (n && cudaMemcpy(p, host, n, cudaMemcpyHostToDevice) != cudaSuccess) return xkb_set_error(XKB_ECUDA, "xkrt_task_wait: copy");
        return XKB_OK;
    }
};

// Moldable execution of long axpby tasks: a built-in axpby task over more than SPLIT elements
// runs as ceil(len / SPLIT) slice tasks plus a no-op join task. Every predecessor of the task
// precedes each slice, each slice precedes the join, and the join precedes the task's
// successors -- the same order constraints, with the element range spread over many teams of
// the persistent kernel instead of one.
constexpr int64_t AXPBY_SPLIT = int64_t(1) << 15;

struct SplitGraph {
    DevArray succ_ptr, succ, npred;
    std::vector<xkb_task_desc_t> descs;
    xkb_task_graph_t g{};
};

// false: nothing to split (descs / g unchanged).
static int split_moldable(const xkb_task_desc_t * descs, size_t nt, const xkb_task_graph_t & g, SplitGraph & out, bool & split)
{
    split = false;
    std::vector<uint32_t> k(nt);
    size_t nnew = 0;
    for (size_t t = 0; t < nt; ++t)
    {
        const xkb_task_desc_t & d = descs[t];
        const int64_t len = d.kind == XKB_TASK_AXPBY ? d.u.axpby.hi - d.u.axpby.lo : 0;
        k[t] = len > AXPBY_SPLIT ? (uint32_t) ((len + AXPBY_SPLIT - 1) / AXPBY_SPLIT) : 1u;
        if (k[t] > 1) split = true;
        nnew += k[t] > 1 ? k[t] + 1 : 1;
    }
    if (!split) return XKB_OK;
    if (nnew >= (size_t(1) << 31)) return xkb_set_error(XKB_ERANGE, "xkrt_task_wait: %zu tasks after splitting", nnew);
    std::vector<uint32_t> ptr(nt + 1), succ(g.nedges), npred(nt);
    if (cudaMemcpy(ptr.data(), g.succ_ptr, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess ||
        (g.nedges && cudaMemcpy(succ.data(), g.succ, g.nedges * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        cudaMemcpy(npred.data(), g.npred, nt * sizeof(uint32_t), cudaMemcpyDeviceToHost) != cudaSuccess)
        return xkb_set_error(XKB_ECUDA, "xkrt_task_wait: graph download");
    std::vector<uint32_t> first(nt);                         // new id of the task's first node
    out.descs.resize(nnew);
    std::vector<uint32_t> np(nnew), nsucc(nnew, 0);
    uint32_t id = 0;
    for (size_t t = 0; t < nt; ++t)
    {
        first[t] = id;
        if (k[t] == 1) { out.descs[id] = descs[t]; np[id] = npred[t]; ++id; continue; }
        const xkb_task_desc_t & d = descs[t];
        for (uint32_t i = 0; i < k[t]; ++i)
        {
            xkb_task_desc_t q = d;
            q.u.axpby.lo = d.u.axpby.lo + (int64_t) i * AXPBY_SPLIT;
            q.u.axpby.hi = std::min<int64_t>(q.u.axpby.lo + AXPBY_SPLIT, d.u.axpby.hi);
            out.descs[id] = q; np[id] = npred[t]; ++id;
        }
        xkb_task_desc_t j;
        memset(&j, 0, sizeof(j));
        j.kind = XKB_TASK_NOOP;
        out.descs[id] = j; np[id] = k[t]; ++id;
    }
    auto exit_of = [&](size_t t) { return k[t] == 1 ? first[t] : first[t] + k[t]; };
    // successor counts, then CSR fill in ascending order
    for (size_t t = 0; t < nt; ++t)
    {
        const uint32_t e = exit_of(t);
        for (uint32_t i = ptr[t]; i < ptr[t + 1]; ++i) nsucc[e] += k[succ[i]];
        if (k[t] > 1) for (uint32_t i = 0; i < k[t]; ++i) nsucc[first[t] + i] = 1;
    }
    std::vector<uint32_t> nptr(nnew + 1, 0);
    for (size_t v = 0; v < nnew; ++v) nptr[v + 1] = nptr[v] + nsucc[v];
    std::vector<uint32_t> nsc(nptr[nnew]);
    for (size_t t = 0; t < nt; ++t)
    {
        uint32_t at = nptr[exit_of(t)];
        for (uint32_t i = ptr[t]; i < ptr[t + 1]; ++i)
            for (uint32_t s2 = 0; s2 < k[succ[i]]; ++s2) nsc[at++] = first[succ[i]] + s2;
        if (k[t] > 1) for (uint32_t i = 0; i < k[t]; ++i) nsc[nptr[first[t] + i]] = first[t] + k[t];
    }
    int rc;
    if ((rc = out.succ_ptr.put(nptr.data(), nptr.size() * sizeof(uint32_t))) ||
        (rc = out.succ.put(nsc.data(), std::max<size_t>(nsc.size(), 1) * sizeof(uint32_t))) ||
        (rc = out.npred.put(np.data(), np.size() * sizeof(uint32_t))))
        return rc;
    out.g.ntasks = nnew; out.g.nedges = nsc.size();
    out.g.succ_ptr = (const uint32_t *) out.succ_ptr.p; out.g.succ = (const uint32_t *) out.succ.p;
    out.g.npred = (const uint32_t *) out.npred.p;
    return XKB_OK;
}


// Records of tasks [t0, t1) (accesses [a0, a1)) into R->recs at their access indices, then into
// the batch's resolver: directly when every task has a tracked access, else compacted with a
// one-byte virtual read of the task's own Task object for a task without one (nothing else
// touches it), so that task numbering stays dense.
// Resolve tasks [t0, t1) (accesses [a0, a1)); *mark (optional) receives the resolver's edge mark
// before them.
// before_add (optional) runs once the records are converted, before the resolver works on them.
static int resolve_range(xkb_runtime * R, size_t t0, size_t t1, size_t a0, size_t a1, xkb_edge_mark_t * mark = nullptr,
                         const std::function<int()> * before_add = nullptr)
{
    if (t0 >= t1) return XKB_OK;
    if (!R->recs.resize(a1)) return xkb_set_error(XKB_ENOMEM, "xkrt_task_wait: out of host memory");
    xkb_access_rec_t * recs = R->recs.data();
    // the pools do not move while this runs (fixed reservations, or no spawn during the wait)
    const Task * tasks = R->pending.data();
    const xkrt_access_t * accs = R->acc_pool.data();
    std::atomic<bool> dense(true);
    parallel_chunks(t1 - t0, [&](size_t b, size_t e) {
        bool d = true;
        for (size_t t = t0 + b; t < t0 + e; ++t)
        {
            const Task & T = tasks[t];
            bool any = false;
            for (uint32_t k = 0; k < T.nacc; ++k)
            {
                xkb_access_rec_t & r = recs[T.acc_off + k];
                if (to_rec(accs[T.acc_off + k], (uint32_t) t, r)) any = true;
                else { r.type = REC_NONE; d = false; }
            }
            d = d && any;
        }
        if (!d) dense = false;
    });
    std::vector<xkb_access_rec_t> all;
    if (!dense)
    {
        all.reserve(a1 - a0 + 16);
        for (size_t t = t0; t < t1; ++t)
        {
            const Task & T = R->pending[t];
            bool any = false;
            for (uint32_t k = 0; k < T.nacc; ++k)
                if (recs[T.acc_off + k].type != REC_NONE) { all.push_back(recs[T.acc_off + k]); any = true; }
            if (!any)
            {
                xkb_access_rec_t r;
                memset(&r, 0, sizeof(r));
                r.task = (uint32_t) t; r.type = XKB_ACCESS_TYPE_SEGMENT; r.mode = XKB_ACCESS_MODE_R | XKB_ACCESS_MODE_V;
                r.addr = (uint64_t) &R->pending[t]; r.ld = r.addr + 1;
                all.push_back(r);
            }
        }
    }
    const xkb_access_rec_t * feed = dense ? recs + a0 : all.data();
    const size_t nfeed = dense ? a1 - a0 : all.size();
    int rc = XKB_OK;
    if (!R->res && (rc = xkb_resolver_create(&R->res, R->stream))) return rc;
    if (R->res_stale && (rc = xkb_internal_resolver_reset(R->res))) return rc;
    R->res_stale = false;
    if (mark && (rc = xkb_internal_resolver_edge_mark(R->res, mark))) return rc;
    if (before_add && (rc = (*before_add)())) return rc;
    for (size_t b = 0; b < nfeed && rc == XKB_OK;)
    {
        size_t e = std::min(nfeed, b + R->chunk);
        while (e < nfeed && feed[e].task == feed[e - 1].task) ++e;     // whole tasks per batch
        rc = xkb_resolver_add(R->res, feed + b, e - b);
        b = e;
    }
    return rc;
}

static int stream_prepare(xkb_runtime * R, size_t t0, size_t t1, size_t a0, size_t a1, bool * ok);
static int stream_launch(xkb_runtime * R, const xkb_edge_mark_t & mark);

static void bg_worker(xkb_runtime * R)
{
    cudaSetDevice(R->device);
    static const bool trace = getenv("XKB_TRACE_WAIT") != nullptr;
    for (;;)
    {
        size_t t0, t1, a0, a1;
        bool failed;
        {
            std::unique_lock<std::mutex> lk(R->mu);
            R->cv.wait(lk, [&] { return R->stop || R->handed > R->claimed; });
            if (R->handed == R->claimed) return;          // stop, nothing pending
            // one hand-over at a time: windows of about a resolver batch, so the GPU starts on
            // the first ones while later ones are resolved
            t0 = R->claimed; t1 = R->hand_q.front().first;
            a0 = R->pending[t0].acc_off; a1 = R->hand_q.front().second;
            R->hand_q.pop_front();
            R->claimed = t1;
            failed = R->bg_rc != XKB_OK;
        }
        xkb_edge_mark_t mark{};
        const auto w0 = std::chrono::steady_clock::now();
        bool streamed = false;
        const std::function<int()> prep = [&] { return stream_prepare(R, t0, t1, a0, a1, &streamed); };
        int rc = failed ? XKB_OK : resolve_range(R, t0, t1, a0, a1, &mark, &prep);
        const double res_ms = ms_since(w0);
        if (!failed && rc == XKB_OK && streamed) rc = stream_launch(R, mark);
        if (rc) streamed = false;
        if (trace)
            fprintf(stderr, "worker: tasks [%zu, %zu) prepared and resolved in %.1f ms, %s in %.1f ms (at %.1f ms)\n", t0, t1, res_ms,
                    streamed ? "launched" : "kept", ms_since(w0) - res_ms, trace_clock_ms());
        {
            std::lock_guard<std::mutex> lk(R->mu);
            if (rc && R->bg_rc == XKB_OK) { R->bg_rc = rc; R->bg_err = xkb_last_error(); }
            if (streamed) R->streamed = t1;
            else if (R->stream_ok) { R->stream_ok = false; R->rest_mark = mark; }
            R->done = t1;
        }
        R->cv.notify_all();
    }
}

// Hand the tasks spawned since the last hand-over to the worker: once they hold a batch's worth
// of accesses, or all of them (final) when the program waits.
static void bg_hand_over(xkb_runtime * R, bool final)
{
    const size_t nacc = R->acc_pool.size(), nt = R->pending.size();
    // the first hand-over of a batch comes early (a 32nd of a batch), so that the GPU starts on
    // the first window while the rest is spawned: a small first window also makes only part of
    // the data coherent, the rest coming with the next windows while the GPU runs
    const size_t want = R->handed ? R->chunk : std::max<size_t>(16, R->chunk / 32);
    if (nt == R->handed || (!final && nacc - R->handed_acc < want)) return;
    {
        std::lock_guard<std::mutex> lk(R->mu);
        R->handed = nt; R->handed_acc = nacc;
        R->hand_q.emplace_back(nt, nacc);
    }
    static const bool trace = getenv("XKB_TRACE_WAIT") != nullptr;
    if (trace) fprintf(stderr, "hand-over: tasks up to %zu (at %.1f ms)\n", nt, trace_clock_ms());
    if (!R->worker.joinable()) R->worker = std::thread(bg_worker, R);
    R->cv.notify_all();
}

// Wait until the worker has resolved everything handed to it.
static void bg_wait_done(xkb_runtime * R)
{
    std::unique_lock<std::mutex> lk(R->mu);
    R->cv.wait(lk, [&] { return R->done == R->handed; });
}

// End of a batch: no work in flight, counters and the batch's resolver reset.
static void bg_finish(xkb_runtime * R)
{
    if (R->worker.joinable()) bg_wait_done(R);
    R->handed = R->handed_acc = R->claimed = R->done = 0;
    R->hand_q.clear();
    R->bg_rc = XKB_OK;
    R->bg_err.clear();
    R->streamed = 0;
    R->stream_ok = true;
    R->dset.reset();
    R->dfirst.clear();
    R->hmap.clear();                      // every task of the batch completed: no handle orders anything
    R->res_stale = R->res != nullptr;     // kept with its buffers; reset when the next batch starts
}

// Reference mode: the leading dimension (in elements) of each device view of the task run_one is
// making coherent on this thread (-1: the host layout's).
thread_local std::vector<int64_t> g_view_ld;

// Reference mode: a built-in body on the per-access allocations its accesses were fetched into --
// heat: access 0 the halo-expanded source tile, access 1 the destination tile, re-based on the
// tile's first cell as the reference's launcher does (examples/heat-diffusion-2d/src/main.cc:
// 214-219); axpby: access 0 the x range, access 1 the y range.
static int run_builtin_views(xkb_runtime * R, Task & T, size_t t, const xkb_access_rec_t * recs, xkb_task_desc_t d,
                             cudaStream_t stream)
{
    if (d.kind == XKB_TASK_NOOP) return XKB_OK;
    if (T.nacc < 2) return xkb_set_error(XKB_EINVAL, "built-in task %zu: needs its two data accesses in reference mode", t);
    const xkb_access_rec_t & r0 = recs[T.acc_off], & r1 = recs[T.acc_off + 1];
    uint8_t * p0 = (uint8_t *) R->replica_pool[T.acc_off], * p1 = (uint8_t *) R->replica_pool[T.acc_off + 1];
    if (!p0 || !p1) return xkb_set_error(XKB_EINVAL, "built-in task %zu: accesses without device views", t);
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        const auto & h = d.u.heat;
        const int64_t es = d.kind == XKB_TASK_HEAT_F64 ? 8 : 4, l0 = g_view_ld[0], l1 = g_view_ld[1];
        if (r0.type != XKB_ACCESS_TYPE_BLAS_MATRIX || r1.type != XKB_ACCESS_TYPE_BLAS_MATRIX || l0 <= 0 || l1 <= 0)
            return xkb_set_error(XKB_EINVAL, "heat task %zu: accesses 0 and 1 must be matrix tiles in reference mode", t);
        const uint8_t * src = p0 + (((int64_t) h.x0 - (int64_t) r0.offset_m) + ((int64_t) h.y0 - (int64_t) r0.offset_n) * l0) * es;
        uint8_t * dst = p1 + (((int64_t) h.x0 - (int64_t) r1.offset_m) + ((int64_t) h.y0 - (int64_t) r1.offset_n) * l1) * es;
        return xkb_internal_diffusion_box(d.kind == XKB_TASK_HEAT_F64 ? XKB_F64 : XKB_F32, stream, src, l0, dst, l1, h.x0, h.y0,
                                          (int64_t) h.x1 - h.x0, (int64_t) h.y1 - h.y0, h.nx, h.ny, h.c);
    }
    if (d.kind == XKB_TASK_AXPBY)
    {
        d.u.axpby.x = (uint64_t) (uintptr_t) (p0 - d.u.axpby.lo * 8);
        d.u.axpby.y = (uint64_t) (uintptr_t) (p1 - d.u.axpby.lo * 8);
        return xkb_internal_launch_task(&d, stream);
    }
    return xkb_set_error(XKB_EINVAL, "built-in task %zu: unknown kind %u", t, d.kind);
}

// The body of a task built with the C++ source API: each access's device_view points at the
// access's first element where the body runs (its leading dimension in elements), then the
// format's function is called as f(runtime, device, task) with the program's runtime_t and
// task_t (a CUDA-target body on the worker's stream; a device task without format runs nothing).
static int run_cxx_body(xkb_runtime * R, Task & T, size_t t, bool dev, cudaStream_t stream, bool * deferred)
{
    xkrt::task_t * task = (xkrt::task_t *) cxx_of(T);
    xkrt::access_t * acc = (task->flags & TASK_FLAG_DEPENDENT) ? xkrt::TASK_ACCESSES(task) : nullptr;
    for (uint32_t a = 0; a < T.nacc && acc; ++a)
    {
        const uintptr_t addr = (uintptr_t) R->replica_pool[T.acc_off + a];
        const xkrt::memory_view_t & h = acc[a].host_view;
        const int64_t vld = a < g_view_ld.size() ? g_view_ld[a] : -1;
        acc[a].device_view = xkrt::memory_replica_view_t(addr, vld >= 0 ? (size_t) vld : acc[a].type == ACCESS_TYPE_BLAS_MATRIX ? h.ld : h.m);
        acc[a].state = xkrt::ACCESS_STATE_FETCHED;
    }
    task->state.value = xkrt::TASK_STATE_EXECUTING;
    const Format & f = R->formats[T.fmtid];
    typedef void (*body3_t)(void *, void *, void *);
    if (dev)
    {
        if (!f.f[XKRT_TASK_FORMAT_TARGET_CUDA]) return XKB_OK;
        g_stream = stream;
        ((body3_t) f.f[XKRT_TASK_FORMAT_TARGET_CUDA])(R->cxx_rt, &R->devices[1], task);
        g_stream = nullptr;
        if (deferred) { *deferred = true; return XKB_OK; }        // the caller tracks its completion
        if (cudaStreamSynchronize(stream) != cudaSuccess) return xkb_set_error(XKB_ECUDA, "task %zu: device body", t);
        return XKB_OK;
    }
    if (f.f[XKRT_TASK_FORMAT_TARGET_HOST])
    {
        if (R->cxx_task_first) ((body3_t) f.f[XKRT_TASK_FORMAT_TARGET_HOST])(task, &R->devices[0], task);
        else ((body3_t) f.f[XKRT_TASK_FORMAT_TARGET_HOST])(R->cxx_rt, &R->devices[0], task);
        return XKB_OK;
    }
    return T.fmtid ? xkb_set_error(XKB_EINVAL, "task %zu: its format has no host body", t) : XKB_OK;
}

// One task of a non-fused batch on the calling worker: its accesses made coherent where it runs
// (planner fetches and their copies, completed before the planner is released, so the planner's
// state always describes data that is in place; skipped when the batch was made coherent up
// front), then its body; a device body runs on the worker's stream and, with `deferred` null, is
// complete when this returns. With `deferred` non-null a device body's work may be left in flight
// on `stream`: *deferred is then set and the caller completes the task once the stream has passed
// it. Completing drops the body's reference: a task the body made detachable completes when its
// last reference goes, on whatever thread.
static int run_one(xkb_runtime * R, size_t t, const xkb_access_rec_t * recs, cudaStream_t stream, bool * deferred = nullptr)
{
    Task & T = R->pending[t];
    const bool dev = is_device(R, T);
    int rc = XKB_OK;
    g_view_ld.assign(T.nacc, -1);
    if (!R->preplanned)
    {
        std::lock_guard<std::mutex> lk(R->plan_mu);
        const uint64_t calls0 = R->copy_calls;
        if (R->ref_mode) rc = apply_registrations(R, t);
        for (uint32_t a = 0; a < T.nacc && rc == XKB_OK; ++a)
        {
            const xkb_access_rec_t & r = recs[T.acc_off + a];
            if (r.type == REC_NONE) continue;
            if (r.type == XKB_ACCESS_TYPE_HANDLE) { R->replica_pool[T.acc_off + a] = (void *) (uintptr_t) r.addr; continue; }
            const uint64_t begin = rec_begin(r);
            if (R->ref_mode)
            {
                // the reference's decisions: the access's own device allocation (its view), the
                // copies its memory tree plans; a host access reads the host memory in place
                xkb_view_t v;
                if ((rc = xkb_planner_fetch(R->planner, &r, a, dev ? 1 : 0, &v))) break;
                // each fetch's copies before the next fetch: an eviction by the next one may
                // reuse the memory these copies read
                if ((rc = run_copies(R, stream))) break;
                if (dev)
                {
                    if ((rc = ensure_allocs(R))) break;
                    R->replica_pool[T.acc_off + a] = (uint8_t *) R->allocs[v.alloc] + v.off;
                    g_view_ld[a] = v.ld;
                }
                else R->replica_pool[T.acc_off + a] = (void *) begin;
                continue;
            }
            R->replica_pool[T.acc_off + a] = dev ? mirror_of(R, begin) : (void *) begin;
            // a host task on memory no region covers: that memory never has a device copy;
            // unified memory needs no copy either way
            if (!dev && !mirror_of(R, begin)) continue;
            if (in_unified(R, r)) continue;
            xkb_view_t v;
            rc = xkb_planner_fetch(R->planner, &r, a, dev ? 1 : 0, &v);
        }
        if (rc == XKB_OK) rc = run_copies(R, stream);
        // the task's copies complete before the planner is released (its state then describes data
        // in place); a task that issued none has nothing to wait for
        if (rc == XKB_OK && R->copy_calls != calls0 && cudaStreamSynchronize(stream) != cudaSuccess)
            rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: copies");
    }
    if (rc) return rc;
    const Format & f = R->formats[T.fmtid];
    __atomic_add_fetch(&T.detach, 1, __ATOMIC_ACQ_REL);        // the body's own reference
    g_current = &T;
    if (cxx_of(T)) rc = run_cxx_body(R, T, t, dev, stream, deferred);
    else if (dev && T.fmtid == XKRT_TASK_FORMAT_NULL) {}         // placement only
    else if (dev)
    {
        if (f.builtin >= 0)
        {
            xkb_task_desc_t d;
            if (T.nargs < sizeof(d)) rc = xkb_set_error(XKB_EINVAL, "built-in task %zu: args are not an xkb_task_desc_t", t);
            else if (R->ref_mode)
            {
                memcpy(&d, R->args_pool.data() + T.args_off, sizeof(d));
                d.kind = (uint32_t) f.builtin;
                rc = run_builtin_views(R, T, t, recs, d, stream);
            }
            else
            {
                memcpy(&d, R->args_pool.data() + T.args_off, sizeof(d));
                d.kind = (uint32_t) f.builtin;
                RegionHint h;
                if (!translate_hint(R, d, h)) rc = xkb_set_error(XKB_EINVAL, "built-in task %zu: a grid or vector lies outside every registered region", t);
                else rc = xkb_internal_launch_task(&d, stream);
            }
        }
        else
        {
            g_stream = stream;
            ((void (*)(xkrt_runtime_t *, xkrt_device_t *, xkrt_task_t *)) f.f[XKRT_TASK_FORMAT_TARGET_CUDA])(
                (xkrt_runtime_t *) R, (xkrt_device_t *) &R->devices[1], (xkrt_task_t *) &T);
            g_stream = nullptr;
        }
        if (rc == XKB_OK && deferred) *deferred = true;
        else if (rc == XKB_OK && cudaStreamSynchronize(stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "task %zu: device body", t);
    }
    else if (T.func) T.func((xkrt_runtime_t *) R, (xkrt_device_t *) &R->devices[0], (xkrt_task_t *) &T, T.user_data);
    else if (f.f[XKRT_TASK_FORMAT_TARGET_HOST])
        ((void (*)(xkrt_runtime_t *, xkrt_device_t *, xkrt_task_t *)) f.f[XKRT_TASK_FORMAT_TARGET_HOST])(
            (xkrt_runtime_t *) R, (xkrt_device_t *) &R->devices[0], (xkrt_task_t *) &T);
    else if (T.fmtid) rc = xkb_set_error(XKB_EINVAL, "task %zu: its format has no host body", t);
    g_current = nullptr;
    return rc;
}

// The successor graph of a non-fused batch being executed: wait counters, the ready queue, and
// the number of completed tasks.
struct Dataflow {
    std::mutex mu;
    std::condition_variable cv;
    std::deque<uint32_t> ready;
    std::vector<uint32_t> ptr, succ, wc;
    size_t base = 0;                    // graph task k is the batch's task base + k
    size_t nt = 0, done = 0;
    int err = XKB_OK;
    std::string err_text;
};

// A task of the running batch completed: its successors' wait counters drop, the ready ones are
// queued (src/task.cc:160-245, __task_complete).
static void task_completed(::xkb_runtime * R, Task & T)
{
    if (void * c = cxx_of(T)) ((xkrt::task_t *) c)->state.value = xkrt::TASK_STATE_COMPLETED;
    Dataflow * D = R ? R->df.load(std::memory_order_acquire) : nullptr;
    if (!D) return;
    const size_t g = (size_t) (&T - R->pending.data());
    if (g < D->base || g - D->base >= D->nt) return;
    const size_t t = g - D->base;
    size_t woke = 0;
    bool last;
    {
        std::lock_guard<std::mutex> lk(D->mu);
        for (uint32_t i = D->ptr[t]; i < D->ptr[t + 1]; ++i)
            if (--D->wc[D->succ[i]] == 0) { D->ready.push_back(D->succ[i]); ++woke; }
        last = ++D->done == D->nt;
    }
    // one sleeping worker per task made ready (all of them at the end, so that they leave)
    if (last) D->cv.notify_all();
    else for (size_t k = 0; k < woke; ++k) D->cv.notify_one();
}

// A non-fused batch (its tasks from `base` on; the earlier ones completed): ready tasks (all
// predecessors completed) run on a team of host threads,
// XKB_HOST_THREADS or one per hardware thread (at most 64) -- the reference's host team and
// device threads executing ready tasks as their predecessors complete. A detached task holds no
// thread; the batch ends when every task completed (600 s without progress is an error).
static int fetch_new_to_device(xkb_runtime * R, size_t a0, size_t a1);

// Tasks [t0, t1) (accesses [a0, a1)) when all of them run on the device and every access they
// make lies in a registered region with a device mirror (or is a handle): their distinct records
// are made coherent on the device now, in spawn order (copies complete on return), and each
// access's replica pointer is set, so R->preplanned lets run_one skip the planner. Otherwise
// nothing is done and each task plans its own coherency.
static int preplan_device_batch(xkb_runtime * R, size_t t0, size_t t1, size_t a0, size_t a1)
{
    R->preplanned = false;
    if (!R->gpu || t0 >= t1) return XKB_OK;
    const xkb_access_rec_t * recs = R->recs.data();
    std::lock_guard<std::mutex> lk(R->plan_mu);
    for (size_t t = t0; t < t1; ++t)
    {
        const Task & T = R->pending[t];
        if (!is_device(R, T)) return XKB_OK;
        for (uint32_t a = 0; a < T.nacc; ++a)
        {
            const xkb_access_rec_t & r = recs[T.acc_off + a];
            if (r.type == REC_NONE) continue;
            if (r.type == XKB_ACCESS_TYPE_HANDLE) { R->replica_pool[T.acc_off + a] = (void *) (uintptr_t) r.addr; continue; }
            if (in_unified(R, r)) return XKB_OK;
            void * m = mirror_of(R, rec_begin(r));
            if (!m) return XKB_OK;
            R->replica_pool[T.acc_off + a] = m;
        }
    }
    int rc = fetch_new_to_device(R, a0, a1);
    if (rc == XKB_OK && cudaStreamSynchronize(R->stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: copies");
    if (rc == XKB_OK) R->preplanned = true;
    return rc;
}

static int run_dataflow(xkb_runtime * R, const xkb_task_graph_t & g, const xkb_access_rec_t * recs, size_t base)
{
    const size_t nt = R->pending.size() - base;
    // the replicas the bodies read (xkrt_task_access_replica): set as each task's accesses are
    // made coherent, null until then; only tasks run here have bodies that read them
    if (nt && !R->preplanned)                      // preplanned: already set for every access
    {
        const size_t a0 = R->pending[base].acc_off;
        memset(R->replica_pool.data() + a0, 0, (R->acc_pool.size() - a0) * sizeof(void *));
    }
    Dataflow D;
    D.base = base;
    D.nt = nt;
    D.ptr.resize(nt + 1); D.succ.resize(g.nedges ? g.nedges : 1); D.wc.resize(nt);
    if (cudaMemcpyAsync(D.ptr.data(), g.succ_ptr, (nt + 1) * sizeof(uint32_t), cudaMemcpyDeviceToHost, R->stream) != cudaSuccess ||
        (g.nedges && cudaMemcpyAsync(D.succ.data(), g.succ, g.nedges * sizeof(uint32_t), cudaMemcpyDeviceToHost, R->stream) != cudaSuccess) ||
        cudaMemcpyAsync(D.wc.data(), g.npred, nt * sizeof(uint32_t), cudaMemcpyDeviceToHost, R->stream) != cudaSuccess ||
        cudaStreamSynchronize(R->stream) != cudaSuccess)
        return xkb_set_error(XKB_ECUDA, "xkrt_task_wait: graph download");
    size_t nw = std::thread::hardware_concurrency();
    if (const char * e = getenv("XKB_HOST_THREADS")) nw = strtoul(e, nullptr, 10);
    nw = std::max<size_t>(1, std::min<size_t>({nw ? nw : 1, 64, nt}));
    if (R->ref_mode) nw = 1;             // one task at a time, in spawn order: the canonical schedule
    while (R->wstreams.size() < nw)
    {
        cudaStream_t st;
        if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return xkb_set_error(XKB_ECUDA, "xkrt_task_wait: stream");
        R->wstreams.push_back(st);
    }
    for (size_t t = 0; t < nt; ++t) if (D.wc[t] == 0) D.ready.push_back((uint32_t) t);
    R->df.store(&D, std::memory_order_release);
    // A worker leaves up to MAX_INFLIGHT device bodies in flight on its stream (resident mode):
    // it takes the next ready task while they run, and completes each one -- releasing its
    // successors -- once the stream has passed the event recorded after it. It never sleeps on
    // the ready queue while it holds work in flight: with nothing ready it waits for its oldest.
    // Reference mode runs one task at a time (an eviction may reuse memory a body still reads).
    constexpr size_t MAX_INFLIGHT = 8, GROUP = 4;
    auto worker = [&](size_t k) {
        cudaSetDevice(R->device);
        auto progress = std::chrono::steady_clock::now();
        size_t seen = 0;
        std::vector<cudaEvent_t> evs;                         // this worker's events, reused
        // bodies in flight, oldest first; an event is recorded after every GROUP of them (and
        // before the worker waits), and covers its entry and the ones before it
        std::deque<std::pair<uint32_t, cudaEvent_t>> fl;
        size_t open = 0;                                      // entries at the back with no event yet
        auto fail_with = [&](int rc) {
            std::lock_guard<std::mutex> lk(D.mu);
            if (D.err == XKB_OK) { D.err = rc; D.err_text = xkb_last_error(); }
            D.cv.notify_all();
        };
        auto leave = [&]() {                                  // nothing of this worker stays in flight
            if (!fl.empty()) cudaStreamSynchronize(R->wstreams[k]);
            for (auto & f : fl) if (f.second) evs.push_back(f.second);
            fl.clear(); open = 0;
            for (cudaEvent_t e : evs) cudaEventDestroy(e);
        };
        // an event after the entries that have none (false: none could be recorded; the worker
        // then waits for its stream, and every entry is covered)
        auto close = [&]() -> bool {
            if (!open) return true;
            cudaEvent_t ev = nullptr;
            if (!evs.empty()) { ev = evs.back(); evs.pop_back(); }
            else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) { cudaGetLastError(); ev = nullptr; }
            if (ev && cudaEventRecord(ev, R->wstreams[k]) == cudaSuccess) { fl.back().second = ev; open = 0; return true; }
            if (ev) evs.push_back(ev);
            cudaGetLastError();
            if (cudaStreamSynchronize(R->wstreams[k]) != cudaSuccess) return false;
            // everything is done: complete it all
            while (!fl.empty())
            {
                const uint32_t d = fl.front().first;
                if (fl.front().second) evs.push_back(fl.front().second);
                fl.pop_front();
                if (task_unref(R->pending[base + d])) task_completed(R, R->pending[base + d]);
            }
            open = 0;
            return true;
        };
        // complete the bodies the stream has passed (if `wait`, at least the oldest group)
        auto retire = [&](bool wait) -> bool {
            if (wait && !close()) { fail_with(xkb_set_error(XKB_ECUDA, "xkrt_task_wait: device body")); return false; }
            while (!fl.empty())
            {
                size_t g = 0;
                while (g < fl.size() && !fl[g].second) ++g;
                if (g == fl.size()) return true;              // only the open group is left
                const cudaError_t e = wait ? cudaEventSynchronize(fl[g].second) : cudaEventQuery(fl[g].second);
                if (e == cudaErrorNotReady) return true;
                if (e != cudaSuccess) { fail_with(xkb_set_error(XKB_ECUDA, "task %u: device body: %s", (unsigned) (base + fl[g].first), cudaGetErrorString(e))); return false; }
                evs.push_back(fl[g].second);
                for (size_t q = 0; q <= g; ++q)
                {
                    const uint32_t d = fl.front().first;
                    fl.pop_front();
                    if (task_unref(R->pending[base + d])) task_completed(R, R->pending[base + d]);
                }
                wait = false;
            }
            return true;
        };
        for (;;)
        {
            uint32_t t;
            if (!fl.empty())
            {
                if (!retire(fl.size() >= MAX_INFLIGHT)) { leave(); return; }
                bool got = false;
                {
                    std::lock_guard<std::mutex> lk(D.mu);
                    if (D.err != XKB_OK) got = false;
                    else if (!D.ready.empty()) { t = D.ready.front(); D.ready.pop_front(); got = true; }
                }
                if (!got)
                {
                    bool err;
                    { std::lock_guard<std::mutex> lk(D.mu); err = D.err != XKB_OK; }
                    if (err) { leave(); return; }
                    if (!retire(true)) { leave(); return; }
                    continue;
                }
            }
            else
            {
                std::unique_lock<std::mutex> lk(D.mu);
                D.cv.wait_for(lk, std::chrono::milliseconds(100), [&] { return D.err != XKB_OK || D.done == nt || !D.ready.empty(); });
                if (D.err != XKB_OK || D.done == nt) { lk.unlock(); leave(); return; }
                if (D.ready.empty())
                {
                    if (D.done != seen) { seen = D.done; progress = std::chrono::steady_clock::now(); }
                    else if (ms_since(progress) > 600e3)
                    {
                        D.err = xkb_set_error(XKB_ETIMEDOUT, "xkrt_task_wait: %zu of %zu tasks completed, none for 600 s (a detached task never completed?)", D.done, nt);
                        D.err_text = xkb_last_error();
                        D.cv.notify_all();
                        lk.unlock();
                        leave();
                        return;
                    }
                    continue;
                }
                if (R->ref_mode)
                {
                    // the ready task spawned first (with one worker: the next one in spawn order)
                    auto it = std::min_element(D.ready.begin(), D.ready.end());
                    t = *it; D.ready.erase(it);
                }
                else { t = D.ready.front(); D.ready.pop_front(); }
            }
            bool deferred = false;
            const int rc = run_one(R, base + t, recs, R->wstreams[k], R->ref_mode ? nullptr : &deferred);
            if (rc) { fail_with(rc); leave(); return; }
            if (deferred)
            {
                fl.emplace_back(t, nullptr);
                if (++open >= GROUP && !close())
                { fail_with(xkb_set_error(XKB_ECUDA, "task %zu: device body", base + t)); leave(); return; }
                continue;
            }
            if (task_unref(R->pending[base + t])) task_completed(R, R->pending[base + t]);
        }
    };
    std::vector<std::thread> team;
    for (size_t k = 1; k < nw; ++k) team.emplace_back(worker, k);
    worker(0);
    for (auto & th : team) th.join();
    R->df.store(nullptr, std::memory_order_release);
    if (D.err != XKB_OK) return xkb_set_error(D.err, "%s", D.err_text.c_str());
    return XKB_OK;
}

// Page-lock the args pool up to `bytes` (rounded up to 2 MB, within the reservation) so that the
// descriptor upload of a fused batch runs at DMA speed instead of through the driver's pageable
// staging. The locked prefix is ONE registration (a copy must not span two), replaced when a
// larger batch needs more, and released with the runtime. If locking fails the pool stays
// pageable and the upload is just slower. Runs on its own thread while the wait plans coherency.
static void pin_args(xkb_runtime * R, size_t bytes)
{
    constexpr size_t STEP = size_t(2) << 20;
    if (!R->args_pool.fixed() || !R->gpu) return;
    const size_t want = std::min((bytes + STEP - 1) & ~(STEP - 1), R->args_pool.capacity_bytes());
    if (want <= R->args_pinned) return;
    cudaSetDevice(R->device);
    if (R->args_pinned)
    {
        cudaStreamSynchronize(R->stream);          // streamed windows may still copy descriptors from it
        cudaHostUnregister(R->args_pool.data());
        R->pinned_ranges.clear();
        R->args_pinned = 0;
    }
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t e = cudaHostRegister(R->args_pool.data(), want, cudaHostRegisterDefault);
    if (getenv("XKB_TRACE_WAIT"))
        fprintf(stderr, "xkrt_task_wait: page-locking %zu MB of descriptors: %s, %.1f ms\n", want >> 20, cudaGetErrorString(e),
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    if (e != cudaSuccess) { cudaGetLastError(); return; }
    R->pinned_ranges.push_back({R->args_pool.data(), want});
    R->args_pinned = want;
}

// Translate and check the built-in descriptors of tasks [t0, t1) for the device (host grid and
// vector pointers to the mirrors), into `out` when given. Otherwise dense args (one descriptor
// per task, back to back) are rewritten in place (nothing reads them as args after that), or
// `copy` receives them.
// *descs points at the result; *long_axpby tells whether some axpby task must be split.
static int translate_descs(xkb_runtime * R, size_t t0, size_t t1, std::vector<xkb_task_desc_t> & copy, xkb_task_desc_t ** descs,
                           bool * long_axpby, xkb_task_desc_t * out = nullptr)
{
    const size_t nt = t1 - t0;
    const bool dense_args = R->args_dense && !out;
    xkb_task_desc_t * d = (xkb_task_desc_t *) R->args_pool.data() + t0;
    if (out) d = out;
    else if (!dense_args) { copy.resize(nt); d = copy.data(); }
    std::atomic<size_t> bad_args(SIZE_MAX), bad_ptr(SIZE_MAX);     // first failing task, if any
    std::atomic<bool> longa(false);
    parallel_chunks(nt, [&](size_t b, size_t e) {
        RegionHint h;
        for (size_t k = b; k < e; ++k)
        {
            const size_t t = t0 + k;
            const Task & T = R->pending[t];
            if (!dense_args)
            {
                if (T.nargs < sizeof(xkb_task_desc_t)) { size_t x = bad_args; while (t < x && !bad_args.compare_exchange_weak(x, t)) {} continue; }
                memcpy(&d[k], R->args_pool.data() + T.args_off, sizeof(xkb_task_desc_t));
            }
            d[k].kind = (uint32_t) R->formats[T.fmtid].builtin;
            if (!translate_hint(R, d[k], h) || !xkb_internal_task_valid(d[k]))
            { size_t x = bad_ptr; while (t < x && !bad_ptr.compare_exchange_weak(x, t)) {} }
            if (d[k].kind == XKB_TASK_AXPBY && d[k].u.axpby.hi - d[k].u.axpby.lo > AXPBY_SPLIT && !longa)
                longa.store(true, std::memory_order_relaxed);
        }
    });
    *descs = d;
    *long_axpby = longa;
    if (bad_args != SIZE_MAX) return xkb_set_error(XKB_EINVAL, "built-in task %zu: args are not an xkb_task_desc_t", (size_t) bad_args);
    if (bad_ptr != SIZE_MAX)
        return xkb_set_error(XKB_EINVAL, "built-in task %zu: a grid or vector lies outside every registered region, or the "
                                         "tile or range is malformed", (size_t) bad_ptr);
    return XKB_OK;
}

// Warps per task: heat tiles (one warp strip covers 128 rows in FP64 and FP32) run best one warp
// per task, axpby slices two (measured on the 16384^2 graphs and the axpby chains).
static int team_for(xkb_runtime * R, const xkb_task_desc_t * d, size_t n)
{
    bool heat = true;
    for (size_t t = 0; t < n && heat; t += 1 + n / 64) heat = d[t].kind == XKB_TASK_HEAT_F32 || d[t].kind == XKB_TASK_HEAT_F64;
    return xkb_sched_set_team(R->sched, heat ? 1 : 2);
}

// Make the new distinct records of accesses [a0, a1) coherent on the device (copies issued on the
// runtime's stream, in order).
static int fetch_new_to_device(xkb_runtime * R, size_t a0, size_t a1)
{
    const size_t first = add_distinct(R, a0, a1);
    const xkb_access_rec_t * recs = R->recs.data();
    int rc = XKB_OK;
    for (size_t j = first; j < R->dfirst.size() && rc == XKB_OK; ++j)
    {
        const uint32_t k = R->dfirst[j];
        rc = xkb_planner_fetch(R->planner, &recs[k], (uint32_t) (k - R->pending[recs[k].task].acc_off), 1, nullptr);
    }
    if (rc == XKB_OK) rc = run_copies(R, R->stream);
    return rc;
}

// Streaming a window of tasks [t0, t1) (accesses [a0, a1)) to the GPU while the program keeps
// spawning, when the batch is still streamable: every task so far a built-in device body with
// one descriptor as args, no axpby long enough to be split. In two halves around the window's
// dependency resolution, so that the host work of the first half overlaps the GPU's run of the
// previous window:
//  * prepare (records converted, not yet resolved; under the planner lock, as the program may
//    register memory meanwhile): the window's new distinct records made coherent on the device
//    (copies in stream order), its descriptors translated into a page-locked slot and their copy
//    queued; *ok = false when the window cannot go (nothing done; streaming stops for the batch);
//  * launch (resolved): the window's graph (the edges among its tasks; those from earlier tasks
//    are satisfied, as the earlier windows run before it on the same stream) and one persistent
//    launch, not waited for.
static int stream_prepare(xkb_runtime * R, size_t t0, size_t t1, size_t a0, size_t a1, bool * ok)
{
    *ok = false;
    if (!R->stream_ok || !R->stream_on || !R->args_dense || !R->sched || t0 != R->streamed || t0 >= t1) return XKB_OK;
    const xkb_task_desc_t * raw = (const xkb_task_desc_t *) R->args_pool.data();
    for (size_t t = t0; t < t1; ++t)
    {
        const Task & T = R->pending[t];
        const int b = R->formats[T.fmtid].builtin;
        if (b < 0 || !is_device(R, T)) return XKB_OK;
        if (b == XKB_TASK_AXPBY && raw[t].u.axpby.hi - raw[t].u.axpby.lo > AXPBY_SPLIT) return XKB_OK;
    }
    std::lock_guard<std::mutex> lk(R->plan_mu);
    static const bool trace = getenv("XKB_TRACE_WAIT") != nullptr;
    const auto w0 = std::chrono::steady_clock::now();
    const uint64_t issued0 = trace ? xkb_internal_issued_host_copies() : 0;
    int rc = fetch_new_to_device(R, a0, a1);
    double f_ms = ms_since(w0), copy_ms = 0;
    if (trace && rc == XKB_OK)
    {
        // traces only: wait for the window's copies to see how long they take
        cudaStreamSynchronize(R->stream);
        copy_ms = ms_since(w0) - f_ms;
        fprintf(stderr, "  window coherency: %llu host copies issued, done %.1f ms after issue\n",
                (unsigned long long) (xkb_internal_issued_host_copies() - issued0), copy_ms);
        f_ms = ms_since(w0);
    }
    // a slot whose previous copy is done
    xkb_runtime::DescSlot & sl = R->dslot[R->dslot_next];
    R->dslot_next ^= 1;
    const size_t n = t1 - t0;
    if (rc == XKB_OK && sl.ev && cudaEventSynchronize(sl.ev) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt: descriptor slot");
    if (rc == XKB_OK && n > sl.cap)
    {
        if (sl.p) cudaFreeHost(sl.p);
        sl.p = nullptr; sl.cap = 0;
        const size_t c = n + n / 4;
        if (cudaHostAlloc((void **) &sl.p, c * sizeof(xkb_task_desc_t), cudaHostAllocDefault) != cudaSuccess)
            rc = xkb_set_error(XKB_ENOMEM, "xkrt: %zu page-locked descriptors", c);
        else sl.cap = c;
    }
    if (rc == XKB_OK && !sl.ev && cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming) != cudaSuccess)
        rc = xkb_set_error(XKB_ECUDA, "xkrt: event");
    std::vector<xkb_task_desc_t> copy;
    xkb_task_desc_t * descs = nullptr;
    bool longa = false;
    if (rc == XKB_OK) rc = translate_descs(R, t0, t1, copy, &descs, &longa, sl.p);
    const double d_ms = ms_since(w0) - f_ms;
    if (rc == XKB_OK) rc = team_for(R, descs, n);
    if (rc == XKB_OK) rc = xkb_internal_sched_upload_window(R->sched, descs, n);
    if (rc == XKB_OK && cudaEventRecord(sl.ev, R->stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt: event");
    if (trace)
        fprintf(stderr, "  window: coherency %.1f ms, descriptors %.1f ms, upload %.1f ms\n", f_ms, d_ms, ms_since(w0) - f_ms - d_ms);
    if (rc == XKB_OK) *ok = true;
    return rc;
}

static int stream_launch(xkb_runtime * R, const xkb_edge_mark_t & mark)
{
    xkb_task_graph_t g;
    int rc = xkb_internal_resolver_window_graph(R->res, &mark, &g);
    if (rc == XKB_OK) rc = xkb_internal_sched_launch_window(R->sched, &g);
    return rc;
}

static int wait_batch(xkb_runtime * R)
{
    R->last_tasks = R->pending.size(); R->last_edges = 0; R->last_fused = 0;
    for (double & m : R->last_ms) m = 0;
    if (R->pending.empty()) return XKB_OK;
    if (!R->gpu) return xkb_set_error(XKB_ENODEV, "xkrt_task_wait: dependency resolution runs on the GPU and none is visible");
    auto t0 = std::chrono::steady_clock::now();
    // (1) dependencies: everything not yet handed to the background worker is resolved now
    // (by the worker when it runs, so that chunks stay in spawn order; it also streams the last
    // window when it can), then the graph of the tasks not yet on the GPU is built
    const size_t nacc = R->acc_pool.size(), ntasks = R->pending.size();
    int rc = XKB_OK;
    if (R->worker.joinable())
    {
        bg_hand_over(R, true);
        bg_wait_done(R);
        if ((rc = R->bg_rc)) xkb_set_error(rc, "%s", R->bg_err.c_str());
    }
    else
        rc = resolve_range(R, 0, ntasks, 0, nacc);
    if (rc == XKB_OK && (!R->replica_pool.resize(nacc) || !R->recs.resize(nacc)))
        rc = xkb_set_error(XKB_ENOMEM, "xkrt_task_wait: out of host memory");
    if (rc)
    {
        if (R->streamed) xkb_internal_sched_windows_wait(R->sched, nullptr);      // nothing left running
        return rc;
    }
    xkb_access_rec_t * recs = R->recs.data();
    const double records_ms = ms_since(t0);
    // tasks [P, ntasks) still to run; [0, P) were streamed to the GPU during the spawns
    const size_t P = R->streamed;
    const size_t a_P = P < ntasks ? R->pending[P].acc_off : nacc;
    xkb_resolver_t * res = R->res;
    xkb_task_graph_t g{};
    if (P == 0) rc = xkb_resolver_graph(res, &g);
    else if (P < ntasks) rc = xkb_internal_resolver_window_graph(res, &R->rest_mark, &g);
    if (rc) { if (P) xkb_internal_sched_windows_wait(R->sched, nullptr); return rc; }
    R->last_edges = P == 0 ? g.nedges : xkb_internal_resolver_nedges(res);
    R->last_ms[0] = ms_since(t0);
    if (getenv("XKB_TRACE_WAIT"))
        fprintf(stderr, "xkrt_task_wait: %zu records %.1f ms, resolver %.1f ms, %zu of %zu tasks streamed (at %.1f ms)\n", nacc,
                records_ms, R->last_ms[0] - records_ms, P, ntasks, trace_clock_ms());

    bool fused = !R->ref_mode;       // reference mode: every task through the dataflow path, one at a time
    for (size_t t = P; t < ntasks && fused; ++t) fused = is_device(R, R->pending[t]) && R->formats[R->pending[t].fmtid].builtin >= 0;

    const bool all_streamed = fused && P == ntasks;
    if (all_streamed)
    {
        // every window already on the GPU: the write-back below is planned and its copies queued
        // behind the last windows while they run; the wait for them comes after it
        R->last_fused = 1;
    }
    else if (fused)
    {
        // (2) every access made coherent on the device up front: with no host task in the batch
        // the host data cannot change meanwhile, so the first-touch copies can all go first.
        // Meanwhile another thread page-locks the descriptors for their upload.
        t0 = std::chrono::steady_clock::now();
        std::thread pinner;
        if (R->args_dense) pinner = std::thread(pin_args, R, ntasks * sizeof(xkb_task_desc_t));
        rc = fetch_new_to_device(R, a_P, nacc);
        const double fetch_ms = ms_since(t0);
        std::vector<xkb_task_desc_t> copy;
        xkb_task_desc_t * descs = nullptr;
        bool long_axpby = false;
        const size_t nt = ntasks - P;
        if (rc == XKB_OK) rc = translate_descs(R, P, ntasks, copy, &descs, &long_axpby);
        if (pinner.joinable()) pinner.join();
        const double desc_ms = ms_since(t0) - fetch_ms;
        SplitGraph sg;
        bool split = false;
        if (rc == XKB_OK && long_axpby) rc = split_moldable(descs, nt, g, sg, split);
        const xkb_task_graph_t & run_g = split ? sg.g : g;
        const xkb_task_desc_t * run_d = split ? sg.descs.data() : descs;
        const size_t run_n = split ? sg.descs.size() : nt;
        if (rc == XKB_OK) rc = team_for(R, run_d, run_n);
        if (P == 0)
        {
            if (rc == XKB_OK) rc = xkb_internal_sched_set_tasks_device(R->sched, run_d, run_n, true);
            if (getenv("XKB_TRACE_WAIT"))
                fprintf(stderr, "xkrt_task_wait: fetches + copies %.1f ms, descriptors %.1f ms, upload %.1f ms\n", fetch_ms, desc_ms,
                        ms_since(t0) - fetch_ms - desc_ms);
            if (rc == XKB_OK && cudaStreamSynchronize(R->stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: stream");
            R->last_ms[1] = ms_since(t0);
            t0 = std::chrono::steady_clock::now();
            if (rc == XKB_OK) rc = xkb_sched_run(R->sched, &run_g, XKB_FORM_PERSISTENT);
            uint64_t ran = 0;
            if (rc == XKB_OK) rc = xkb_sched_wait(R->sched, &ran);
        }
        else
        {
            // the rest of a streamed batch: one more window behind the streamed ones
            if (rc == XKB_OK) rc = xkb_internal_sched_run_window(R->sched, run_d, run_n, &run_g);
            R->last_ms[1] = ms_since(t0);
            t0 = std::chrono::steady_clock::now();
            uint64_t ran = 0;
            const int wrc = xkb_internal_sched_windows_wait(R->sched, &ran);
            if (rc == XKB_OK) rc = wrc;
        }
        R->last_ms[2] = ms_since(t0);
        R->last_fused = 1;
    }
    else
    {
        // (3) the rest of the batch as a dataflow graph on a team of host threads, once the
        // streamed windows (its completed predecessors) are done
        t0 = std::chrono::steady_clock::now();
        if (P) rc = xkb_internal_sched_windows_wait(R->sched, nullptr);
        // a batch of device tasks only (program-defined CUDA bodies included): as for a fused
        // batch, host data cannot change while it runs, so every access is made coherent on the
        // device up front and the team's tasks skip the planner (and its lock)
        if (rc == XKB_OK && !R->ref_mode) rc = preplan_device_batch(R, P, ntasks, a_P, nacc);
        if (rc == XKB_OK) rc = run_dataflow(R, g, recs, P);
        R->preplanned = false;
        if (rc == XKB_OK && cudaStreamSynchronize(R->stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: stream");
        R->last_ms[2] = ms_since(t0);
    }
    // (4) host memory coherent again: read back every block a device task wrote
    if (rc == XKB_OK)
    {
        t0 = std::chrono::steady_clock::now();
        // every block whose only coherent copy is on the GPU (exactly the blocks device tasks
        // wrote: each wait leaves the host coherent), one walk over the planner's partition;
        // reference mode: the reference's fetch to the host of every written access
        // (memory_coherent_async's host reads, src/memory/coherent.cc:137-231), in spawn order
        if (R->ref_mode)
        {
            rc = apply_registrations(R, SIZE_MAX);
            for (size_t t = P; t < ntasks && rc == XKB_OK; ++t)
            {
                const Task & T = R->pending[t];
                if (!is_device(R, T)) continue;
                for (uint32_t a = 0; a < T.nacc && rc == XKB_OK; ++a)
                {
                    const xkb_access_rec_t & r = recs[T.acc_off + a];
                    if ((r.type == XKB_ACCESS_TYPE_BLAS_MATRIX || r.type == XKB_ACCESS_TYPE_SEGMENT) && (r.mode & XKB_ACCESS_MODE_W))
                        rc = xkb_planner_fetch(R->planner, &r, a, 0, nullptr);
                }
            }
        }
        else
            rc = xkb_planner_flush_to_host(R->planner);
        const double fetch_ms = ms_since(t0);
        if (rc == XKB_OK) rc = run_copies(R, R->stream);
        if (all_streamed)
        {
            // the windows (and the copies queued behind them) end here
            const auto tw = std::chrono::steady_clock::now();
            uint64_t ran = 0;
            const int wrc = xkb_internal_sched_windows_wait(R->sched, &ran);
            if (rc == XKB_OK) rc = wrc;
            R->last_ms[2] = ms_since(tw);
        }
        if (rc == XKB_OK && cudaStreamSynchronize(R->stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: stream");
        R->last_ms[3] = ms_since(t0) - (all_streamed ? R->last_ms[2] : 0.0);
        if (getenv("XKB_TRACE_WAIT"))
            fprintf(stderr, "xkrt_task_wait: write-back fetches %.1f ms, copies %.1f ms\n", fetch_ms, R->last_ms[3] - fetch_ms);
    }
    return rc;
}

extern "C" int xkb_runtime_last_wait_bytes(xkrt_runtime_t * runtime, uint64_t * h2d_bytes, uint64_t * d2h_bytes)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return xkb_set_error(XKB_EINVAL, "xkb_runtime_last_wait_bytes: null runtime");
    if (h2d_bytes) *h2d_bytes = R->last_h2d_bytes;
    if (d2h_bytes) *d2h_bytes = R->last_d2h_bytes;
    return XKB_OK;
}

extern "C" int xkb_runtime_last_wait_times(xkrt_runtime_t * runtime, double * resolve_ms, double * coherency_ms, double * run_ms,
                                           double * writeback_ms)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return xkb_set_error(XKB_EINVAL, "xkb_runtime_last_wait_times: null runtime");
    if (resolve_ms) *resolve_ms = R->last_ms[0];
    if (coherency_ms) *coherency_ms = R->last_ms[1];
    if (run_ms) *run_ms = R->last_ms[2];
    if (writeback_ms) *writeback_ms = R->last_ms[3];
    return XKB_OK;
}

extern "C" void xkrt_task_wait(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return;
    R->in_wait = true;
    const auto w0 = std::chrono::steady_clock::now();
    fail(R, wait_batch(R));
    const double wb_ms = ms_since(w0);
    bg_finish(R);
    if (getenv("XKB_TRACE_WAIT")) fprintf(stderr, "xkrt_task_wait: %.1f ms in all, %.1f ms to finish\n", wb_ms, ms_since(w0) - wb_ms);
    R->last_h2d = R->cur_h2d; R->last_d2h = R->cur_d2h; R->last_h2d_bytes = R->cur_h2d_bytes; R->last_d2h_bytes = R->cur_d2h_bytes;
    R->cur_h2d = R->cur_d2h = R->cur_h2d_bytes = R->cur_d2h_bytes = R->cur_d2d = 0;
    R->in_wait = false;
    R->pending.clear(); R->args_pool.clear(); R->acc_pool.clear(); R->replica_pool.clear(); R->recs.clear();
    R->args_dense = true;
}

// ---- C++ source API bridge (include/xkrt/b200/api.hpp) ----------------------------------------

extern "C" void xkb_cxx_bind(xkrt_runtime_t * runtime, void * cxx_runtime)
{
    if (xkb_runtime * R = RT(runtime)) R->cxx_rt = cxx_runtime;
}

// A hand-built task joins the batch like a spawned one: its accesses (the first dep_info->ac of
// them when it is DEPENDENT) become the C API's access records, its target the device the
// runtime runs it on (TASK_FLAG_DEVICE: the targeted device, or the GPU when unspecified), its
// detachable counter's initial value is kept (src/task.cc:249-288), and its body gets the task.
extern "C" void xkb_cxx_commit(xkrt_runtime_t * runtime, void * task)
{
    xkb_runtime * R = RT(runtime);
    xkrt::task_t * t = (xkrt::task_t *) task;
    if (!R || !t || t->magic != xkrt::TASK_MAGIC)
    {
        fail(R, xkb_set_error(XKB_EINVAL, "task_commit: not a task built with the C++ source API"));
        return;
    }
    const uint8_t flags = t->flags & ~TASK_FLAG_REQUEUE;
    const size_t n = (flags & TASK_FLAG_DEPENDENT) ? xkrt::TASK_DEP_INFO(t)->ac : 0;
    static thread_local std::vector<xkrt_access_t> acc;
    acc.resize(n);
    const xkrt::access_t * a = n ? xkrt::TASK_ACCESSES(t) : nullptr;
    for (size_t i = 0; i < n; ++i)
    {
        xkrt_access_t & c = acc[i];
        memset(&c, 0, sizeof(c));
        c.concurrency = a[i].concurrency; c.mode = a[i].mode; c.scope = a[i].scope; c.type = a[i].type;
        const xkrt::memory_view_t & h = a[i].host_view;
        if (c.type == ACCESS_TYPE_HANDLE) c.region.handle.addr = (void *) h.addr;
        else if (c.type == ACCESS_TYPE_SEGMENT) { c.region.segment.a = (void *) h.addr; c.region.segment.b = (void *) (h.addr + h.m); }
        else if (c.type == ACCESS_TYPE_BLAS_MATRIX)
            c.region.matrix = {h.storage, (void *) h.addr, h.ld, h.offset_m, h.offset_n, h.m, h.n, h.sizeof_type};
    }
    xkrt_device_global_id_t device = HOST_DEVICE_GLOBAL_ID;
    if (flags & TASK_FLAG_DEVICE)
    {
        device = xkrt::TASK_DEV_INFO(t)->targeted_device_id;
        if (device == UNSPECIFIED_DEVICE_GLOBAL_ID || device > 1) device = R->gpu ? 1 : HOST_DEVICE_GLOBAL_ID;
        xkrt::TASK_DEV_INFO(t)->elected_device_id = device;
    }
    const int detach0 = (flags & TASK_FLAG_DETACHABLE) ? (int) xkrt::TASK_DET_INFO(t)->wc.load() : 0;
    if (flags & TASK_FLAG_DEPENDENT) xkrt::TASK_DEP_INFO(t)->wc.store(0);
    spawn(R, device, flags, t->fmtid, nullptr, 0, acc.data(), n, nullptr, nullptr, t, detach0);
}

// +1: detachable_incr, -1: detachable_decr, 0: complete -- on the batch task a commit made.
extern "C" void xkb_cxx_detachable(xkrt_runtime_t * runtime, void * task, int delta)
{
    xkb_runtime * R = RT(runtime);
    xkrt::task_t * t = (xkrt::task_t *) task;
    if (!R || !t || t->magic != xkrt::TASK_MAGIC || t->impl >= R->pending.size() || cxx_of(R->pending[t->impl]) != task)
    {
        fail(R, xkb_set_error(XKB_EINVAL, "task_detachable: not a committed task of this runtime"));
        return;
    }
    xkrt_task_t * T = (xkrt_task_t *) &R->pending[t->impl];
    if (delta > 0) xkrt_task_detachable_incr(runtime, T);
    else if (delta < 0) xkrt_task_detachable_decr(runtime, T);
    else xkrt_task_complete(runtime, T);
}

// The launcher gets the C++ runtime, the device, the task and a queue_cu_t whose stream is the one
// of the thread running the CUDA body and whose event 0 the launcher may record (the reference's
// launcher records it to signal completion, src/sched.cc:469-505); the task completes when the
// stream's work did.
extern "C" void xkb_cxx_kernel_launch(xkrt_runtime_t * runtime, void * device, void * task, int synchronous,
                                      xkrt_kernel_launcher_t launcher)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !launcher) { fail(R, xkb_set_error(XKB_EINVAL, "task_kernel_launch: no runtime or launcher")); return; }
    if (!g_stream) { fail(R, xkb_set_error(XKB_EINVAL, "task_kernel_launch: called outside a CUDA task body")); return; }
    static thread_local cudaEvent_t ev = nullptr;
    if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
    {
        fail(R, xkb_set_cuda_error(cudaGetLastError()));
        return;
    }
    xkrt::queue_cu_t q;
    q.driver_type = XKRT_DRIVER_TYPE_CUDA; q.qtype = XKRT_QUEUE_TYPE_KERN;
    q.cu.handle.high = q.cu.handle.low = g_stream;
    q.cu.events.buffer = &ev; q.cu.events.capacity = 1;
    launcher(R->cxx_rt, device, task, &q, nullptr, 0);
    if (synchronous && cudaStreamSynchronize(g_stream) != cudaSuccess) fail(R, xkb_set_cuda_error(cudaGetLastError()));
}

// Task memory of a thread: 64-byte aligned pieces of 64 MiB chunks (pages backed on first touch),
// never freed one by one -- the reference's per-thread task stack (src/thread/thread.cc:105-124).
namespace {
struct TaskArena {
    std::vector<std::pair<void *, size_t>> chunks;
    uint8_t * cur = nullptr;
    size_t left = 0;
    void release()
    {
        for (auto & c : chunks) munmap(c.first, c.second);
        chunks.clear(); cur = nullptr; left = 0;
    }
    ~TaskArena() { release(); }
};
thread_local TaskArena g_task_arena;
} // namespace

extern "C" void * xkb_cxx_allocate_task(size_t size)
{
    TaskArena & A = g_task_arena;
    size = (size + 63) & ~(size_t) 63;
    if (size > A.left)
    {
        const size_t chunk = std::max<size_t>(size_t(64) << 20, (size + 4095) & ~(size_t) 4095);
        void * p = mmap(nullptr, chunk, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE, -1, 0);
        if (p == MAP_FAILED) return nullptr;
        A.chunks.emplace_back(p, chunk);
        A.cur = (uint8_t *) p; A.left = chunk;
    }
    void * r = A.cur;
    A.cur += size; A.left -= size;
    return r;
}

extern "C" void xkb_cxx_release_tasks(void) { g_task_arena.release(); }
