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
// runs as one persistent-scheduler launch, any other batch runs task by task in spawn order
// (a topological order). Host memory is coherent again when xkrt_task_wait returns.
#include "common.cuh"
#include "internal.h"
#include "../../include/xkrt_capi.h"

#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

namespace {

struct Format {
    bool used = false;
    std::string label;
    xkrt_task_format_func_t f[XKRT_TASK_FORMAT_TARGET_MAX] = {};
    int builtin = -1;                     // XKB_TASK_* for built-in device bodies
};

struct Task {
    uint8_t fmtid = 0, flags = 0;
    xkrt_device_global_id_t device = 0;
    std::vector<uint8_t> args;
    std::vector<xkrt_access_t> acc;
    std::vector<void *> replica;
    xkrt_task_func_t func = nullptr;      // team / plain function spawns
    void * user_data = nullptr;
};

struct Region { uint64_t size; void * mirror; bool pinned_by_us; int32_t id; };

} // namespace

struct xkb_runtime {
    Format formats[256];
    int next_fmtid = 1;
    std::vector<std::unique_ptr<Task>> pending;
    std::map<uint64_t, Region> regions;               // host base -> region
    xkb_planner_t * planner = nullptr;
    xkb_sched_t * sched = nullptr;
    cudaStream_t stream = nullptr;
    bool gpu = false;
    int status = XKB_OK;
    uint64_t last_tasks = 0, last_edges = 0, last_h2d = 0, last_d2h = 0;
    int last_fused = 0;
    int dummy_team = 0;
};

static xkb_runtime * RT(xkrt_runtime_t * r) { return (xkb_runtime *) r; }

static void fail(xkb_runtime * R, int rc)
{
    if (R && rc != XKB_OK && R->status == XKB_OK) R->status = rc;
}

extern "C" int xkrt_init(xkrt_runtime_t ** out)
{
    if (!out) return xkb_set_error(XKB_EINVAL, "xkrt_init: null output");
    xkb_runtime * R = new (std::nothrow) xkb_runtime();
    if (!R) return xkb_set_error(XKB_ENOMEM, "xkrt_init: out of host memory");
    int n = 0;
    R->gpu = cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
    int rc = xkb_planner_create_resident(&R->planner);
    if (rc == XKB_OK && R->gpu)
    {
        if (cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_init: stream");
        else rc = xkb_sched_create(&R->sched, R->stream);
    }
    if (rc) { delete R; return rc; }
    *out = (xkrt_runtime_t *) R;
    return XKB_OK;
}

extern "C" int xkrt_deinit(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return xkb_set_error(XKB_EINVAL, "xkrt_deinit: null runtime");
    if (!R->pending.empty()) xkrt_task_wait(runtime);
    if (R->stream) cudaStreamSynchronize(R->stream);
    for (auto & kv : R->regions)
    {
        if (kv.second.mirror) cudaFree(kv.second.mirror);
        if (kv.second.pinned_by_us) cudaFreeHost((void *) kv.first);
    }
    if (R->sched) xkb_sched_destroy(R->sched);
    if (R->planner) xkb_planner_destroy(R->planner);
    if (R->stream) cudaStreamDestroy(R->stream);
    const int st = R->status;
    delete R;
    return st;
}

extern "C" void xkrt_reset(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (R) R->pending.clear();
}

static int add_region(xkb_runtime * R, void * ptr, size_t size, bool pinned)
{
    int32_t id = -1;
    int rc = xkb_planner_add_region(R->planner, (uint64_t) ptr, size, &id);
    if (rc) return rc;
    void * mirror = nullptr;
    if (R->gpu)
    {
        cudaError_t e = cudaMalloc(&mirror, size);
        if (e != cudaSuccess) return xkb_set_cuda_error(e);
    }
    R->regions[(uint64_t) ptr] = Region{size, mirror, pinned, id};
    return XKB_OK;
}

extern "C" int xkrt_memory_register(xkrt_runtime_t * runtime, void * ptr, size_t size)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !ptr || !size) return xkb_set_error(XKB_EINVAL, "xkrt_memory_register: bad arguments");
    if (R->gpu) cudaHostRegister(ptr, size, cudaHostRegisterDefault);     // pinned copies when possible
    cudaGetLastError();
    return add_region(R, ptr, size, false);
}

extern "C" int xkrt_memory_unregister(xkrt_runtime_t * runtime, void * ptr, size_t size)
{
    xkb_runtime * R = RT(runtime);
    if (!R || !ptr) return xkb_set_error(XKB_EINVAL, "xkrt_memory_unregister: bad arguments");
    (void) size;
    if (R->gpu) { cudaHostUnregister(ptr); cudaGetLastError(); }
    return XKB_OK;                       // the mirror stays until xkrt_deinit
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
    const int s = R->status;
    R->status = XKB_OK;
    return s;
}

extern "C" void * xkb_runtime_stream(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    return R ? (void *) R->stream : nullptr;
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

static void spawn(xkb_runtime * R, xkrt_device_global_id_t device, xkrt_task_flag_bitfield_t flags, xkrt_task_format_id_t fmtid,
                  const void * args, size_t args_size, const xkrt_access_t * acc, size_t nacc, xkrt_task_func_t func, void * ud)
{
    if (!R) return;
    if (nacc && !acc) { fail(R, xkb_set_error(XKB_EINVAL, "spawn: null accesses")); return; }
    for (size_t i = 0; i < nacc; ++i)
        if (acc[i].type == ACCESS_TYPE_HANDLE)
        { fail(R, xkb_set_error(XKB_EINVAL, "spawn: handle accesses are not supported")); return; }
    std::unique_ptr<Task> t(new (std::nothrow) Task());
    if (!t) { fail(R, XKB_ENOMEM); return; }
    t->fmtid = fmtid; t->flags = flags; t->device = device;
    if (args_size) t->args.assign((const uint8_t *) args, (const uint8_t *) args + args_size);
    t->acc.assign(acc, acc + nacc);
    t->replica.assign(nacc, nullptr);
    t->func = func; t->user_data = ud;
    R->pending.push_back(std::move(t));
}

extern "C" void xkrt_task_spawn_generic(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                        const xkrt_task_flag_bitfield_t flags, const xkrt_task_format_id_t fmtid,
                                        const void * args, const size_t args_size, const xkrt_access_t * accesses,
                                        const xkrt_task_access_counter_type_t naccesses,
                                        const xkrt_task_access_counter_type_t ocr_access,
                                        const xkrt_task_wait_counter_type_t detachable_counter_initial)
{
    (void) ocr_access; (void) detachable_counter_initial;
    spawn(RT(runtime), device_global_id, flags, fmtid, args, args_size, accesses, naccesses, nullptr, nullptr);
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

// ---- task accessors --------------------------------------------------------------------------

extern "C" void * xkrt_task_args(xkrt_task_t * task) { Task * t = (Task *) task; return t && !t->args.empty() ? t->args.data() : nullptr; }
extern "C" xkrt_access_t * xkrt_task_accesses(xkrt_task_t * task) { Task * t = (Task *) task; return t && !t->acc.empty() ? t->acc.data() : nullptr; }
extern "C" xkrt_access_t * xkrt_task_access(xkrt_task_t * task, xkrt_task_access_counter_type_t i)
{
    Task * t = (Task *) task;
    return t && i < t->acc.size() ? &t->acc[i] : nullptr;
}
extern "C" void * xkrt_task_access_replica(xkrt_task_t * task, xkrt_task_access_counter_type_t i)
{
    Task * t = (Task *) task;
    return t && i < t->replica.size() ? t->replica[i] : nullptr;
}

// ---- wait --------------------------------------------------------------------------------------

static bool to_rec(const xkrt_access_t & a, uint32_t task, xkb_access_rec_t & r)
{
    memset(&r, 0, sizeof(r));
    r.task = task;
    r.mode = (uint8_t) a.mode;
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
    return (t.flags & TASK_FLAG_DEVICE) && t.device != HOST_DEVICE_GLOBAL_ID && (f.builtin >= 0 || f.f[XKRT_TASK_FORMAT_TARGET_CUDA]);
}

static void * mirror_of(xkb_runtime * R, uint64_t host)
{
    auto it = R->regions.upper_bound(host);
    if (it == R->regions.begin()) return nullptr;
    --it;
    if (host >= it->first + it->second.size || !it->second.mirror) return nullptr;
    return (uint8_t *) it->second.mirror + (host - it->first);
}

static int run_copies(xkb_runtime * R)
{
    size_t n = 0;
    int rc = xkb_planner_copies(R->planner, nullptr, 0, &n, 0);
    if (rc || !n) return rc;
    std::vector<xkb_copy_t> c(n);
    if ((rc = xkb_planner_copies(R->planner, c.data(), n, &n, 1))) return rc;
    std::vector<void *> ptrs(R->regions.size(), nullptr);
    for (auto & kv : R->regions) ptrs[kv.second.id] = kv.second.mirror;
    for (const xkb_copy_t & k : c) (k.kind == XKB_COPY_H2D ? R->last_h2d : R->last_d2h) += 1;
    return xkb_plan_execute(c.data(), n, ptrs.data(), ptrs.size(), R->stream);
}

// Point a built-in descriptor's host addresses at the device mirrors.
static int translate(xkb_runtime * R, xkb_task_desc_t & d)
{
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        void * s = mirror_of(R, d.u.heat.src), * t = mirror_of(R, d.u.heat.dst);
        if (!s || !t) return xkb_set_error(XKB_EINVAL, "heat task: grid outside every registered region");
        d.u.heat.src = (uint64_t) s; d.u.heat.dst = (uint64_t) t;
    }
    else if (d.kind == XKB_TASK_AXPBY)
    {
        void * x = mirror_of(R, d.u.axpby.x), * y = mirror_of(R, d.u.axpby.y);
        if (!x || !y) return xkb_set_error(XKB_EINVAL, "axpby task: vector outside every registered region");
        d.u.axpby.x = (uint64_t) x; d.u.axpby.y = (uint64_t) y;
    }
    return XKB_OK;
}

static int wait_batch(xkb_runtime * R)
{
    R->last_tasks = R->pending.size(); R->last_edges = 0; R->last_h2d = R->last_d2h = 0; R->last_fused = 0;
    if (R->pending.empty()) return XKB_OK;
    if (!R->gpu) return xkb_set_error(XKB_ENODEV, "xkrt_task_wait: dependency resolution runs on the GPU and none is visible");
    // (1) dependencies
    std::vector<xkb_access_rec_t> recs;
    std::vector<std::pair<size_t, size_t>> rec_of;      // (task, access) of every record
    for (size_t t = 0; t < R->pending.size(); ++t)
        for (size_t a = 0; a < R->pending[t]->acc.size(); ++a)
        {
            xkb_access_rec_t r;
            if (to_rec(R->pending[t]->acc[a], (uint32_t) t, r)) { recs.push_back(r); rec_of.push_back({t, a}); }
        }
    xkb_resolver_t * res = nullptr;
    int rc = xkb_resolver_create(&res, R->stream);
    if (rc) return rc;
    // every task needs a record for the task numbering to stay dense: a task without data
    // accesses gets a zero-byte stand-in? -- no: give it a one-byte virtual read of its own
    // descriptor, which nothing else touches
    std::vector<xkb_access_rec_t> all;
    {
        size_t k = 0;
        for (size_t t = 0; t < R->pending.size(); ++t)
        {
            bool any = false;
            while (k < recs.size() && recs[k].task == t) { all.push_back(recs[k++]); any = true; }
            if (!any)
            {
                xkb_access_rec_t r;
                memset(&r, 0, sizeof(r));
                r.task = (uint32_t) t; r.type = XKB_ACCESS_TYPE_SEGMENT; r.mode = XKB_ACCESS_MODE_R | XKB_ACCESS_MODE_V;
                r.addr = (uint64_t) R->pending[t].get(); r.ld = r.addr + 1;
                all.push_back(r);
            }
        }
    }
    rc = xkb_resolver_add(res, all.data(), all.size());
    xkb_task_graph_t g;
    if (rc == XKB_OK) rc = xkb_resolver_graph(res, &g);
    if (rc) { xkb_resolver_destroy(res); return rc; }
    R->last_edges = g.nedges;

    bool fused = true;
    for (auto & t : R->pending) if (!is_device(R, *t) || R->formats[t->fmtid].builtin < 0) { fused = false; break; }

    if (fused)
    {
        // (2) every access made coherent on the device up front: with no host task in the batch
        // the host data cannot change meanwhile, so the first-touch copies can all go first
        for (size_t k = 0; k < recs.size(); ++k)
            if ((rc = xkb_planner_fetch(R->planner, &recs[k], (uint32_t) rec_of[k].second, 1, nullptr))) break;
        if (rc == XKB_OK) rc = run_copies(R);
        std::vector<xkb_task_desc_t> descs(R->pending.size());
        for (size_t t = 0; t < R->pending.size() && rc == XKB_OK; ++t)
        {
            if (R->pending[t]->args.size() < sizeof(xkb_task_desc_t)) { rc = xkb_set_error(XKB_EINVAL, "built-in task %zu: args are not an xkb_task_desc_t", t); break; }
            memcpy(&descs[t], R->pending[t]->args.data(), sizeof(xkb_task_desc_t));
            descs[t].kind = (uint32_t) R->formats[R->pending[t]->fmtid].builtin;
            rc = translate(R, descs[t]);
        }
        if (rc == XKB_OK) rc = xkb_sched_set_tasks(R->sched, descs.data(), descs.size());
        if (rc == XKB_OK) rc = xkb_sched_run(R->sched, &g, XKB_FORM_PERSISTENT);
        uint64_t ran = 0;
        if (rc == XKB_OK) rc = xkb_sched_wait(R->sched, &ran);
        R->last_fused = 1;
    }
    else
    {
        // (3) task by task in spawn order
        size_t k = 0;
        for (size_t t = 0; t < R->pending.size() && rc == XKB_OK; ++t)
        {
            Task & T = *R->pending[t];
            const bool dev = is_device(R, T);
            for (; k < recs.size() && rec_of[k].first == t; ++k)
            {
                const uint64_t begin = recs[k].type == XKB_ACCESS_TYPE_SEGMENT ? recs[k].addr
                                     : recs[k].addr + (recs[k].offset_n * recs[k].ld + recs[k].offset_m) * recs[k].sizeof_type;
                T.replica[rec_of[k].second] = dev ? mirror_of(R, begin) : (void *) begin;
                // a host task on memory no region covers: that memory never has a device copy
                if (!dev && !mirror_of(R, begin)) continue;
                xkb_view_t v;
                if ((rc = xkb_planner_fetch(R->planner, &recs[k], (uint32_t) rec_of[k].second, dev ? 1 : 0, &v))) break;
            }
            if (rc) break;
            if ((rc = run_copies(R))) break;
            const Format & f = R->formats[T.fmtid];
            if (dev)
            {
                if (f.builtin >= 0)
                {
                    xkb_task_desc_t d;
                    if (T.args.size() < sizeof(d)) { rc = xkb_set_error(XKB_EINVAL, "built-in task %zu: args are not an xkb_task_desc_t", t); break; }
                    memcpy(&d, T.args.data(), sizeof(d));
                    d.kind = (uint32_t) f.builtin;
                    if ((rc = translate(R, d)) || (rc = xkb_internal_launch_task(&d, R->stream))) break;
                }
                else
                    ((void (*)(xkrt_runtime_t *, xkrt_device_t *, xkrt_task_t *)) f.f[XKRT_TASK_FORMAT_TARGET_CUDA])(
                        (xkrt_runtime_t *) R, (xkrt_device_t *) (uintptr_t) 1, (xkrt_task_t *) &T);
            }
            else
            {
                if (cudaStreamSynchronize(R->stream) != cudaSuccess) { rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: stream"); break; }
                if (T.func) T.func((xkrt_runtime_t *) R, (xkrt_device_t *) nullptr, (xkrt_task_t *) &T, T.user_data);
                else if (f.f[XKRT_TASK_FORMAT_TARGET_HOST])
                    ((void (*)(xkrt_runtime_t *, xkrt_device_t *, xkrt_task_t *)) f.f[XKRT_TASK_FORMAT_TARGET_HOST])(
                        (xkrt_runtime_t *) R, (xkrt_device_t *) nullptr, (xkrt_task_t *) &T);
                else if (T.fmtid) { rc = xkb_set_error(XKB_EINVAL, "task %zu: its format has no host body", t); break; }
            }
        }
    }
    // (4) host memory coherent again: read back every block a device task wrote
    if (rc == XKB_OK)
    {
        for (size_t k = 0; k < recs.size() && rc == XKB_OK; ++k)
            if ((recs[k].mode & XKB_ACCESS_MODE_W) && is_device(R, *R->pending[rec_of[k].first]))
            {
                xkb_access_rec_t r = recs[k];
                r.mode = XKB_ACCESS_MODE_R;
                rc = xkb_planner_fetch(R->planner, &r, 0, 0, nullptr);
            }
        if (rc == XKB_OK) rc = run_copies(R);
        if (rc == XKB_OK && cudaStreamSynchronize(R->stream) != cudaSuccess) rc = xkb_set_error(XKB_ECUDA, "xkrt_task_wait: stream");
    }
    xkb_resolver_destroy(res);
    return rc;
}

extern "C" void xkrt_task_wait(xkrt_runtime_t * runtime)
{
    xkb_runtime * R = RT(runtime);
    if (!R) return;
    fail(R, wait_batch(R));
    R->pending.clear();
}
