// Reference-backed transfer-plan oracle (test infrastructure; never part of the product).
//
// Drives the reference's own coherency controller, KBLASMemoryTree::fetch
// (include/xkrt/memory/access/blas/memory-tree.hpp:1805-1874), for one host (device 0) and one
// GPU (device 1) under the CANONICAL schedule: tasks in spawn order, each task's accesses in
// declaration order, every access fetched to device 1, and every copy it issues completed
// (its callback run, FIFO, including copies issued by callbacks) before the next fetch.
// An access whose record has bit 0 of `reserved` set is fetched to the host instead (a host
// task's access: write-back, fetch_list_to_host :1185-1215).
// Device allocation and copies go through link seams (oracle/ref/seams.cc): allocation k
// gets the fake device address (k + 1) << 40, so device addresses decode into
// (allocation ordinal, byte offset).
//
// Output <out>.plan : int64 records {task, access, kind(0 H2D, 1 D2H, 2 D2D), src_dev, src_alloc,
//                     src_off, src_ld, dst_dev, dst_alloc, dst_off, dst_ld, m, n, sizeof}
//                     (host endpoints: alloc = -1, off = host byte address)
//        <out>.allocs: int64 {bytes} per allocation, in allocation order
//        <out>.views : int64 {task, access, alloc, off, ld} -- the device view each access gets
//        stdout      : one JSON line of counts
//
// Optional third argument: a file of int64 registration events {before_task, kind (1 register,
// 2 unregister), ptr, size}, applied before the first fetch of task `before_task` the way
// runtime_t::memory_register / memory_unregister (src/memory/register.cc:89-262) tell the trees
// of the calling task's domain under the reference's default build (overflow protection, page
// rounding and assisted registration on; one driver that registers host memory): the range is
// rounded out to pages (include/xkrt/memory/pageas.h), only its pieces not yet registered
// (register) or its registered intervals (unregister) go to every existing tree
// (KBLASMemoryTree::registered / unregistered, memory-tree.hpp:2184-2240), and a tree created
// later first receives every registered piece (src/task/task.cc:88-94, 127-133).
#include <xkrt/runtime.h>
#include <xkrt/task/task.hpp>
#include <xkrt/memory/access/access.hpp>
#include <xkrt/memory/access/blas/memory-tree.hpp>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <deque>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include <xkrt/memory/access/common/interval-set.hpp>
#include <xkrt/memory/pageas.h>

#include <algorithm>
#include <array>

#include "../access_stream.h"
#include "seams.h"

XKRT_NAMESPACE_USE;

static const int64_t FAKE_SHIFT = 40;
static std::vector<int64_t> g_allocs;
static std::vector<std::array<int64_t, 14>> g_plan;
static std::deque<callback_t> g_pending;
static int64_t g_task = -1, g_access = -1;

static void decode(device_global_id_t dev, uintptr_t addr, int64_t & alloc, int64_t & off)
{
    if (dev == HOST_DEVICE_GLOBAL_ID) { alloc = -1; off = (int64_t) addr; return; }
    alloc = (int64_t) (addr >> FAKE_SHIFT) - 1;
    off = (int64_t) (addr & ((1ull << FAKE_SHIFT) - 1));
}

static void record(device_global_id_t dst_dev, uintptr_t dst, size_t dst_ld, device_global_id_t src_dev,
                   uintptr_t src, size_t src_ld, size_t m, size_t n, size_t s)
{
    std::array<int64_t, 14> r;
    r[0] = g_task; r[1] = g_access;
    r[2] = src_dev == HOST_DEVICE_GLOBAL_ID ? 0 : (dst_dev == HOST_DEVICE_GLOBAL_ID ? 1 : 2);
    r[3] = src_dev; decode(src_dev, src, r[4], r[5]); r[6] = (int64_t) src_ld;
    r[7] = dst_dev; decode(dst_dev, dst, r[8], r[9]); r[10] = (int64_t) dst_ld;
    r[11] = (int64_t) m; r[12] = (int64_t) n; r[13] = (int64_t) s;
    g_plan.push_back(r);
}

static void hook_copy2d(runtime_t *, device_global_id_t, const memory_view_t & host_view, device_global_id_t dst_dev,
                        const memory_replica_view_t & dst, device_global_id_t src_dev,
                        const memory_replica_view_t & src, const callback_t & cb)
{
    record(dst_dev, dst.addr, dst.ld, src_dev, src.addr, src.ld, host_view.m, host_view.n, host_view.sizeof_type);
    g_pending.push_back(cb);
}

static void hook_copy1d(runtime_t *, device_global_id_t, size_t size, device_global_id_t dst_dev, uintptr_t dst,
                        device_global_id_t src_dev, uintptr_t src, const callback_t & cb)
{
    record(dst_dev, dst, 0, src_dev, src, 0, size, 1, 1);
    g_pending.push_back(cb);
}

static device_t * g_fake_device = (device_t *) 0x1;
static device_t * hook_device_get(runtime_t *, device_global_id_t) { return g_fake_device; }

static area_chunk_t * hook_allocate(runtime_t *, device_global_id_t, size_t size)
{
    area_chunk_t * c = (area_chunk_t *) calloc(1, sizeof(area_chunk_t));
    c->ptr = (uintptr_t) (g_allocs.size() + 1) << FAKE_SHIFT;
    c->size = size;
    g_allocs.push_back((int64_t) size);
    return c;
}

static void hook_deallocate(runtime_t *, device_global_id_t, area_chunk_t *) {}
static void hook_execute(runtime_t *, device_t *, task_t *) {}

using Trees = std::map<std::pair<size_t, size_t>, BLASMemoryTree *>;
static IntervalSet<uintptr_t> g_pages;                  // runtime_t::registered_pages
static std::map<uintptr_t, size_t> g_registered;        // runtime_t::registered_memory

static void apply_register(Trees & trees, uintptr_t ptr, size_t size)
{
    uintptr_t a; size_t sz;
    pageas((void *) ptr, size, &a, &sz);
    const uintptr_t b = a + sz;
    std::vector<Interval> iv;
    g_pages.find(a, b, iv);
    unsigned i = 0;
    uintptr_t p1 = a;
    while (1)
    {
        const uintptr_t p2 = (i == iv.size()) ? b : iv[i].a;
        if (p1 < p2)
        {
            g_registered[p1] = p2 - p1;
            for (auto & kv : trees) kv.second->registered(p1, p2 - p1);
        }
        if (i == iv.size()) break;
        p1 = iv[i].b;
        ++i;
    }
    g_pages.fill(a, b);
}

static void apply_unregister(Trees & trees, uintptr_t ptr, size_t size)
{
    uintptr_t a; size_t sz;
    pageas((void *) ptr, size, &a, &sz);
    const uintptr_t b = a + sz;
    std::vector<Interval> iv;
    g_pages.find(a, b, iv);
    std::sort(iv.begin(), iv.end());
    for (const Interval & v : iv)
    {
        g_registered.erase(v.a);
        for (auto & kv : trees) kv.second->unregistered(v.a, v.b - v.a);
    }
    g_pages.unfill(a, b);
}

int main(int argc, char ** argv)
{
    if (argc < 3) { fprintf(stderr, "usage: %s <stream.bin> <out-prefix> [events.bin]\n", argv[0]); return 2; }
    std::vector<xk_stream_rec_t> recs;
    if (xk_stream_read(argv[1], recs)) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }
    std::vector<std::array<int64_t, 4>> events;
    if (argc > 3)
    {
        FILE * ef = fopen(argv[3], "rb");
        if (!ef) { fprintf(stderr, "cannot read %s\n", argv[3]); return 2; }
        std::array<int64_t, 4> e;
        while (fread(e.data(), 8, 4, ef) == 4) events.push_back(e);
        fclose(ef);
    }
    size_t next_event = 0;

    xk_seam_hooks.copy2d = hook_copy2d;
    xk_seam_hooks.copy1d = hook_copy1d;
    xk_seam_hooks.device_get = hook_device_get;
    xk_seam_hooks.allocate = hook_allocate;
    xk_seam_hooks.deallocate = hook_deallocate;
    xk_seam_hooks.execute = hook_execute;

    // the trees only touch runtime->router (get_source) and the seam members
    runtime_t * runtime = (runtime_t *) calloc(1, sizeof(runtime_t));
    new (&runtime->router) RouterAffinity();

    Trees trees;
    std::vector<std::array<int64_t, 5>> views;
    const device_global_id_t GPU = 1;

    size_t i = 0;
    while (i < recs.size())
    {
        const uint32_t tid = recs[i].task;
        while (next_event < events.size() && events[next_event][0] <= (int64_t) tid)
        {
            const auto & e = events[next_event++];
            if (e[1] == 1) apply_register(trees, (uintptr_t) e[2], (size_t) e[3]);
            else apply_unregister(trees, (uintptr_t) e[2], (size_t) e[3]);
        }
        size_t j = i;
        while (j < recs.size() && recs[j].task == tid) ++j;
        const task_access_counter_t AC = (task_access_counter_t) (j - i);
        constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT;
        task_t * task = (task_t *) calloc(1, task_compute_size(flags, AC) + 64);
        new (task) task_t(XKRT_TASK_FORMAT_NULL, flags);
        new (TASK_DEP_INFO(task)) task_dep_info_t(AC);
        access_t * accesses = TASK_ACCESSES(task, flags);
        for (size_t a = i; a < j; ++a)
        {
            const xk_stream_rec_t & r = recs[a];
            const access_mode_t mode = (access_mode_t) r.mode;
            if (r.type == XK_STREAM_MATRIX)
                new (accesses + (a - i)) access_t(task, MATRIX_COLMAJOR, (const void *) r.addr, r.ld,
                                                  r.offset_m, r.offset_n, r.m, r.n, r.sizeof_type, mode);
            else
                new (accesses + (a - i)) access_t(task, (uintptr_t) r.addr, (uintptr_t) r.ld, mode);
        }
        for (size_t a = 0; a < AC; ++a)
        {
            access_t * acc = accesses + a;
            const size_t ld = acc->host_view.ld, s = acc->host_view.sizeof_type;
            BLASMemoryTree *& tree = trees[{ld, s}];
            if (!tree)
            {
                tree = new BLASMemoryTree(runtime, ld, s, false);
                for (const auto & [p, n] : g_registered) tree->registered(p, n);
            }
            g_task = tid; g_access = (int64_t) a;
            // record field `reserved` bit 0 selects the host (device 0) as the fetch target
            const device_global_id_t target = (recs[i + a].reserved & 1) ? HOST_DEVICE_GLOBAL_ID : GPU;
            tree->fetch(acc, target);
            while (!g_pending.empty())
            {
                callback_t cb = g_pending.front();
                g_pending.pop_front();
                cb.func(cb.args);
            }
            int64_t al, off;
            decode(GPU, acc->device_view.addr, al, off);
            views.push_back({(int64_t) tid, (int64_t) a, al, off, (int64_t) acc->device_view.ld});
        }
        i = j;
    }

    const std::string pfx(argv[2]);
    FILE * f = fopen((pfx + ".plan").c_str(), "wb");
    for (auto & r : g_plan) fwrite(r.data(), 8, 14, f);
    fclose(f);
    f = fopen((pfx + ".allocs").c_str(), "wb");
    fwrite(g_allocs.data(), 8, g_allocs.size(), f);
    fclose(f);
    f = fopen((pfx + ".views").c_str(), "wb");
    for (auto & v : views) fwrite(v.data(), 8, 5, f);
    fclose(f);
    size_t h2d = 0, d2d = 0, d2h = 0;
    for (auto & r : g_plan) (r[2] == 0 ? h2d : r[2] == 1 ? d2h : d2d)++;
    printf("{\"copies\": %zu, \"h2d\": %zu, \"d2d\": %zu, \"d2h\": %zu, \"allocs\": %zu}\n",
           g_plan.size(), h2d, d2d, d2h, g_allocs.size());
    return 0;
}
