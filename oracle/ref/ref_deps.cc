// Reference-backed dependency oracle (test infrastructure; never part of the product).
//
// Drives the reference's own dependency domains exactly as a spawning thread does:
// for every task, construct its access_t records with the reference constructors
// (include/xkrt/memory/access/access.hpp:479-574) and call
// task_dependency_resolve() from src/task/task.cc:285-299 (LINK all accesses, then PUT all)
// on one implicit domain task (include/xkrt/thread/thread.h:159-196). No task ever commits
// or completes, so every edge the trees find is kept (include/xkrt/task/task.hpp:452-512).
// Handle accesses carry their concurrency (record field `reserved` >> 8); the handle map's
// extra empty writer tasks (include/xkrt/memory/access/handle/dependency-map.hpp:93-137) come
// from the calling thread's task stack (thread_t::allocate_task, src/thread/thread.cc:105-123),
// so the ones a task's resolution created are the stack range it grew by; each is numbered in
// creation order, before the task whose resolution created it.
//
// Input : access stream file (oracle/access_stream.h layout).
// Output: <out>.edges  = sorted unique (pred, succ) task pairs as uint32 pairs,
//         <out>.wc     = per-task predecessor count (uint32): the wait counter minus the commit
//                        token a spawned task still holds (an extra task gave its token back),
//         stdout       = one JSON line of counts.
#include <xkrt/task/task.hpp>
#include <xkrt/memory/access/access.hpp>
#include <xkrt/thread/thread.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../access_stream.h"

XKRT_NAMESPACE_USE;

int main(int argc, char ** argv)
{
    if (argc < 3) { fprintf(stderr, "usage: %s <stream.bin> <out-prefix>\n", argv[0]); return 2; }
    std::vector<xk_stream_rec_t> recs;
    if (xk_stream_read(argv[1], recs)) { fprintf(stderr, "cannot read %s\n", argv[1]); return 2; }

    // implicit domain task
    const size_t dsz = task_compute_size(TASK_FLAG_DOMAIN, 0);
    task_t * dom = (task_t *) calloc(1, dsz + 64);
    new (dom) task_t(XKRT_TASK_FORMAT_NULL, TASK_FLAG_DOMAIN);
    new (TASK_DOM_INFO(dom)) task_dom_info_t();

    thread_t * thread = thread_t::get_tls();
    const size_t extra_size = task_compute_size(TASK_FLAG_DEPENDENT, 1);
    std::vector<task_t *> tasks;
    std::vector<bool> extra;
    std::unordered_map<const task_t *, uint32_t> index;
    size_t nspawned = 0;
    auto t0 = std::chrono::steady_clock::now();

    size_t i = 0;
    while (i < recs.size())
    {
        const uint32_t tid = recs[i].task;
        size_t j = i;
        while (j < recs.size() && recs[j].task == tid) ++j;
        const task_access_counter_t AC = (task_access_counter_t) (j - i);

        constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT;
        const size_t size = task_compute_size(flags, AC);
        task_t * task = (task_t *) calloc(1, size + 64);
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
            else if (r.type == XK_STREAM_HANDLE)
            {
                const int c = r.reserved >> 8;
                const access_concurrency_t conc = c ? (access_concurrency_t) c : ACCESS_CONCURRENCY_SEQUENTIAL;
                new (accesses + (a - i)) access_t(task, (const void *) r.addr, mode, conc);
            }
            else
                new (accesses + (a - i)) access_t(task, (uintptr_t) r.addr, (uintptr_t) r.ld, mode);
        }
        uint8_t * const stack0 = thread->memory_stack_ptr;
        task_dependency_resolve(dom, accesses, AC);
        for (uint8_t * p = stack0; p < thread->memory_stack_ptr; p += extra_size)
        {
            index[(task_t *) p] = (uint32_t) tasks.size();
            tasks.push_back((task_t *) p);
            extra.push_back(true);
        }
        index[task] = (uint32_t) tasks.size();
        if (tid != nspawned++) { fprintf(stderr, "task ids must be dense and ordered\n"); return 2; }
        tasks.push_back(task);
        extra.push_back(false);
        i = j;
    }
    auto t1 = std::chrono::steady_clock::now();

    std::vector<std::pair<uint32_t, uint32_t>> edges;
    size_t raw = 0;
    for (uint32_t t = 0; t < tasks.size(); ++t)
    {
        task_t * task = tasks[t];
        const task_access_counter_t AC = TASK_DEP_INFO(task)->ac;
        access_t * accesses = TASK_ACCESSES(task, task->flags);
        for (task_access_counter_t a = 0; a < AC; ++a)
            for (access_t * s : accesses[a].successors)
            {
                edges.emplace_back(t, index.at(s->task));
                ++raw;
            }
    }
    std::sort(edges.begin(), edges.end());
    edges.erase(std::unique(edges.begin(), edges.end()), edges.end());

    std::string pfx(argv[2]);
    FILE * f = fopen((pfx + ".edges").c_str(), "wb");
    for (auto & e : edges) { uint32_t v[2] = {e.first, e.second}; fwrite(v, 4, 2, f); }
    fclose(f);
    f = fopen((pfx + ".wc").c_str(), "wb");
    uint32_t maxwc = 0;
    for (uint32_t t = 0; t < tasks.size(); ++t)
    {
        task_t * task = tasks[t];
        uint32_t wc = (uint32_t) TASK_DEP_INFO(task)->wc.load() - (extra[t] ? 0u : 1u);
        maxwc = std::max(maxwc, wc);
        fwrite(&wc, 4, 1, f);
    }
    fclose(f);
    printf("{\"ntasks\": %zu, \"extra_tasks\": %zu, \"naccesses\": %zu, \"raw_edges\": %zu, \"unique_edges\": %zu, "
           "\"max_wc\": %u, \"resolve_s\": %.6f}\n",
           tasks.size(), tasks.size() - nspawned, recs.size(), raw, edges.size(), maxwc,
           std::chrono::duration<double>(t1 - t0).count());
    return 0;
}
