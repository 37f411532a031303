// Reference-backed CPU baseline for the axpby task chains (test infrastructure; never part of
// the product): the reference's own host-only runtime (runtime_t with the host driver, built
// from its sources by oracle/ref/build_ref.sh) running y = a*x + b*y over N FP64 elements in
// PASSES passes of seeded chunks, each task with a segment access R on its x chunk and RW on
// its y chunk (the access pattern of examples/task-axpby.cc:108-118), executed by a HOST-format
// body. The chunk plan and the inputs come from the same seeded generator as the library's
// example program (xkaapi_b200/examples/axpby_xkrt.c), so both run the same graph.
//
// usage: ref_axpby N PASSES SEED CMIN CMAX [out.bin]  -> JSON line {tasks, seconds, tasks_per_s, checksum}
#include <xkrt/internals.h>
#include <xkrt/runtime.h>
#include <xkrt/thread/thread.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

XKRT_NAMESPACE_USE;

static runtime_t runtime;
static task_format_id_t axpby_fmt;

struct args_t { const double * x; double * y; int64_t lo, hi; double a, b; };

static void axpby_body(runtime_t *, device_t *, task_t * task)
{
    constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT;
    const args_t * g = (const args_t *) TASK_ARGS(task, task_compute_size(flags, 2));
    for (int64_t i = g->lo; i < g->hi; ++i) g->y[i] = g->a * g->x[i] + g->b * g->y[i];
}

static uint64_t splitmix(uint64_t * s)
{
    uint64_t z = (*s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
static double unit(uint64_t * s) { return (double) (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

static void spawn_chunk(const double * x, double * y, int64_t lo, int64_t hi, double a, double b)
{
    thread_t * thread = thread_t::get_tls();
    constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT;
    constexpr size_t task_size = task_compute_size(flags, 2);
    task_t * task = thread->allocate_task(task_size + sizeof(args_t));
    new (task) task_t(axpby_fmt, flags);
    new (TASK_DEP_INFO(task)) task_dep_info_t(2);
    args_t * args = (args_t *) TASK_ARGS(task, task_size);
    *args = args_t{x, y, lo, hi, a, b};
    access_t * acc = TASK_ACCESSES(task, flags);
    new (acc + 0) access_t(task, (uintptr_t) (x + lo), (uintptr_t) (x + hi), ACCESS_MODE_R);
    new (acc + 1) access_t(task, (uintptr_t) (y + lo), (uintptr_t) (y + hi), ACCESS_MODE_RW);
    thread->resolve(acc, 2);
    runtime.task_commit(task);
}

int main(int argc, char ** argv)
{
    if (argc < 6) { fprintf(stderr, "usage: %s N PASSES SEED CMIN CMAX [out.bin]\n", argv[0]); return 2; }
    const int64_t n = atoll(argv[1]);
    const int passes = atoi(argv[2]);
    const uint64_t seed = strtoull(argv[3], nullptr, 10);
    const double cmin = atof(argv[4]), cmax = atof(argv[5]);
    if (runtime.init() != 0) { fprintf(stderr, "runtime init failed\n"); return 1; }
    task_format_t format;
    memset(&format, 0, sizeof(format));
    format.f[XKRT_TASK_FORMAT_TARGET_HOST] = (task_format_func_t) axpby_body;
    snprintf(format.label, sizeof(format.label), "axpby");
    axpby_fmt = runtime.task_format_create(&format);

    std::vector<double> x(n), y(n);
    // the segment coherency controller, created here on the spawning thread instead of lazily by
    // the first concurrent fetches (an unlocked check-then-create, src/task/task.cc:69-95)
    {
        thread_t * thread = thread_t::get_tls();
        access_t proto(thread->current_task, (uintptr_t) x.data(), (uintptr_t) (x.data() + 1), ACCESS_MODE_R);
        task_get_memory_controller(&runtime, thread->current_task, &proto);
    }
    uint64_t s = seed;
    for (int64_t i = 0; i < n; ++i) x[i] = 2.0 * unit(&s) - 1.0;
    for (int64_t i = 0; i < n; ++i) y[i] = 2.0 * unit(&s) - 1.0;
    struct Chunk { int64_t lo, hi; double a, b; };
    std::vector<Chunk> plan;
    const double lmin = std::log(cmin), lmax = std::log(cmax);
    for (int p = 0; p < passes; ++p)
    {
        const double a = 4.0 * unit(&s) - 2.0, b = 4.0 * unit(&s) - 2.0;
        int64_t at = 0;
        bool first = true;
        while (at < n)
        {
            int64_t len = (int64_t) (std::exp(lmin + (lmax - lmin) * unit(&s)) / 8.0);
            if (len < 1) len = 1;
            if (first) { len = 1 + (int64_t) (unit(&s) * (double) len); first = false; }
            const int64_t hi = at + len < n ? at + len : n;
            plan.push_back({at, hi, a, b});
            at = hi;
        }
    }
    auto t0 = std::chrono::steady_clock::now();
    for (const Chunk & c : plan) spawn_chunk(x.data(), y.data(), c.lo, c.hi, c.a, c.b);
    runtime.task_wait();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    double checksum = 0;
    for (int64_t i = 0; i < n; ++i) checksum += y[i];
    if (argc >= 7)
    {
        FILE * f = fopen(argv[6], "wb");
        fwrite(y.data(), sizeof(double), (size_t) n, f);
        fclose(f);
    }
    printf("{\"tasks\": %zu, \"seconds\": %.6f, \"tasks_per_s\": %.1f, \"checksum\": %.17g}\n", plan.size(), secs,
           plan.size() / secs, checksum);
    fflush(stdout);
    // The result is out; the process ends here instead of in runtime.deinit(): the reference's
    // thread_t destructor frees memory_stack_ptr, not memory_stack_bottom
    // (include/xkrt/thread/thread.h:211-214), a pointer into the middle of its task stack once a
    // task was allocated, and glibc then aborts or crashes depending on the bytes before it.
    std::_Exit(0);
}
