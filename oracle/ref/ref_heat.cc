// Reference-backed CPU baseline for the heat-diffusion-2d graph (test infrastructure; never part
// of the product): the reference's own host-only runtime (runtime_t with the host driver, built
// from its sources by oracle/ref/build_ref.sh) running the heat example's task graph --
// tile tasks spawned as examples/heat-diffusion-2d/src/main.cc:508-581 does (R on the
// halo-expanded source tile, W on the interior destination tile, tile_x outer / tile_y inner),
// each executed by a HOST-format body applying update_cpu's formula (main.cc:408-421) to its
// tile. The team size comes from the reference's configuration (DRIVERS / XKRT_DRIVERS
// "host,N").
//
// usage: ref_heat NX NY TS STEPS [init.bin out.bin]   -> JSON line {tasks, seconds, tasks_per_s}
#include <xkrt/internals.h>
#include <xkrt/runtime.h>
#include <xkrt/thread/thread.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>

XKRT_NAMESPACE_USE;

static runtime_t runtime;
static long NX, NY, TS;
static const double C = 0.2;
static task_format_id_t heat_fmt;

struct args_t { double * src; double * dst; int tile_x; int tile_y; };

static void heat_body(runtime_t *, device_t *, task_t * task)
{
    constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT;
    const args_t * a = (const args_t *) TASK_ARGS(task, task_compute_size(flags, 2));
    const long x0 = std::max<long>(a->tile_x * TS, 1), x1 = std::min<long>(a->tile_x * TS + TS, NX - 1);
    const long y0 = std::max<long>(a->tile_y * TS, 1), y1 = std::min<long>(a->tile_y * TS + TS, NY - 1);
    for (long j = y0; j < y1; ++j)
    {
        const double * w = a->src + (j - 1) * NX, * s = a->src + j * NX, * e = a->src + (j + 1) * NX;
        double * d = a->dst + j * NX;
        for (long i = x0; i < x1; ++i)
            d[i] = s[i] + C * (((s[i + 1] - 2 * s[i]) + s[i - 1]) + ((e[i] - 2 * s[i]) + w[i]));
    }
}

static void spawn_tile(double * src, double * dst, int tx, int ty)
{
    thread_t * thread = thread_t::get_tls();
    constexpr task_flag_bitfield_t flags = TASK_FLAG_DEPENDENT;
    constexpr size_t task_size = task_compute_size(flags, 2);
    task_t * task = thread->allocate_task(task_size + sizeof(args_t));
    new (task) task_t(heat_fmt, flags);
    new (TASK_DEP_INFO(task)) task_dep_info_t(2);
    args_t * args = (args_t *) TASK_ARGS(task, task_size);
    *args = args_t{src, dst, tx, ty};
    access_t * acc = TASK_ACCESSES(task, flags);
    const long x = tx * TS, y = ty * TS;
    {
        const long x0 = std::max<long>(x - 1, 0), y0 = std::max<long>(y - 1, 0);
        const long x1 = std::min<long>(x + TS + 1, NX), y1 = std::min<long>(y + TS + 1, NY);
        new (acc + 0) access_t(task, MATRIX_COLMAJOR, src, NX, x0, y0, x1 - x0, y1 - y0, sizeof(double), ACCESS_MODE_R);
    }
    {
        const long x0 = std::max<long>(x, 1), y0 = std::max<long>(y, 1);
        const long x1 = std::min<long>(x + TS, NX - 1), y1 = std::min<long>(y + TS, NY - 1);
        new (acc + 1) access_t(task, MATRIX_COLMAJOR, dst, NX, x0, y0, x1 - x0, y1 - y0, sizeof(double), ACCESS_MODE_W);
    }
    thread->resolve(acc, 2);
    runtime.task_commit(task);
}

int main(int argc, char ** argv)
{
    if (argc < 5) { fprintf(stderr, "usage: %s NX NY TS STEPS [init.bin out.bin]\n", argv[0]); return 2; }
    NX = atol(argv[1]); NY = atol(argv[2]); TS = atol(argv[3]);
    const int steps = atoi(argv[4]);
    if (runtime.init() != 0) { fprintf(stderr, "runtime init failed\n"); return 1; }
    task_format_t format;
    memset(&format, 0, sizeof(format));
    format.f[XKRT_TASK_FORMAT_TARGET_HOST] = (task_format_func_t) heat_body;
    snprintf(format.label, sizeof(format.label), "heat");
    heat_fmt = runtime.task_format_create(&format);

    double * a = (double *) aligned_alloc(4096, ((NX * NY * sizeof(double)) + 4095) & ~4095ul);
    double * b = (double *) aligned_alloc(4096, ((NX * NY * sizeof(double)) + 4095) & ~4095ul);
    if (argc >= 7)
    {
        FILE * f = fopen(argv[5], "rb");
        if (!f || fread(a, sizeof(double), NX * NY, f) != (size_t) (NX * NY)) return 3;
        fclose(f);
    }
    else
    {
        std::mt19937_64 rng(42);
        std::uniform_real_distribution<double> u(0.0, 1.0);
        for (long j = 0; j < NY; ++j)
            for (long i = 0; i < NX; ++i)
                a[j * NX + i] = (i == 0 || j == 0 || i == NX - 1 || j == NY - 1) ? 0.0 : u(rng);
    }
    memcpy(b, a, NX * NY * sizeof(double));
    // The reference creates a domain's coherency controller lazily, from the first fetch of an
    // access of that (ld, sizeof), without a lock (src/task/task.cc:50-150 called from
    // src/sched.cc:232): device threads fetching their first tasks at the same time push onto the
    // same std::vector and one of them can read a freed buffer (SIGSEGV in
    // task_get_memory_controller). Creating it here, on the spawning thread, before any task
    // exists, is what that first fetch does in a run without the race.
    {
        thread_t * thread = thread_t::get_tls();
        access_t proto(thread->current_task, MATRIX_COLMAJOR, a, NX, 0, 0, 1, 1, sizeof(double), ACCESS_MODE_R);
        task_get_memory_controller(&runtime, thread->current_task, &proto);
    }
    const long ntx = (NX + TS - 1) / TS, nty = (NY + TS - 1) / TS;
    auto t0 = std::chrono::steady_clock::now();
    double * src = a, * dst = b;
    for (int s = 0; s < steps; ++s)
    {
        for (int tx = 0; tx < ntx; ++tx)
            for (int ty = 0; ty < nty; ++ty)
                spawn_tile(src, dst, tx, ty);
        std::swap(src, dst);
    }
    runtime.task_wait();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (argc >= 7)
    {
        FILE * f = fopen(argv[6], "wb");
        fwrite(src, sizeof(double), NX * NY, f);
        fclose(f);
    }
    const long tasks = ntx * nty * (long) steps;
    printf("{\"tasks\": %ld, \"seconds\": %.6f, \"tasks_per_s\": %.1f}\n", tasks, secs, tasks / secs);
    fflush(stdout);
    // The result is out; the process ends here instead of in runtime.deinit(): the reference's
    // thread_t destructor frees memory_stack_ptr, not memory_stack_bottom
    // (include/xkrt/thread/thread.h:211-214), a pointer into the middle of its task stack once a
    // task was allocated, and glibc then aborts or crashes depending on the bytes before it.
    std::_Exit(0);
}
