// heat-diffusion-2d through the XKRT C++ source API, written the way the reference's example
// builds its tasks (examples/heat-diffusion-2d/src/main.cc:425-566): a task format whose CUDA
// target launches the program's own tile kernel through task_detachable_kernel_launch, tasks
// built by hand (thread_t::allocate_task, task_t / task_dep_info_t / task_dev_info_t placement,
// args, access_t constructors, thread_t::resolve, runtime_t::task_commit), the grids placed with
// distribute_async before the timed part. FP64 grids, seeded U[0,1) interior, Dirichlet 0
// boundary, c = 0.2; the tile body is heat_cxx_kernel.cu.
//
// One repetition = runtime init, grids, placement (untimed), then the timed part -- spawn every
// tile task of every step, task_wait -- then deinit.
//
// usage: heat_cxx NX NY TS STEPS [REPS [init.bin out.bin]]   (HEAT_CXX_PLACE=0: no placement tasks)
// Output: one JSON line per repetition {rep, tasks, seconds, tasks_per_s, spawn_s, checksum, grid_a, grid_b}.
#include <xkrt/runtime.h>
#include <xkrt/driver/driver-cu.h>

#include <time.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

XKRT_NAMESPACE_USE;

extern "C" void heat_cxx_tile(cudaStream_t stream, const double * src, long ld_src, double * dst, long ld_dst, long nx, long ny,
                              long x, long y, long ts, double c);

static runtime_t runtime;
static long NX, NY, TS;
static const double C = 0.2;
static task_format_id_t heat_format;

struct args_t { double * src; double * dst; int tile_x; int tile_y; };

static double now_s()
{
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

// the kernel launcher: device pointers of the two accesses re-based on the tile's cell (x, y)
static void launcher(runtime_t *, device_t *, task_t * task, queue_cu_t * queue, command_t *, queue_command_list_counter_t idx)
{
    const args_t * args = (const args_t *) TASK_ARGS(task);
    const access_t * acc = TASK_ACCESSES(task);
    const double * src = (const double *) acc[0].device_view.addr;
    double * dst = (double *) acc[1].device_view.addr;
    const long ld_src = (long) acc[0].device_view.ld, ld_dst = (long) acc[1].device_view.ld;
    if (args->tile_x > 0) src += 1; else dst -= 1;
    if (args->tile_y > 0) src += ld_src; else dst -= ld_dst;
    cudaStream_t stream = queue->cu.handle.high;
    heat_cxx_tile(stream, src, ld_src, dst, ld_dst, NX, NY, args->tile_x * TS, args->tile_y * TS, TS, C);
    cudaEventRecord(queue->cu.events.buffer[idx], stream);
}

static void routine(runtime_t * rt, device_t * device, task_t * task)
{
    rt->task_detachable_kernel_launch(device, task, (kernel_launcher_t) launcher);
}

static void update_tile(double * src, double * dst, int tile_x, int tile_y)
{
    thread_t * thread = thread_t::get_tls();
    constexpr task_flag_bitfield_t flags = TASK_FLAG_DEVICE | TASK_FLAG_DEPENDENT | TASK_FLAG_DETACHABLE;
    constexpr size_t task_size = task_compute_size(flags, 2);
    task_t * task = thread->allocate_task(task_size + sizeof(args_t));
    new (task) task_t(heat_format, flags);
    new (TASK_DEP_INFO(task)) task_dep_info_t(2);
    new (TASK_DEV_INFO(task)) task_dev_info_t(UNSPECIFIED_DEVICE_GLOBAL_ID, 0);
    *(args_t *) TASK_ARGS(task, task_size) = args_t{src, dst, tile_x, tile_y};
    access_t * acc = TASK_ACCESSES(task, flags);
    const long x = tile_x * TS, y = tile_y * TS;
    {
        const long x0 = MAX(x - 1, 0), y0 = MAX(y - 1, 0), x1 = MIN(x + TS + 1, NX), y1 = MIN(y + TS + 1, NY);
        new (acc + 0) access_t(task, MATRIX_COLMAJOR, src, NX, x0, y0, x1 - x0, y1 - y0, sizeof(double), ACCESS_MODE_R);
    }
    {
        const long x0 = MAX(x, 1), y0 = MAX(y, 1), x1 = MIN(x + TS, NX - 1), y1 = MIN(y + TS, NY - 1);
        new (acc + 1) access_t(task, MATRIX_COLMAJOR, dst, NX, x0, y0, x1 - x0, y1 - y0, sizeof(double), ACCESS_MODE_W);
    }
    thread->resolve(acc, 2);
    runtime.task_commit(task);
}

// seeded U[0,1) interior, Dirichlet 0 boundary (splitmix64, top 53 bits; as examples/heat_xkrt.c)
static void seeded_grid(double * g, long nx, long ny, uint64_t seed)
{
    uint64_t s = seed;
    for (long j = 0; j < ny; ++j)
        for (long i = 0; i < nx; ++i)
        {
            s += 0x9e3779b97f4a7c15ull;
            uint64_t z = s;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            z ^= z >> 31;
            const double u = (double) (z >> 11) * (1.0 / 9007199254740992.0);
            g[j * nx + i] = (i == 0 || j == 0 || i == nx - 1 || j == ny - 1) ? 0.0 : u;
        }
}

int main(int argc, char ** argv)
{
    if (argc < 5) { fprintf(stderr, "usage: %s NX NY TS STEPS [REPS [init.bin out.bin]]\n", argv[0]); return 2; }
    NX = atol(argv[1]); NY = atol(argv[2]); TS = atol(argv[3]);
    const int steps = atoi(argv[4]);
    const int reps = argc > 5 ? atoi(argv[5]) : 1;
    const char * init_path = argc > 7 ? argv[6] : nullptr, * out_path = argc > 7 ? argv[7] : nullptr;
    if (NX < 3 || NY < 3 || TS < 1 || steps < 1 || reps < 1) { fprintf(stderr, "bad sizes\n"); return 2; }
    const size_t cells = (size_t) NX * (size_t) NY;
    double * init = (double *) malloc(cells * sizeof(double));
    if (!init) return 3;
    if (init_path)
    {
        FILE * f = fopen(init_path, "rb");
        if (!f || fread(init, sizeof(double), cells, f) != cells) { fprintf(stderr, "cannot read %s\n", init_path); return 3; }
        fclose(f);
    }
    else
        seeded_grid(init, NX, NY, 42);
    const int ntx = (int) NUM_OF_TILES(NX, TS), nty = (int) NUM_OF_TILES(NY, TS);
    const char * pe = getenv("HEAT_CXX_PLACE");
    const bool place = !pe || atoi(pe) != 0;       // HEAT_CXX_PLACE=0: no distribute_async before the timed part
    for (int rep = 0; rep < reps; ++rep)
    {
        if (runtime.init() != 0) { fprintf(stderr, "init: %s\n", xkb_last_error()); return 1; }
        task_format_t format;
        memset(&format, 0, sizeof(format));
        format.f[XKRT_TASK_FORMAT_TARGET_CUDA] = (task_format_func_t) routine;
        snprintf(format.label, sizeof(format.label), "heat-cxx");
        heat_format = runtime.task_format_create(&format);
        double * a = (double *) runtime.memory_host_allocate(0, cells * sizeof(double));
        double * b = (double *) runtime.memory_host_allocate(0, cells * sizeof(double));
        if (!a || !b) { fprintf(stderr, "host allocation: %s\n", xkb_last_error()); return 1; }
        memcpy(a, init, cells * sizeof(double));
        memcpy(b, init, cells * sizeof(double));
        if (place)
        {
            runtime.distribute_async(XKRT_DISTRIBUTION_TYPE_CYCLIC2D, MATRIX_COLMAJOR, a, NX, NX, NY, TS, TS, sizeof(double), 1, 1);
            runtime.distribute_async(XKRT_DISTRIBUTION_TYPE_CYCLIC2D, MATRIX_COLMAJOR, b, NX, NX, NY, TS, TS, sizeof(double), 1, 1);
            runtime.task_wait();
        }

        const double t0 = now_s();
        double * src = a, * dst = b;
        for (int s = 0; s < steps; ++s)
        {
            for (int tx = 0; tx < ntx; ++tx)
                for (int ty = 0; ty < nty; ++ty)
                    update_tile(src, dst, tx, ty);
            double * t = src; src = dst; dst = t;
        }
        const double t1 = now_s();
        runtime.task_wait();
        const double t2 = now_s();
        const int st = xkb_runtime_status(runtime.capi);
        if (st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
        double checksum = 0;
        for (size_t k = 0; k < cells; ++k) checksum += src[k];
        if (out_path && rep == reps - 1)
        {
            FILE * f = fopen(out_path, "wb");
            if (!f || fwrite(src, sizeof(double), cells, f) != cells) return 3;
            fclose(f);
        }
        const long tasks = (long) ntx * nty * steps;
        if (runtime.deinit() != 0) { fprintf(stderr, "deinit: %s\n", xkb_last_error()); return 1; }
        printf("{\"rep\": %d, \"tasks\": %ld, \"seconds\": %.6f, \"tasks_per_s\": %.1f, \"spawn_s\": %.6f, \"checksum\": %.17g, "
               "\"grid_a\": %llu, \"grid_b\": %llu}\n", rep, tasks, t2 - t0, (double) tasks / (t2 - t0), t1 - t0, checksum,
               (unsigned long long) (uintptr_t) a, (unsigned long long) (uintptr_t) b);
        fflush(stdout);
    }
    free(init);
    return 0;
}
