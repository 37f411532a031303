/* heat-diffusion-2d through the XKRT C API on libxkb200, timed the way the reference's host
 * runtime is timed on the same graph: from the first spawn to the return of xkrt_task_wait.
 *
 * The task graph is the heat example's (examples/heat-diffusion-2d/src/main.cc:508-581): per
 * step, one tile task per tile (tile_x outer, tile_y inner) with R on the halo-expanded source
 * tile and W on the destination tile clipped to the interior; the grids alternate between
 * steps. The device body is the library's built-in tile body (xkb_task_format_builtin).
 *
 * One repetition = xkrt_init, two host grids from xkrt_memory_host_allocate filled with the
 * seeded initial grid (untimed), then the timed part -- spawn every task, xkrt_task_wait, which
 * resolves the dependencies on the GPU, copies both grids to the device, runs the graph on the
 * persistent scheduler and copies the written blocks back -- then xkrt_deinit (untimed). Each
 * repetition thus moves both grids host -> device and the written interior back.
 *
 * usage: heat_xkrt NX NY TS STEPS [REPS [F32 [init.bin out.bin]]]
 *   F32 = 1: FP32 storage (the FP32 tile body); init.bin / out.bin hold FP64 grids (NX*NY,
 *   row-major) -- the FP32 grid starts from the FP64 values rounded to float.
 * Output: one JSON line per repetition {rep, tasks, seconds, tasks_per_s, spawn_s, resolve_ms,
 * coherency_ms, run_ms, writeback_ms, edges, h2d, d2h (copies), h2d_bytes, d2h_bytes, fused, checksum, grid_a,
 * grid_b}. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "xkrt_capi.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

/* seeded U[0,1) interior, Dirichlet 0 boundary: splitmix64, top 53 bits */
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

static xkrt_access_t tile(xkrt_access_mode_t mode, void * grid, long ld, unsigned long esz, long x0, long y0, long x1, long y1)
{
    xkrt_access_t a;
    memset(&a, 0, sizeof(a));
    a.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; a.mode = mode; a.scope = ACCESS_SCOPE_NONUNIFIED;
    a.type = ACCESS_TYPE_BLAS_MATRIX;
    a.region.matrix.storage = MATRIX_COLMAJOR; a.region.matrix.addr = grid; a.region.matrix.ld = (unsigned long) ld;
    a.region.matrix.offset_m = (unsigned long) x0; a.region.matrix.offset_n = (unsigned long) y0;
    a.region.matrix.m = (unsigned long) (x1 - x0); a.region.matrix.n = (unsigned long) (y1 - y0);
    a.region.matrix.sizeof_type = esz;
    return a;
}

int main(int argc, char ** argv)
{
    if (argc < 5)
    {
        fprintf(stderr, "usage: %s NX NY TS STEPS [REPS [F32 [init.bin out.bin]]]\n", argv[0]);
        return 2;
    }
    const long NX = atol(argv[1]), NY = atol(argv[2]), TS = atol(argv[3]);
    const int steps = atoi(argv[4]);
    const int reps = argc > 5 ? atoi(argv[5]) : 1;
    const int f32 = argc > 6 ? atoi(argv[6]) : 0;
    const char * init_path = argc > 8 ? argv[7] : NULL, * out_path = argc > 8 ? argv[8] : NULL;
    if (NX < 3 || NY < 3 || TS < 1 || steps < 1 || reps < 1) { fprintf(stderr, "bad sizes\n"); return 2; }
    const size_t cells = (size_t) NX * (size_t) NY;
    const unsigned long esz = f32 ? sizeof(float) : sizeof(double);

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

    const long ntx = (NX + TS - 1) / TS, nty = (NY + TS - 1) / TS;
    for (int rep = 0; rep < reps; ++rep)
    {
        xkrt_runtime_t * rt;
        if (xkrt_init(&rt) != 0) { fprintf(stderr, "xkrt_init: %s\n", xkb_last_error()); return 1; }
        void * a = xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, cells * esz);
        void * b = xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, cells * esz);
        if (!a || !b) { fprintf(stderr, "host allocation: %s\n", xkb_last_error()); return 1; }
        if (f32) for (size_t k = 0; k < cells; ++k) ((float *) a)[k] = (float) init[k];
        else memcpy(a, init, cells * sizeof(double));
        memcpy(b, a, cells * esz);
        const xkrt_task_format_id_t fmt = xkb_task_format_builtin(rt, f32 ? XKB_TASK_HEAT_F32 : XKB_TASK_HEAT_F64);

        const double t0 = now_s();
        void * src = a, * dst = b;
        xkb_task_desc_t d;
        memset(&d, 0, sizeof(d));
        d.kind = f32 ? XKB_TASK_HEAT_F32 : XKB_TASK_HEAT_F64;
        d.u.heat.ld = NX; d.u.heat.nx = (int32_t) NX; d.u.heat.ny = (int32_t) NY; d.u.heat.c = 0.2;
        for (int s = 0; s < steps; ++s)
        {
            d.u.heat.src = (uint64_t) (uintptr_t) src; d.u.heat.dst = (uint64_t) (uintptr_t) dst;
            for (long tx = 0; tx < ntx; ++tx)
                for (long ty = 0; ty < nty; ++ty)
                {
                    const long x = tx * TS, y = ty * TS;
                    xkrt_access_t acc[2];
                    acc[0] = tile(ACCESS_MODE_R, src, NX, esz, x > 0 ? x - 1 : 0, y > 0 ? y - 1 : 0,
                                  x + TS + 1 < NX ? x + TS + 1 : NX, y + TS + 1 < NY ? y + TS + 1 : NY);
                    acc[1] = tile(ACCESS_MODE_W, dst, NX, esz, x > 1 ? x : 1, y > 1 ? y : 1,
                                  x + TS < NX - 1 ? x + TS : NX - 1, y + TS < NY - 1 ? y + TS : NY - 1);
                    d.u.heat.x0 = (int32_t) x; d.u.heat.x1 = (int32_t) (x + TS < NX ? x + TS : NX);
                    d.u.heat.y0 = (int32_t) y; d.u.heat.y1 = (int32_t) (y + TS < NY ? y + TS : NY);
                    xkrt_task_spawn_with_format_with_accesses(rt, 1, fmt, &d, sizeof(d), acc, 2);
                }
            void * t = src; src = dst; dst = t;
        }
        const double t1 = now_s();
        xkrt_task_wait(rt);
        const double t2 = now_s();

        uint64_t tasks = 0, edges = 0, h2d = 0, d2h = 0, h2d_bytes = 0, d2h_bytes = 0;
        int fused = 0;
        double ms[4] = {0, 0, 0, 0};
        xkb_runtime_last_wait(rt, &tasks, &edges, &h2d, &d2h, &fused);
        xkb_runtime_last_wait_times(rt, &ms[0], &ms[1], &ms[2], &ms[3]);
        xkb_runtime_last_wait_bytes(rt, &h2d_bytes, &d2h_bytes);
        double checksum = 0;
        for (size_t k = 0; k < cells; ++k) checksum += f32 ? (double) ((const float *) src)[k] : ((const double *) src)[k];
        if (out_path && rep == reps - 1)
        {
            FILE * f = fopen(out_path, "wb");
            if (!f) return 3;
            for (size_t k = 0; k < cells; ++k)
            {
                const double v = f32 ? (double) ((const float *) src)[k] : ((const double *) src)[k];
                fwrite(&v, sizeof(v), 1, f);
            }
            fclose(f);
        }
        const int st = xkb_runtime_status(rt);
        if (st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
        if (xkrt_deinit(rt) != 0) { fprintf(stderr, "xkrt_deinit: %s\n", xkb_last_error()); return 1; }
        printf("{\"rep\": %d, \"tasks\": %llu, \"seconds\": %.6f, \"tasks_per_s\": %.1f, \"spawn_s\": %.6f, "
               "\"resolve_ms\": %.3f, \"coherency_ms\": %.3f, \"run_ms\": %.3f, \"writeback_ms\": %.3f, \"edges\": %llu, "
               "\"h2d\": %llu, \"d2h\": %llu, \"h2d_bytes\": %llu, \"d2h_bytes\": %llu, \"fused\": %d, \"checksum\": %.17g, "
               "\"grid_a\": %llu, \"grid_b\": %llu}\n",
               rep, (unsigned long long) tasks, t2 - t0, (double) tasks / (t2 - t0), t1 - t0, ms[0], ms[1], ms[2], ms[3],
               (unsigned long long) edges, (unsigned long long) h2d, (unsigned long long) d2h, (unsigned long long) h2d_bytes,
               (unsigned long long) d2h_bytes, fused, checksum, (unsigned long long) (uintptr_t) a, (unsigned long long) (uintptr_t) b);
        fflush(stdout);
    }
    free(init);
    return 0;
}
