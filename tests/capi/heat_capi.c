/* The heat-diffusion-2d example (examples/heat-diffusion-2d/src/main.cc:508-663) through the
 * XKRT C API on libxkb200: two host grids from xkrt_memory_host_allocate, one tile task per
 * tile and step with R on the halo-expanded source tile and W on the destination interior,
 * the built-in FP64 tile body as the device format, xkrt_task_wait. With EXPORT_EVERY > 0 a host
 * task reads the whole current grid every EXPORT_EVERY steps and records its sum (the example's
 * VTK export task, main.cc:115-163) -- the batch then mixes host and device tasks.
 * usage: heat_capi NX NY TS STEPS EXPORT_EVERY init.bin out.bin sums.txt */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "xkrt_capi.h"

static long NX, NY, TS;
static FILE * sums;

static void export_sum(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev;
    const double * g = (const double *) xkrt_task_access_replica(task, 0);
    double s = 0;
    for (long k = 0; k < NX * NY; ++k) s += g[k];
    fprintf(sums, "%d %.17g\n", *(const int *) xkrt_task_args(task), s);
}

static xkrt_access_t tile(xkrt_access_mode_t mode, double * grid, long x0, long y0, long x1, long y1)
{
    xkrt_access_t a = {ACCESS_CONCURRENCY_SEQUENTIAL, mode, ACCESS_SCOPE_NONUNIFIED, ACCESS_TYPE_BLAS_MATRIX, {{0}}};
    a.region.matrix.storage = MATRIX_COLMAJOR; a.region.matrix.addr = grid; a.region.matrix.ld = NX;
    a.region.matrix.offset_m = x0; a.region.matrix.offset_n = y0;
    a.region.matrix.m = x1 - x0; a.region.matrix.n = y1 - y0; a.region.matrix.sizeof_type = sizeof(double);
    return a;
}

int main(int argc, char ** argv)
{
    if (argc < 9) return 2;
    NX = atol(argv[1]); NY = atol(argv[2]); TS = atol(argv[3]);
    const int steps = atoi(argv[4]), every = atoi(argv[5]);
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) { fprintf(stderr, "init: %s\n", xkb_last_error()); return 1; }
    double * a = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, NX * NY * sizeof(double));
    double * b = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, NX * NY * sizeof(double));
    FILE * f = fopen(argv[6], "rb");
    if (!f || fread(a, sizeof(double), NX * NY, f) != (size_t) (NX * NY)) return 3;
    fclose(f);
    memcpy(b, a, NX * NY * sizeof(double));
    sums = fopen(argv[8], "w");

    const xkrt_task_format_id_t heat = xkb_task_format_builtin(rt, XKB_TASK_HEAT_F64);
    const xkrt_task_format_id_t exp = xkrt_task_format_put(rt, "export");
    xkrt_task_format_set(rt, exp, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) export_sum);
    const long ntx = (NX + TS - 1) / TS, nty = (NY + TS - 1) / TS;
    double * src = a, * dst = b;
    for (int s = 0; s < steps; ++s)
    {
        for (long tx = 0; tx < ntx; ++tx)
            for (long ty = 0; ty < nty; ++ty)
            {
                const long x = tx * TS, y = ty * TS;
                xkrt_access_t acc[2];
                acc[0] = tile(ACCESS_MODE_R, src, x > 0 ? x - 1 : 0, y > 0 ? y - 1 : 0,
                              x + TS + 1 < NX ? x + TS + 1 : NX, y + TS + 1 < NY ? y + TS + 1 : NY);
                acc[1] = tile(ACCESS_MODE_W, dst, x > 1 ? x : 1, y > 1 ? y : 1,
                              x + TS < NX - 1 ? x + TS : NX - 1, y + TS < NY - 1 ? y + TS : NY - 1);
                xkb_task_desc_t d;
                memset(&d, 0, sizeof(d));
                d.kind = XKB_TASK_HEAT_F64;
                d.u.heat.src = (uint64_t) src; d.u.heat.dst = (uint64_t) dst; d.u.heat.ld = NX;
                d.u.heat.nx = (int32_t) NX; d.u.heat.ny = (int32_t) NY;
                d.u.heat.x0 = (int32_t) x; d.u.heat.x1 = (int32_t) (x + TS < NX ? x + TS : NX);
                d.u.heat.y0 = (int32_t) y; d.u.heat.y1 = (int32_t) (y + TS < NY ? y + TS : NY);
                d.u.heat.c = 0.2;
                xkrt_task_spawn_with_format_with_accesses(rt, 1, heat, &d, sizeof(d), acc, 2);
            }
        double * t = src; src = dst; dst = t;
        if (every > 0 && (s + 1) % every == 0)
        {
            xkrt_access_t all = tile(ACCESS_MODE_R, src, 0, 0, NX, NY);
            const int step = s + 1;
            xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, exp, &step, sizeof(step), &all, 1);
        }
    }
    xkrt_task_wait(rt);
    uint64_t tasks, edges, h2d, d2h; int fused;
    xkb_runtime_last_wait(rt, &tasks, &edges, &h2d, &d2h, &fused);
    f = fopen(argv[7], "wb");
    fwrite(src, sizeof(double), NX * NY, f);
    fclose(f);
    fclose(sums);
    const int st = xkb_runtime_status(rt);
    if (xkrt_deinit(rt) != 0 || st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
    printf("{\"tasks\": %llu, \"edges\": %llu, \"h2d\": %llu, \"d2h\": %llu, \"fused\": %d}\n", (unsigned long long) tasks,
           (unsigned long long) edges, (unsigned long long) h2d, (unsigned long long) d2h, fused);
    return 0;
}
