/* The heat example through the XKRT C API with an xkrt_task_wait every WAIT_EVERY steps in the
 * same runtime: each batch depends on the previous one only through the grids (resolved anew,
 * the runtime's resolver reused, host memory coherent between batches), and the program
 * re-initialises no data between waits. WAIT_EVERY < 0: a wait after steps 1, 2, 4, 8, ... (and
 * the last), so every batch is larger than the one before.
 * With a ninth argument "reset": after every wait but the last the program halves the source
 * grid in host memory, outside any task, and calls xkrt_reset, which makes the runtime forget its
 * device copies; the next batch then reads the halved grid (not the device's copy of the old one).
 * usage: heat_waits_capi NX NY TS STEPS WAIT_EVERY init.bin out.bin [reset] */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "xkrt_capi.h"

static xkrt_access_t tile(xkrt_access_mode_t mode, double * g, long ld, long x0, long y0, long x1, long y1)
{
    xkrt_access_t a;
    memset(&a, 0, sizeof(a));
    a.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; a.mode = mode; a.type = ACCESS_TYPE_BLAS_MATRIX;
    a.region.matrix.storage = MATRIX_COLMAJOR; a.region.matrix.addr = g; a.region.matrix.ld = (unsigned long) ld;
    a.region.matrix.offset_m = (unsigned long) x0; a.region.matrix.offset_n = (unsigned long) y0;
    a.region.matrix.m = (unsigned long) (x1 - x0); a.region.matrix.n = (unsigned long) (y1 - y0);
    a.region.matrix.sizeof_type = sizeof(double);
    return a;
}

int main(int argc, char ** argv)
{
    if (argc < 8) return 2;
    const long NX = atol(argv[1]), NY = atol(argv[2]), TS = atol(argv[3]);
    const int steps = atoi(argv[4]), every = atoi(argv[5]);
    const int reset = argc > 8 && strcmp(argv[8], "reset") == 0;
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) return 1;
    double * a = (double *) malloc(NX * NY * sizeof(double)), * b = (double *) malloc(NX * NY * sizeof(double));
    FILE * f = fopen(argv[6], "rb");
    if (!a || !b || !f || fread(a, sizeof(double), NX * NY, f) != (size_t) (NX * NY)) return 3;
    fclose(f);
    memcpy(b, a, NX * NY * sizeof(double));
    /* user memory registered (not allocated by the runtime) */
    if (xkrt_memory_register(rt, a, NX * NY * sizeof(double)) || xkrt_memory_register(rt, b, NX * NY * sizeof(double))) return 1;
    const xkrt_task_format_id_t heat = xkb_task_format_builtin(rt, XKB_TASK_HEAT_F64);
    double * src = a, * dst = b;
    int waits = 0;
    for (int s = 0; s < steps; ++s)
    {
        for (long x = 0; x < NX; x += TS)
            for (long y = 0; y < NY; y += TS)
            {
                xkrt_access_t acc[2] = {
                    tile(ACCESS_MODE_R, src, NX, x > 0 ? x - 1 : 0, y > 0 ? y - 1 : 0, x + TS + 1 < NX ? x + TS + 1 : NX,
                         y + TS + 1 < NY ? y + TS + 1 : NY),
                    tile(ACCESS_MODE_W, dst, NX, x > 1 ? x : 1, y > 1 ? y : 1, x + TS < NX - 1 ? x + TS : NX - 1,
                         y + TS < NY - 1 ? y + TS : NY - 1)};
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
        const int at = every > 0 ? (s + 1) % every == 0 : ((s + 1) & s) == 0;
        if (at || s + 1 == steps)
        {
            xkrt_task_wait(rt);
            ++waits;
            if (reset && s + 1 < steps)
            {
                for (long i = 0; i < NX * NY; ++i) src[i] *= 0.5;
                xkrt_reset(rt);
            }
        }
    }
    f = fopen(argv[7], "wb");
    fwrite(src, sizeof(double), NX * NY, f);
    fclose(f);
    const int st = xkb_runtime_status(rt);
    if (xkrt_deinit(rt) != 0 || st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
    printf("{\"waits\": %d, \"grid_a\": %llu, \"grid_b\": %llu}\n", waits, (unsigned long long) (uintptr_t) a,
           (unsigned long long) (uintptr_t) b);
    return 0;
}
