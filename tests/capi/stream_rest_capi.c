/* A batch whose first windows run on the GPU while the program spawns and whose rest cannot:
 * short axpby chunks, then chunks long enough to be split into slices (streaming stops there),
 * then short chunks again, over x and y from xkrt_memory_host_allocate. The rest of the batch
 * runs at xkrt_task_wait behind the streamed windows, on the graph window from its first task.
 * y is checked against the same passes computed on the host, bit for bit (a*x + b*y, two
 * roundings and a sum, as the device body does).
 * usage: stream_rest_capi. Output: one JSON line; exit status 0 = success. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "xkrt_capi.h"

enum { N = 1 << 20 };

static xkrt_access_t segment(xkrt_access_mode_t mode, const double * base, long lo, long hi)
{
    xkrt_access_t a;
    memset(&a, 0, sizeof(a));
    a.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; a.mode = mode; a.type = ACCESS_TYPE_SEGMENT;
    a.region.segment.a = (void *) (base + lo); a.region.segment.b = (void *) (base + hi);
    return a;
}

int main(void)
{
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) { fprintf(stderr, "init: %s\n", xkb_last_error()); return 1; }
    double * x = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, N * sizeof(double));
    double * y = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, N * sizeof(double));
    double * yr = (double *) malloc(N * sizeof(double));
    if (!x || !y || !yr) return 1;
    for (long i = 0; i < N; ++i) { x[i] = (double) (i % 1000) * 0.001 - 0.25; y[i] = 1.0 + (double) (i % 7) * 0.125; yr[i] = y[i]; }
    const xkrt_task_format_id_t fmt = xkb_task_format_builtin(rt, XKB_TASK_AXPBY);
    /* passes: chunk length (elements) and coefficients */
    const long len[3] = {2048, 65536, 4096};
    const double ca[3] = {0.5, -1.25, 0.75}, cb[3] = {1.5, 0.5, -0.25};
    long tasks = 0;
    for (int p = 0; p < 3; ++p)
    {
        xkb_task_desc_t d;
        memset(&d, 0, sizeof(d));
        d.kind = XKB_TASK_AXPBY;
        d.u.axpby.x = (uint64_t) (uintptr_t) x; d.u.axpby.y = (uint64_t) (uintptr_t) y;
        d.u.axpby.a = ca[p]; d.u.axpby.b = cb[p];
        for (long lo = 0; lo < N; lo += len[p], ++tasks)
        {
            const long hi = lo + len[p] < N ? lo + len[p] : N;
            d.u.axpby.lo = lo; d.u.axpby.hi = hi;
            xkrt_access_t acc[2] = {segment(ACCESS_MODE_R, x, lo, hi), segment(ACCESS_MODE_RW, y, lo, hi)};
            xkrt_task_spawn_with_format_with_accesses(rt, 1, fmt, &d, sizeof(d), acc, 2);
        }
        for (long i = 0; i < N; ++i)
        {
            const double u = ca[p] * x[i], v = cb[p] * yr[i];
            yr[i] = u + v;
        }
    }
    xkrt_task_wait(rt);
    uint64_t ran = 0, edges = 0;
    int fused = 0;
    xkb_runtime_last_wait(rt, &ran, &edges, NULL, NULL, &fused);
    const int st = xkb_runtime_status(rt);
    if (st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
    long bad = 0;
    for (long i = 0; i < N; ++i) bad += memcmp(&y[i], &yr[i], sizeof(double)) != 0;
    if (xkrt_deinit(rt) != 0) return 1;
    printf("{\"tasks\": %ld, \"ran\": %llu, \"edges\": %llu, \"fused\": %d, \"mismatches\": %ld}\n", tasks, (unsigned long long) ran,
           (unsigned long long) edges, fused, bad);
    free(yr);
    return bad != 0 || (long) ran != tasks;
}
