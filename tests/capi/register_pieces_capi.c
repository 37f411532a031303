/* Registered memory that is partly page-locked: a second registration made while tasks are
 * pending, touching the first one (they share a page), is not page-locked, except that shared
 * page, which the first registration's lock covers. Device tasks (the library's axpby body) read
 * a vector that starts in that shared page, so its first-touch copy runs across the end of the
 * locked piece; the runtime cuts such copies at the piece's ends. Then an axpby whose element
 * range leaves its vector's region is refused (XKB_EINVAL), not run.
 * Output: one JSON line {"ok": 1, "refused": 1}. Exit status 0 = success. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "xkrt_capi.h"

static xkrt_access_t segment(xkrt_access_mode_t mode, void * a, void * b)
{
    xkrt_access_t x;
    memset(&x, 0, sizeof(x));
    x.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; x.mode = mode; x.scope = ACCESS_SCOPE_NONUNIFIED;
    x.type = ACCESS_TYPE_SEGMENT; x.region.segment.a = a; x.region.segment.b = b;
    return x;
}

static void spawn_axpby(xkrt_runtime_t * rt, xkrt_task_format_id_t ax, double * x, double * y, long lo, long hi, double a, double b)
{
    xkb_task_desc_t d;
    memset(&d, 0, sizeof(d));
    d.kind = XKB_TASK_AXPBY;
    d.u.axpby.x = (uint64_t) (uintptr_t) x; d.u.axpby.y = (uint64_t) (uintptr_t) y;
    d.u.axpby.lo = lo; d.u.axpby.hi = hi; d.u.axpby.a = a; d.u.axpby.b = b;
    xkrt_access_t acc[2] = {segment(ACCESS_MODE_R, x + lo, x + hi), segment(ACCESS_MODE_RW, y + lo, y + hi)};
    xkrt_task_spawn_with_format_with_accesses(rt, 1, ax, &d, sizeof(d), acc, 2);
}

int main(void)
{
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) return 1;
    enum { N1 = 100003, N2 = 200001 };
    unsigned char * buf = (unsigned char *) malloc((N1 + N2) * sizeof(double) + 4096 + 64);
    double * x1 = (double *) (buf + 104);                /* not page-aligned */
    double * x2 = x1 + N1;                               /* shares a page with x1's last one */
    double * y1 = (double *) malloc(N1 * sizeof(double)), * y2 = (double *) malloc(N2 * sizeof(double));
    for (long i = 0; i < N1; ++i) { x1[i] = (double) i; y1[i] = 1.0; }
    for (long i = 0; i < N2; ++i) { x2[i] = (double) (i % 97); y2[i] = 2.0; }
    const xkrt_task_format_id_t ax = xkb_task_format_builtin(rt, XKB_TASK_AXPBY);
    if (xkrt_memory_register(rt, x1, N1 * sizeof(double)) || xkrt_memory_register(rt, y1, N1 * sizeof(double)) ||
        xkrt_memory_register(rt, y2, N2 * sizeof(double)))
        return 1;
    spawn_axpby(rt, ax, x1, y1, 0, N1, 2.0, 3.0);          /* a task pending ... */
    if (xkrt_memory_register(rt, x2, N2 * sizeof(double))) return 1;   /* ... while x2 is registered */
    for (long lo = 0; lo < N2; lo += 65536)
        spawn_axpby(rt, ax, x2, y2, lo, lo + 65536 < N2 ? lo + 65536 : N2, 0.5, -1.0);
    xkrt_task_wait(rt);
    int st = xkb_runtime_status(rt);
    if (st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
    for (long i = 0; i < N1; ++i)
        if (y1[i] != 2.0 * (double) i + 3.0) { fprintf(stderr, "y1[%ld] = %g\n", i, y1[i]); return 1; }
    for (long i = 0; i < N2; ++i)
        if (y2[i] != 0.5 * (double) (i % 97) - 2.0) { fprintf(stderr, "y2[%ld] = %g\n", i, y2[i]); return 1; }
    /* x1's region does not hold elements [N1 - 10, N1 + 10) of x1: refused, nothing runs */
    spawn_axpby(rt, ax, x1, y2, N1 - 10, N1 + 10, 1.0, 1.0);
    xkrt_task_wait(rt);
    const int refused = xkb_runtime_status(rt) == XKB_EINVAL;
    xkrt_deinit(rt);
    printf("{\"ok\": 1, \"refused\": %d}\n", refused);
    return 0;
}
