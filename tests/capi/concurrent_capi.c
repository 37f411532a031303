/* Concurrent-mode handle accesses through the C API, the shapes of the reference handle map's
 * diagrams (include/xkrt/memory/access/handle/dependency-map.hpp:200-223, :247-262):
 *   T0 W                      x = 1
 *   T1..T4 concurrent W       x += 10 each (atomically; they may overlap)
 *   T5..T7 R                  read x: 41 (an extra writer task runs between the CNC-Ws and T5)
 *   T8, T9 concurrent W       x += 100 each (an extra writer task between T5..T7 and T8)
 *   T10 W                     x *= 2: 482
 * Every task logs its start and end on one clock; the program checks the order the map demands
 * (each CNC-W after T0 and before T5..T7, T8 and T9 after T5..T7, T10 after T8 and T9) and that
 * two extra tasks ran. A concurrent access to a segment must be refused.
 * usage: concurrent_capi. Output: one JSON line; exit status 0 = success. */
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "xkrt_capi.h"

enum { NT = 11 };
static long x;
static int clock_;
static int start_[NT], end_[NT];
static long seen[NT];

static void body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev;
    const int * a = (const int *) xkrt_task_args(task);
    const int t = a[0], op = a[1];
    start_[t] = __atomic_add_fetch(&clock_, 1, __ATOMIC_SEQ_CST);
    struct timespec ts = {0, 2000000};
    nanosleep(&ts, NULL);                              /* gives concurrent writers a chance to overlap */
    if (op == 0) __atomic_store_n(&x, 1, __ATOMIC_SEQ_CST);
    else if (op == 1) __atomic_add_fetch(&x, 10, __ATOMIC_SEQ_CST);
    else if (op == 2) seen[t] = __atomic_load_n(&x, __ATOMIC_SEQ_CST);
    else if (op == 3) __atomic_add_fetch(&x, 100, __ATOMIC_SEQ_CST);
    else __atomic_store_n(&x, 2 * __atomic_load_n(&x, __ATOMIC_SEQ_CST), __ATOMIC_SEQ_CST);
    end_[t] = __atomic_add_fetch(&clock_, 1, __ATOMIC_SEQ_CST);
}

static int before(int p, int s) { return end_[p] < start_[s]; }

int main(void)
{
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) { fprintf(stderr, "init: %s\n", xkb_last_error()); return 1; }
    const xkrt_task_format_id_t fmt = xkrt_task_format_put(rt, "op");
    xkrt_task_format_set(rt, fmt, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) body);
    static int h;
    const int op[NT] = {0, 1, 1, 1, 1, 2, 2, 2, 3, 3, 4};
    for (int t = 0; t < NT; ++t)
    {
        xkrt_access_t a;
        memset(&a, 0, sizeof(a));
        a.type = ACCESS_TYPE_HANDLE; a.region.handle.addr = &h;
        a.mode = op[t] == 2 ? ACCESS_MODE_R : ACCESS_MODE_W;
        a.concurrency = op[t] == 1 || op[t] == 3 ? ACCESS_CONCURRENCY_CONCURRENT : ACCESS_CONCURRENCY_SEQUENTIAL;
        const int args[2] = {t, op[t]};
        xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, fmt, args, sizeof(args), &a, 1);
    }
    xkrt_task_wait(rt);
    uint64_t ran = 0, edges = 0;
    xkb_runtime_last_wait(rt, &ran, &edges, NULL, NULL, NULL);
    int st = xkb_runtime_status(rt);
    if (st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }

    int order = 1;
    for (int w = 1; w <= 4; ++w)
    {
        order &= before(0, w);
        for (int r = 5; r <= 7; ++r) order &= before(w, r);
    }
    for (int r = 5; r <= 7; ++r) order &= before(r, 8) && before(r, 9) && seen[r] == 41;
    order &= before(8, 10) && before(9, 10);

    /* concurrent mode on a segment: refused */
    static double seg[8];
    xkrt_access_t s;
    memset(&s, 0, sizeof(s));
    s.type = ACCESS_TYPE_SEGMENT; s.mode = ACCESS_MODE_W; s.concurrency = ACCESS_CONCURRENCY_CONCURRENT;
    s.region.segment.a = seg; s.region.segment.b = seg + 8;
    const int args[2] = {0, 0};
    xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, fmt, args, sizeof(args), &s, 1);
    const int refused = xkb_runtime_status(rt) == XKB_EINVAL;
    xkrt_task_wait(rt);
    xkb_runtime_status(rt);

    if (xkrt_deinit(rt) != 0) return 1;
    printf("{\"x\": %ld, \"ran\": %llu, \"edges\": %llu, \"order\": %d, \"refused\": %d}\n", x, (unsigned long long) ran,
           (unsigned long long) edges, order, refused);
    return !(x == 482 && ran == NT + 2 && order && refused);
}
