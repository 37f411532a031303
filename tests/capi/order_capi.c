/* Ordering tests through the XKRT C API, restating the reference's tests:
 *   tests/task-dependency-interval.cc:83-121         W [x-64,x+64) -> R [x,x+76) -> RW [x-12,x+48)
 *   tests/task-dependency-interval-matrix.cc:84-160  interval W [0,100) -> matrix W (3, ld 8, 8x8, s=1)
 *                                                    -> interval W [0,100)
 *   tests/api/c/task-with-access.c:52-90             a team task with a VW segment access
 *   tests/task-dependency-handle.cc:86-119           W -> R -> RW on one handle
 * Each chain's host task bodies check that they run in spawn order (each finds its chain's counter
 * at its own index); independent chains may run at the same time. Exit status 0 = success. */
#include <stdio.h>
#include <stdlib.h>

#include "xkrt_capi.h"

static int counter[3] = {0, 0, 0}, errors = 0, with_access_ran = 0;

/* args: {chain, position in the chain}; tasks of one chain never overlap in time */
static void ordered(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev;
    const int * a = (const int *) xkrt_task_args(task);
    if (a[1] != counter[a[0]]) { fprintf(stderr, "chain %d task %d ran at position %d\n", a[0], a[1], counter[a[0]]); __atomic_add_fetch(&errors, 1, __ATOMIC_RELAXED); }
    ++counter[a[0]];
}

static void with_access(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task, void * ud)
{
    (void) rt; (void) dev; (void) task; (void) ud;
    with_access_ran = 1;
}

static xkrt_access_t segment(xkrt_access_mode_t mode, void * a, void * b)
{
    xkrt_access_t x = {ACCESS_CONCURRENCY_SEQUENTIAL, mode, ACCESS_SCOPE_NONUNIFIED, ACCESS_TYPE_SEGMENT, {{0}}};
    x.region.segment.a = a; x.region.segment.b = b;
    return x;
}

int main(void)
{
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) { fprintf(stderr, "init: %s\n", xkb_last_error()); return 1; }
    xkrt_task_format_id_t fmt = xkrt_task_format_put(rt, "ordered");
    xkrt_task_format_set(rt, fmt, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) ordered);

    /* interval chain */
    static int x[64];
    char * X = (char *) &x[32];
    xkrt_access_mode_t modes[3] = {ACCESS_MODE_W, ACCESS_MODE_R, ACCESS_MODE_RW};
    char * lo[3] = {X - 64, X, X - 12}, * hi[3] = {X + 64, X + 76, X + 48};
    for (int t = 0; t < 3; ++t)
    {
        xkrt_access_t a = segment(modes[t], lo[t], hi[t]);
        const int args[2] = {0, t};
        xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, fmt, args, sizeof(args), &a, 1);
    }
    /* interval -> matrix -> interval */
    for (int t = 3; t < 6; ++t)
    {
        xkrt_access_t a;
        if (t == 4)
        {
            a = (xkrt_access_t) {ACCESS_CONCURRENCY_SEQUENTIAL, ACCESS_MODE_W, ACCESS_SCOPE_NONUNIFIED, ACCESS_TYPE_BLAS_MATRIX, {{0}}};
            a.region.matrix.storage = MATRIX_COLMAJOR; a.region.matrix.addr = (void *) 3; a.region.matrix.ld = 8;
            a.region.matrix.m = 8; a.region.matrix.n = 8; a.region.matrix.sizeof_type = 1;
        }
        else a = segment(ACCESS_MODE_W, (void *) 0, (void *) 100);
        const int args[2] = {1, t - 3};
        xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, fmt, args, sizeof(args), &a, 1);
    }
    xkrt_task_wait(rt);
    uint64_t tasks = 0, edges = 0;
    xkb_runtime_last_wait(rt, &tasks, &edges, NULL, NULL, NULL);

    /* handle chain: the handle names an object, not memory */
    for (int t = 6; t < 9; ++t)
    {
        xkrt_access_t a = {ACCESS_CONCURRENCY_SEQUENTIAL, modes[t - 6], ACCESS_SCOPE_NONUNIFIED, ACCESS_TYPE_HANDLE, {{0}}};
        a.region.handle.addr = &counter[2];
        const int args[2] = {2, t - 6};
        xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, fmt, args, sizeof(args), &a, 1);
    }
    xkrt_task_wait(rt);
    uint64_t hedges = 0;
    xkb_runtime_last_wait(rt, NULL, &hedges, NULL, NULL, NULL);

    /* team task with a virtual write */
    xkrt_team_t * team = xkrt_team_driver_device_get(rt, XKRT_DRIVER_TYPE_HOST, 0);
    xkrt_access_t vw = segment(ACCESS_MODE_VW, (void *) 0, (void *) 1);
    xkrt_team_task_spawn_with_accesses(rt, team, with_access, NULL, &vw, 1);
    xkrt_task_wait(rt);

    const int st = xkb_runtime_status(rt);
    if (xkrt_deinit(rt) != 0 || st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
    if (counter[0] != 3 || counter[1] != 3 || counter[2] != 3 || errors || !with_access_ran)
    { fprintf(stderr, "counters %d %d %d errors %d\n", counter[0], counter[1], counter[2], errors); return 1; }
    printf("{\"tasks\": %llu, \"edges\": %llu, \"handle_edges\": %llu}\n", (unsigned long long) tasks, (unsigned long long) edges,
           (unsigned long long) hedges);
    return 0;
}
