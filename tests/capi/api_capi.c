/* The rest of the XKRT C API on libxkb200: device and driver objects, the current task, detached
 * completion from another thread (restating the detachable pattern of tests/api/c), unified
 * memory used in place by a device task, and the calls this runtime refuses (commit, enqueue).
 * Exit status 0 = success. */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "xkrt_capi.h"

static xkrt_runtime_t * RT;
static int order[4], norder = 0, errors = 0;

struct detach_arg { xkrt_task_t * task; };

static void * finish_later(void * p)
{
    struct detach_arg * a = (struct detach_arg *) p;
    struct timespec d = {0, 20 * 1000 * 1000};
    nanosleep(&d, NULL);                         /* the successor must not run before this */
    order[norder++] = 1;
    xkrt_task_detachable_decr(RT, a->task);
    return NULL;
}

static pthread_t thr;
static struct detach_arg darg;

static void detached_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    if (xkrt_task_current(rt) != task) ++errors;
    if (dev != xkrt_device_get(rt, HOST_DEVICE_GLOBAL_ID)) ++errors;
    if (xkrt_device_driver_get(rt, dev) != xkrt_driver_get(rt, XKRT_DRIVER_TYPE_HOST)) ++errors;
    order[norder++] = 0;
    xkrt_task_detachable_incr(rt, task);
    darg.task = task;
    pthread_create(&thr, NULL, finish_later, &darg);
}

static void after_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev; (void) task;
    order[norder++] = 2;
}

static double sum_y;
static void read_unified(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev;
    const double * y = (const double *) xkrt_task_access_replica(task, 0);
    for (int i = 0; i < 1000; ++i) sum_y += y[i];
}

static xkrt_access_t segment(xkrt_access_mode_t mode, void * a, void * b)
{
    xkrt_access_t x;
    memset(&x, 0, sizeof(x));
    x.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; x.mode = mode; x.type = ACCESS_TYPE_SEGMENT;
    x.region.segment.a = a; x.region.segment.b = b;
    return x;
}

int main(void)
{
    if (xkrt_init(&RT) != 0) return 1;
    if (xkrt_get_ndevices(RT) != 2 || xkrt_get_ndevices_max(RT) < 2) { fprintf(stderr, "devices\n"); return 1; }
    if (!xkrt_driver_get(RT, XKRT_DRIVER_TYPE_CUDA) || xkrt_driver_get(RT, XKRT_DRIVER_TYPE_ZE)) { fprintf(stderr, "drivers\n"); return 1; }
    if (xkrt_device_driver_get(RT, xkrt_device_get(RT, 1)) != xkrt_driver_get(RT, XKRT_DRIVER_TYPE_CUDA)) { fprintf(stderr, "gpu driver\n"); return 1; }
    xkrt_logger_info("api_capi: logger reachable");

    /* detached task, then a successor on the same handle */
    static int obj;
    xkrt_task_format_id_t d = xkrt_task_format_put(RT, "detached"), a = xkrt_task_format_put(RT, "after");
    xkrt_task_format_set(RT, d, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) detached_body);
    xkrt_task_format_set(RT, a, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) after_body);
    xkrt_access_t h;
    memset(&h, 0, sizeof(h));
    h.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; h.mode = ACCESS_MODE_RW; h.type = ACCESS_TYPE_HANDLE; h.region.handle.addr = &obj;
    xkrt_task_spawn_with_format_with_accesses(RT, HOST_DEVICE_GLOBAL_ID, d, NULL, 0, &h, 1);
    xkrt_task_spawn_with_format_with_accesses(RT, HOST_DEVICE_GLOBAL_ID, a, NULL, 0, &h, 1);
    xkrt_task_wait(RT);
    pthread_join(thr, NULL);
    if (norder != 3 || order[0] != 0 || order[1] != 1 || order[2] != 2 || errors) { fprintf(stderr, "detach order\n"); return 1; }

    /* unified memory: a device axpby task on it, then a host task reading it in place */
    double * x = (double *) xkrt_memory_unified_allocate(RT, 1, 1000 * sizeof(double));
    double * y = (double *) xkrt_memory_unified_allocate(RT, 1, 1000 * sizeof(double));
    if (!x || !y) { fprintf(stderr, "unified: %s\n", xkb_last_error()); return 1; }
    for (int i = 0; i < 1000; ++i) { x[i] = i; y[i] = 1.0; }
    xkrt_task_format_id_t ax = xkb_task_format_builtin(RT, XKB_TASK_AXPBY), rd = xkrt_task_format_put(RT, "read");
    xkrt_task_format_set(RT, rd, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) read_unified);
    xkb_task_desc_t t;
    memset(&t, 0, sizeof(t));
    t.kind = XKB_TASK_AXPBY; t.u.axpby.x = (uint64_t) (uintptr_t) x; t.u.axpby.y = (uint64_t) (uintptr_t) y;
    t.u.axpby.lo = 0; t.u.axpby.hi = 1000; t.u.axpby.a = 2.0; t.u.axpby.b = 3.0;
    xkrt_access_t acc[2] = {segment(ACCESS_MODE_R, x, x + 1000), segment(ACCESS_MODE_RW, y, y + 1000)};
    xkrt_task_spawn_with_format_with_accesses(RT, 1, ax, &t, sizeof(t), acc, 2);
    xkrt_access_t ry = segment(ACCESS_MODE_R, y, y + 1000);
    xkrt_task_spawn_with_format_with_accesses(RT, HOST_DEVICE_GLOBAL_ID, rd, NULL, 0, &ry, 1);
    xkrt_task_wait(RT);
    uint64_t h2d = 0, d2h = 0;
    xkb_runtime_last_wait_bytes(RT, &h2d, &d2h);
    double want = 0;
    for (int i = 0; i < 1000; ++i) want += 2.0 * i + 3.0;
    if (sum_y != want || h2d != 0 || d2h != 0) { fprintf(stderr, "unified: sum %g want %g, copies %llu/%llu\n", sum_y, want,
                                                (unsigned long long) h2d, (unsigned long long) d2h); return 1; }

    /* refused calls record an error and leave the runtime usable */
    if (xkb_runtime_status(RT) != 0) { fprintf(stderr, "status: %s\n", xkb_last_error()); return 1; }
    xkrt_task_commit(RT, NULL);
    if (xkb_runtime_status(RT) != XKB_EINVAL) { fprintf(stderr, "commit not refused\n"); return 1; }
    if (xkrt_deinit(RT) != 0) return 1;
    printf("{\"ok\": 1}\n");
    return 0;
}
