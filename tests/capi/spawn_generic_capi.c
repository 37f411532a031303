/* xkrt_task_spawn_generic through the XKRT C API on libxkb200 (api/c/include/xkrt/xkrt.h:160-171):
 *   1. a DETACHABLE task spawned with detachable_counter_initial = 2: its body returns, but the
 *      task completes only after two xkrt_task_detachable_decr (made 50 ms later by a thread the
 *      body starts), so its successor (RW on the same segment) runs after them
 *      (api/c/src/xkrt.cc:507-511, src/task.cc:249-288);
 *   2. a DETACHABLE task with counter 0 completes when its body returns;
 *   3. device tasks (the library's axpby body) spawned with a non-default ocr_access: with one GPU
 *      every owner of that access is the GPU, so the hint only has to be accepted -- y is right.
 * Output: one JSON line {"order": 1, "early": 1, "axpby": 1}. Exit status 0 = success. */
#include <pthread.h>
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "xkrt_capi.h"

static xkrt_runtime_t * rt;
static char seg_a[64], seg_b[64];
static volatile int decrements = 0, succ_saw = -1, early_succ_saw = -1, early_done = 0;
static xkrt_task_t * detached = NULL;

static void sleep_ms(int ms)
{
    struct timespec d = {0, ms * 1000L * 1000L};
    nanosleep(&d, NULL);
}

static void * decrementer(void * arg)
{
    (void) arg;
    sleep_ms(50);
    for (int k = 0; k < 2; ++k)
    {
        __atomic_add_fetch(&decrements, 1, __ATOMIC_ACQ_REL);
        xkrt_task_detachable_decr(rt, detached);
        sleep_ms(10);
    }
    return NULL;
}

static pthread_t th;

static void held_body(xkrt_runtime_t * r, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) r; (void) dev;
    detached = task;
    pthread_create(&th, NULL, decrementer, NULL);
}

static void succ_body(xkrt_runtime_t * r, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) r; (void) dev; (void) task;
    succ_saw = __atomic_load_n(&decrements, __ATOMIC_ACQUIRE);
}

static void early_body(xkrt_runtime_t * r, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) r; (void) dev; (void) task;
    early_done = 1;
}

static void early_succ_body(xkrt_runtime_t * r, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) r; (void) dev; (void) task;
    early_succ_saw = early_done;
}

static xkrt_access_t segment(xkrt_access_mode_t mode, void * a, void * b)
{
    xkrt_access_t x;
    memset(&x, 0, sizeof(x));
    x.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; x.mode = mode; x.scope = ACCESS_SCOPE_NONUNIFIED;
    x.type = ACCESS_TYPE_SEGMENT; x.region.segment.a = a; x.region.segment.b = b;
    return x;
}

int main(void)
{
    if (xkrt_init(&rt) != 0) return 1;
    const xkrt_task_format_id_t held = xkrt_task_format_put(rt, "held"), succ = xkrt_task_format_put(rt, "succ");
    const xkrt_task_format_id_t early = xkrt_task_format_put(rt, "early"), esucc = xkrt_task_format_put(rt, "early-succ");
    xkrt_task_format_set(rt, held, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) held_body);
    xkrt_task_format_set(rt, succ, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) succ_body);
    xkrt_task_format_set(rt, early, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) early_body);
    xkrt_task_format_set(rt, esucc, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) early_succ_body);

    xkrt_access_t a = segment(ACCESS_MODE_RW, seg_a, seg_a + 64), b = segment(ACCESS_MODE_RW, seg_b, seg_b + 64);
    xkrt_task_spawn_generic(rt, HOST_DEVICE_GLOBAL_ID, TASK_FLAG_DEPENDENT | TASK_FLAG_DETACHABLE, held, NULL, 0, &a, 1,
                            UNSPECIFIED_TASK_ACCESS, 2);
    xkrt_task_spawn_generic(rt, HOST_DEVICE_GLOBAL_ID, TASK_FLAG_DEPENDENT, succ, NULL, 0, &a, 1, UNSPECIFIED_TASK_ACCESS, 0);
    xkrt_task_spawn_generic(rt, HOST_DEVICE_GLOBAL_ID, TASK_FLAG_DEPENDENT | TASK_FLAG_DETACHABLE, early, NULL, 0, &b, 1,
                            UNSPECIFIED_TASK_ACCESS, 0);
    xkrt_task_spawn_generic(rt, HOST_DEVICE_GLOBAL_ID, TASK_FLAG_DEPENDENT, esucc, NULL, 0, &b, 1, UNSPECIFIED_TASK_ACCESS, 0);
    xkrt_task_wait(rt);
    pthread_join(th, NULL);
    const int st1 = xkb_runtime_status(rt);
    if (st1 != 0) { fprintf(stderr, "host batch: status %d: %s\n", st1, xkb_last_error()); return 1; }

    /* device tasks with ocr_access = 1 (the y access) */
    enum { N = 1 << 16 };
    double * x = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, N * sizeof(double));
    double * y = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, N * sizeof(double));
    for (int i = 0; i < N; ++i) { x[i] = i; y[i] = 1.0; }
    const xkrt_task_format_id_t ax = xkb_task_format_builtin(rt, XKB_TASK_AXPBY);
    for (int c = 0; c < 4; ++c)
    {
        const long lo = (long) c * N / 4, hi = (long) (c + 1) * N / 4;
        xkb_task_desc_t d;
        memset(&d, 0, sizeof(d));
        d.kind = XKB_TASK_AXPBY;
        d.u.axpby.x = (uint64_t) (uintptr_t) x; d.u.axpby.y = (uint64_t) (uintptr_t) y;
        d.u.axpby.lo = lo; d.u.axpby.hi = hi; d.u.axpby.a = 2.0; d.u.axpby.b = 3.0;
        xkrt_access_t acc[2] = {segment(ACCESS_MODE_R, x + lo, x + hi), segment(ACCESS_MODE_RW, y + lo, y + hi)};
        xkrt_task_spawn_generic(rt, 1, TASK_FLAG_DEVICE | TASK_FLAG_DEPENDENT, ax, &d, sizeof(d), acc, 2, 1, 0);
    }
    xkrt_task_wait(rt);
    const int st2 = xkb_runtime_status(rt);
    if (st2 != 0) { fprintf(stderr, "device batch: status %d: %s\n", st2, xkb_last_error()); return 1; }
    int ax_ok = 1;
    for (int i = 0; i < N; ++i) if (y[i] != 2.0 * i + 3.0) { ax_ok = 0; break; }
    if (xkrt_deinit(rt) != 0) { fprintf(stderr, "deinit: %s\n", xkb_last_error()); return 1; }
    printf("{\"order\": %d, \"early\": %d, \"axpby\": %d}\n", succ_saw == 2, early_succ_saw == 1, ax_ok);
    return succ_saw == 2 && early_succ_saw == 1 && ax_ok ? 0 : 1;
}
