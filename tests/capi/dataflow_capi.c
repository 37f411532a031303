/* Dataflow execution of a batch of host tasks through the XKRT C API on libxkb200:
 *   1. WIDE independent tasks that each sleep 20 ms: ready tasks run on several host threads at
 *      once (the peak number of bodies running together is reported with the wall time);
 *   2. K chains of L tasks, chain k updating (RW) its own segment, then one task updating all K
 *      segments: each chain runs in spawn order and the last task runs after every chain;
 *   3. a detached task (xkrt_task_detachable_incr in its body) completed by an independent task's
 *      body (xkrt_task_detachable_decr), restating tests/api/c detachable tasks: its successor runs
 *      after the completion. With one host thread this finishes too, so a detached task holds no
 *      thread while it waits.
 * Output: one JSON line {"peak": P, "wide_s": S}. Exit status 0 = success. */
#include <stdio.h>
#include <string.h>
#include <time.h>

#include "xkrt_capi.h"

enum { WIDE = 48, K = 8, L = 50 };

static int running = 0, peak = 0, errors = 0;
static int chain_pos[K];
static char seg[K][64];

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double) ts.tv_sec + 1e-9 * (double) ts.tv_nsec;
}

static void sleep_ms(int ms)
{
    struct timespec d = {0, ms * 1000L * 1000L};
    nanosleep(&d, NULL);
}

static void wide_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev; (void) task;
    const int r = __atomic_add_fetch(&running, 1, __ATOMIC_ACQ_REL);
    int p = __atomic_load_n(&peak, __ATOMIC_ACQUIRE);
    while (r > p && !__atomic_compare_exchange_n(&peak, &p, r, 0, __ATOMIC_ACQ_REL, __ATOMIC_ACQUIRE)) {}
    sleep_ms(20);
    __atomic_sub_fetch(&running, 1, __ATOMIC_ACQ_REL);
}

/* args {chain, position}; the join task has chain = K */
static void chain_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev;
    const int * a = (const int *) xkrt_task_args(task);
    if (a[0] == K)
    {
        for (int k = 0; k < K; ++k)
            if (chain_pos[k] != L) { fprintf(stderr, "join ran with chain %d at %d\n", k, chain_pos[k]); __atomic_add_fetch(&errors, 1, __ATOMIC_RELAXED); }
        return;
    }
    if (chain_pos[a[0]] != a[1]) { fprintf(stderr, "chain %d task %d ran at %d\n", a[0], a[1], chain_pos[a[0]]); __atomic_add_fetch(&errors, 1, __ATOMIC_RELAXED); }
    seg[a[0]][a[1] % 64] ^= 1;
    ++chain_pos[a[0]];
}

static xkrt_task_t * detached_task = NULL;
static int completer_done = 0, successor_ran = 0;

static void detached_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) dev;
    xkrt_task_detachable_incr(rt, task);
    __atomic_store_n(&detached_task, task, __ATOMIC_RELEASE);
}

static void completer_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) dev; (void) task;
    xkrt_task_t * d;
    const double t0 = now_s();
    while (!(d = __atomic_load_n(&detached_task, __ATOMIC_ACQUIRE)))       /* the detached body ran first */
    {
        if (now_s() - t0 > 30) { fprintf(stderr, "detached body never ran\n"); __atomic_add_fetch(&errors, 1, __ATOMIC_RELAXED); return; }
        sleep_ms(1);
    }
    sleep_ms(10);
    __atomic_store_n(&completer_done, 1, __ATOMIC_RELEASE);
    xkrt_task_detachable_decr(rt, d);
}

static void successor_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev; (void) task;
    if (!__atomic_load_n(&completer_done, __ATOMIC_ACQUIRE)) { fprintf(stderr, "successor ran before the completion\n"); ++errors; }
    successor_ran = 1;
}

static xkrt_access_t segment(xkrt_access_mode_t mode, void * a, void * b)
{
    xkrt_access_t x;
    memset(&x, 0, sizeof(x));
    x.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; x.mode = mode; x.type = ACCESS_TYPE_SEGMENT;
    x.region.segment.a = a; x.region.segment.b = b;
    return x;
}

static xkrt_access_t handle(xkrt_access_mode_t mode, void * h)
{
    xkrt_access_t x;
    memset(&x, 0, sizeof(x));
    x.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; x.mode = mode; x.type = ACCESS_TYPE_HANDLE;
    x.region.handle.addr = h;
    return x;
}

static xkrt_task_format_id_t host_format(xkrt_runtime_t * rt, const char * name, void (*f)(xkrt_runtime_t *, xkrt_device_t *, xkrt_task_t *))
{
    xkrt_task_format_id_t id = xkrt_task_format_put(rt, name);
    xkrt_task_format_set(rt, id, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) f);
    return id;
}

int main(void)
{
    xkrt_runtime_t * rt;
    if (xkrt_init(&rt) != 0) { fprintf(stderr, "init: %s\n", xkb_last_error()); return 1; }

    /* 1. independent tasks */
    const xkrt_task_format_id_t wide = host_format(rt, "wide", wide_body);
    const double t0 = now_s();
    for (int t = 0; t < WIDE; ++t) xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, wide, NULL, 0, NULL, 0);
    xkrt_task_wait(rt);
    const double wide_s = now_s() - t0;

    /* 2. chains, then a join over every chain's segment */
    const xkrt_task_format_id_t chain = host_format(rt, "chain", chain_body);
    for (int p = 0; p < L; ++p)
        for (int k = 0; k < K; ++k)
        {
            const int args[2] = {k, p};
            xkrt_access_t a = segment(ACCESS_MODE_RW, seg[k], seg[k] + 64);
            xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, chain, args, sizeof(args), &a, 1);
        }
    {
        const int args[2] = {K, 0};
        xkrt_access_t a = segment(ACCESS_MODE_RW, seg[0], seg[K - 1] + 64);
        xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, chain, args, sizeof(args), &a, 1);
    }
    xkrt_task_wait(rt);

    /* 3. a detached task completed by an independent task */
    static int h1, h2;
    const xkrt_task_format_id_t det = host_format(rt, "detached", detached_body);
    const xkrt_task_format_id_t cmp = host_format(rt, "completer", completer_body);
    const xkrt_task_format_id_t suc = host_format(rt, "successor", successor_body);
    xkrt_access_t w1 = handle(ACCESS_MODE_W, &h1), r1 = handle(ACCESS_MODE_R, &h1), w2 = handle(ACCESS_MODE_W, &h2);
    xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, det, NULL, 0, &w1, 1);
    xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, cmp, NULL, 0, &w2, 1);
    xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, suc, NULL, 0, &r1, 1);
    xkrt_task_wait(rt);

    const int st = xkb_runtime_status(rt);
    if (xkrt_deinit(rt) != 0 || st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
    for (int k = 0; k < K; ++k)
        if (chain_pos[k] != L) { fprintf(stderr, "chain %d ran %d of %d tasks\n", k, chain_pos[k], L); return 1; }
    if (errors || !successor_ran) { fprintf(stderr, "errors %d successor %d\n", errors, successor_ran); return 1; }
    printf("{\"peak\": %d, \"wide_s\": %.4f}\n", peak, wide_s);
    return 0;
}
