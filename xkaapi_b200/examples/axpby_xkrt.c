/* axpby task chains through the XKRT C API on libxkb200: y = a*x + b*y over N FP64 elements,
 * PASSES passes, each pass cut into seeded chunks whose byte sizes are log-uniform in
 * [CMIN, CMAX] (multiples of 8) with a per-pass random start, so the chunk boundaries of
 * consecutive passes overlap and every chunk task depends on the tasks of the previous pass
 * whose chunks it intersects. A task reads its x chunk (segment access R) and updates its y chunk
 * (segment access RW) -- the access pattern of the reference's axpby example
 * (examples/task-axpby.cc:108-118) with FP64 data. a, b are drawn per pass in [-2, 2].
 *
 * One repetition = xkrt_init, x and y from xkrt_memory_host_allocate filled with the seeded
 * inputs (untimed), then the timed part -- spawn every task, xkrt_task_wait: dependency
 * resolution on the GPU, first-touch copies of x and y to the device, the graph on the
 * persistent scheduler (chunks longer than the runtime's split size run as several slices),
 * the write-back of y -- then xkrt_deinit.
 *
 * usage: axpby_xkrt N PASSES SEED REPS CMIN CMAX [x.bin y.bin out.bin]
 * Output: one JSON line per repetition {rep, tasks, seconds, tasks_per_s, spawn_s, resolve_ms,
 * coherency_ms, run_ms, writeback_ms, edges, h2d_bytes, d2h_bytes, fused, checksum, coef}. */
#include <math.h>
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

static uint64_t splitmix(uint64_t * s)
{
    uint64_t z = (*s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static double unit(uint64_t * s) { return (double) (splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

static xkrt_access_t segment(xkrt_access_mode_t mode, const double * base, int64_t lo, int64_t hi)
{
    xkrt_access_t a;
    memset(&a, 0, sizeof(a));
    a.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; a.mode = mode; a.scope = ACCESS_SCOPE_NONUNIFIED;
    a.type = ACCESS_TYPE_SEGMENT;
    a.region.segment.a = (void *) (base + lo); a.region.segment.b = (void *) (base + hi);
    return a;
}

int main(int argc, char ** argv)
{
    if (argc < 7)
    {
        fprintf(stderr, "usage: %s N PASSES SEED REPS CMIN CMAX [x.bin y.bin out.bin]\n", argv[0]);
        return 2;
    }
    const int64_t n = atoll(argv[1]);
    const int passes = atoi(argv[2]);
    const uint64_t seed = strtoull(argv[3], NULL, 10);
    const int reps = atoi(argv[4]);
    const double cmin = atof(argv[5]), cmax = atof(argv[6]);
    const char * xin = argc > 9 ? argv[7] : NULL, * yin = argc > 9 ? argv[8] : NULL, * out = argc > 9 ? argv[9] : NULL;
    if (n < 1 || passes < 1 || reps < 1 || !(cmin >= 8) || !(cmax >= cmin)) { fprintf(stderr, "bad arguments\n"); return 2; }

    double * x0 = (double *) malloc((size_t) n * sizeof(double)), * y0 = (double *) malloc((size_t) n * sizeof(double));
    if (!x0 || !y0) return 3;
    uint64_t s = seed;
    if (xin)
    {
        FILE * f = fopen(xin, "rb"), * g = fopen(yin, "rb");
        if (!f || !g || fread(x0, sizeof(double), (size_t) n, f) != (size_t) n || fread(y0, sizeof(double), (size_t) n, g) != (size_t) n)
        { fprintf(stderr, "cannot read inputs\n"); return 3; }
        fclose(f); fclose(g);
        s += 2 * (uint64_t) n * 0x9e3779b97f4a7c15ull;   /* the plan draws follow the 2n input draws */
    }
    else
    {
        for (int64_t i = 0; i < n; ++i) x0[i] = 2.0 * unit(&s) - 1.0;
        for (int64_t i = 0; i < n; ++i) y0[i] = 2.0 * unit(&s) - 1.0;
    }
    /* chunk plan and coefficients, one draw sequence for every repetition */
    double * coef = (double *) malloc(2 * (size_t) passes * sizeof(double));
    int64_t cap = 1024, nb = 0;
    int64_t * bounds = (int64_t *) malloc((size_t) cap * sizeof(int64_t));   /* per pass: 0, cuts..., n */
    int * pass_end = (int *) malloc((size_t) passes * sizeof(int));
    if (!coef || !bounds || !pass_end) return 3;
    const double lmin = log(cmin), lmax = log(cmax);
    for (int p = 0; p < passes; ++p)
    {
        coef[2 * p] = 4.0 * unit(&s) - 2.0;
        coef[2 * p + 1] = 4.0 * unit(&s) - 2.0;
        int64_t at = 0;
        int first = 1;
        while (at < n)
        {
            int64_t len = (int64_t) (exp(lmin + (lmax - lmin) * unit(&s)) / 8.0);
            if (len < 1) len = 1;
            if (first) { len = 1 + (int64_t) (unit(&s) * (double) len); first = 0; }   /* per-pass random start */
            if (nb + 2 > cap) { cap *= 2; bounds = (int64_t *) realloc(bounds, (size_t) cap * sizeof(int64_t)); if (!bounds) return 3; }
            bounds[nb++] = at;
            at = at + len < n ? at + len : n;
        }
        bounds[nb++] = n;
        pass_end[p] = (int) nb;
    }

    for (int rep = 0; rep < reps; ++rep)
    {
        xkrt_runtime_t * rt;
        if (xkrt_init(&rt) != 0) { fprintf(stderr, "xkrt_init: %s\n", xkb_last_error()); return 1; }
        double * x = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, (size_t) n * sizeof(double));
        double * y = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, (size_t) n * sizeof(double));
        if (!x || !y) { fprintf(stderr, "host allocation: %s\n", xkb_last_error()); return 1; }
        memcpy(x, x0, (size_t) n * sizeof(double));
        memcpy(y, y0, (size_t) n * sizeof(double));
        const xkrt_task_format_id_t fmt = xkb_task_format_builtin(rt, XKB_TASK_AXPBY);

        const double t0 = now_s();
        xkb_task_desc_t d;
        memset(&d, 0, sizeof(d));
        d.kind = XKB_TASK_AXPBY;
        d.u.axpby.x = (uint64_t) (uintptr_t) x; d.u.axpby.y = (uint64_t) (uintptr_t) y;
        int b = 0;
        for (int p = 0; p < passes; ++p)
        {
            d.u.axpby.a = coef[2 * p]; d.u.axpby.b = coef[2 * p + 1];
            for (; b + 1 < pass_end[p]; ++b)
            {
                d.u.axpby.lo = bounds[b]; d.u.axpby.hi = bounds[b + 1];
                xkrt_access_t acc[2] = {segment(ACCESS_MODE_R, x, bounds[b], bounds[b + 1]),
                                        segment(ACCESS_MODE_RW, y, bounds[b], bounds[b + 1])};
                xkrt_task_spawn_with_format_with_accesses(rt, 1, fmt, &d, sizeof(d), acc, 2);
            }
            ++b;                                          /* skip the pass's closing bound */
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
        for (int64_t i = 0; i < n; ++i) checksum += y[i];
        if (out && rep == reps - 1)
        {
            FILE * f = fopen(out, "wb");
            if (!f || fwrite(y, sizeof(double), (size_t) n, f) != (size_t) n) return 3;
            fclose(f);
        }
        const int st = xkb_runtime_status(rt);
        if (st != 0) { fprintf(stderr, "status %d: %s\n", st, xkb_last_error()); return 1; }
        if (xkrt_deinit(rt) != 0) { fprintf(stderr, "xkrt_deinit: %s\n", xkb_last_error()); return 1; }
        printf("{\"rep\": %d, \"tasks\": %llu, \"seconds\": %.6f, \"tasks_per_s\": %.1f, \"spawn_s\": %.6f, "
               "\"resolve_ms\": %.3f, \"coherency_ms\": %.3f, \"run_ms\": %.3f, \"writeback_ms\": %.3f, \"edges\": %llu, "
               "\"h2d_bytes\": %llu, \"d2h_bytes\": %llu, \"fused\": %d, \"checksum\": %.17g, \"coef\": [",
               rep, (unsigned long long) tasks, t2 - t0, (double) tasks / (t2 - t0), t1 - t0, ms[0], ms[1], ms[2], ms[3],
               (unsigned long long) edges, (unsigned long long) h2d_bytes, (unsigned long long) d2h_bytes, fused, checksum);
        for (int p = 0; p < passes; ++p) printf("%s[%.17g, %.17g]", p ? ", " : "", coef[2 * p], coef[2 * p + 1]);
        printf("]}\n");
        fflush(stdout);
    }
    free(x0); free(y0); free(coef); free(bounds); free(pass_end);
    return 0;
}
