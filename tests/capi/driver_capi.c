/* The driver interface of the XKRT C API on libxkb200 (api/c/include/xkrt/xkrt.h:231-558):
 * driver and device objects, driver memory, synchronous and queued transfers, a module image
 * loaded at run time and its kernel launched with a packed argument buffer -- directly on a queue,
 * and from a CUDA task body through xkrt_task_kernel_launch / xkrt_device_kernel_launch on the
 * task's device replica -- runtime device memory, asynchronous file I/O tasks ordered before a
 * host task reading the buffer, teams, and the energy counter.
 * usage: driver_capi KERNEL.cubin SCRATCH_FILE. Output: one JSON line; exit status 0 = success. */
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "xkrt_capi.h"

#define CHECK(c) do { if (!(c)) { fprintf(stderr, "line %d: %s (%s)\n", __LINE__, #c, xkb_last_error()); return 1; } } while (0)

enum { N = 100003 };

static xkrt_driver_module_fn_t scale_fn;
static int file_checked = 0;

struct scale_args { double * p; double a; unsigned long n; };   /* the kernel's parameters, packed */

static void launcher(void * runtime, void * device, void * task, void * queue, void * cmd, xkrt_queue_command_list_counter_t idx)
{
    (void) cmd;
    struct scale_args a = {(double *) xkrt_task_access_replica((xkrt_task_t *) task, 0), 3.0, N};
    if (xkrt_device_kernel_launch((xkrt_runtime_t *) runtime, (xkrt_device_t *) device, (xkrt_queue_t *) queue, idx,
                                  (const xkrt_driver_module_fn_t *) scale_fn, (N + 255) / 256, 1, 1, 256, 1, 1, 0, &a, sizeof(a)) != 0)
        fprintf(stderr, "device kernel launch: %s\n", xkb_last_error());
}

static void scale_body(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    xkrt_task_kernel_launch(rt, dev, task, 0, launcher);
}

static void check_file(xkrt_runtime_t * rt, xkrt_device_t * dev, xkrt_task_t * task)
{
    (void) rt; (void) dev;
    const unsigned char * b = (const unsigned char *) xkrt_task_access_replica(task, 0);
    for (int i = 0; i < N; ++i)
        if (b[i] != (unsigned char) (i * 7 + 1)) return;
    file_checked = 1;
}

static xkrt_access_t segment(xkrt_access_mode_t mode, void * a, void * b)
{
    xkrt_access_t x;
    memset(&x, 0, sizeof(x));
    x.concurrency = ACCESS_CONCURRENCY_SEQUENTIAL; x.mode = mode; x.type = ACCESS_TYPE_SEGMENT;
    x.region.segment.a = a; x.region.segment.b = b;
    return x;
}

int main(int argc, char ** argv)
{
    if (argc < 3) { fprintf(stderr, "usage: %s KERNEL.cubin SCRATCH_FILE\n", argv[0]); return 2; }
    xkrt_runtime_t * rt;
    CHECK(xkrt_init(&rt) == 0);

    /* drivers and devices */
    xkrt_driver_t * cu = xkrt_driver_get(rt, XKRT_DRIVER_TYPE_CUDA), * host = xkrt_driver_get(rt, XKRT_DRIVER_TYPE_HOST);
    CHECK(cu && host && strcmp(xkrt_driver_get_name(cu), "CUDA") == 0 && strcmp(xkrt_driver_get_name(host), "HOST") == 0);
    CHECK(xkrt_driver_get_ndevices_max(cu) >= 1 && xkrt_driver_get_ndevices_max(host) == 1);
    CHECK(xkrt_driver_init(cu, 1, 0) == 0);
    xkrt_device_t * gpu = xkrt_driver_device_create(cu, 0);
    CHECK(gpu == xkrt_device_get(rt, 1) && xkrt_driver_device_create(host, 0) == xkrt_device_get(rt, HOST_DEVICE_GLOBAL_ID));
    xkrt_driver_device_init(cu, 0);
    xkrt_device_global_id_bitfield_t aff[XKRT_DEVICES_MAX] = {0};
    CHECK(xkrt_driver_device_commit(cu, 0, aff) == 0 && aff[0] == (1u << 1));
    char info[256];
    xkrt_driver_device_info(cu, 0, info, sizeof(info));
    CHECK(strstr(info, "cu device: 1") != NULL);
    CHECK(xkrt_driver_queue_suggest(cu, 0, XKRT_QUEUE_TYPE_KERN) == 8 && xkrt_driver_queue_suggest(cu, 0, XKRT_QUEUE_TYPE_H2D) == 4);

    /* driver memory and transfers: h2d, then d2d and d2h on a queue */
    const size_t bytes = N * sizeof(double);
    double * h = (double *) xkrt_driver_memory_host_allocate(cu, 0, bytes), * h2 = (double *) xkrt_driver_memory_host_allocate(cu, 0, bytes);
    double * d = (double *) xkrt_driver_memory_device_allocate(cu, 0, bytes, 0), * d2 = (double *) xkrt_driver_memory_device_allocate(cu, 0, bytes, 0);
    CHECK(h && h2 && d && d2);
    for (int i = 0; i < N; ++i) { h[i] = 0.5 * i - 7; h2[i] = 0; }
    CHECK(xkrt_driver_transfer_h2d(cu, d, h, bytes) == 0);
    xkrt_queue_t * q = xkrt_driver_queue_create(cu, gpu, XKRT_QUEUE_TYPE_D2D, 4);
    CHECK(q);
    CHECK(xkrt_driver_transfer_d2d_async(cu, d2, d, bytes, q) == 0 && xkrt_driver_transfer_d2h_async(cu, h2, d2, bytes, q) == 0);
    xkrt_driver_queue_delete(cu, q);
    CHECK(memcmp(h, h2, bytes) == 0);

    /* a module image and its kernel on a kernel queue (packed parameters) */
    FILE * f = fopen(argv[1], "rb");
    CHECK(f);
    fseek(f, 0, SEEK_END);
    const long bsz = ftell(f);
    fseek(f, 0, SEEK_SET);
    unsigned char * bin = (unsigned char *) malloc((size_t) bsz + 1);
    CHECK(bin && fread(bin, 1, (size_t) bsz, f) == (size_t) bsz);
    fclose(f);
    xkrt_driver_module_t mod = xkrt_driver_module_load(cu, 0, bin, (size_t) bsz, XKRT_DRIVER_MODULE_FORMAT_NATIVE);
    CHECK(mod);
    scale_fn = xkrt_driver_module_get_fn(cu, mod, "xkb_test_scale");
    CHECK(scale_fn);
    CHECK(xkrt_driver_module_load(host, 0, bin, (size_t) bsz, XKRT_DRIVER_MODULE_FORMAT_NATIVE) == NULL);
    xkrt_queue_t * kq = xkrt_driver_queue_create(cu, gpu, XKRT_QUEUE_TYPE_KERN, 8);
    CHECK(kq);
    struct scale_args sa = {d, -2.0, N};
    CHECK(xkrt_driver_kernel_launch(cu, kq, 5, (const xkrt_driver_module_fn_t *) scale_fn, (N + 127) / 128, 1, 1, 128, 1, 1, 0, &sa, sizeof(sa)) == 0);
    xkrt_driver_queue_delete(cu, kq);
    CHECK(xkrt_driver_transfer_d2h(cu, h2, d, bytes) == 0);
    for (int i = 0; i < N; ++i) CHECK(h2[i] == -2.0 * h[i]);
    xkrt_driver_memory_device_deallocate(cu, 0, d, bytes, 0);
    xkrt_driver_memory_device_deallocate(cu, 0, d2, bytes, 0);

    /* a CUDA task body launching the module's kernel on its replica of a host region */
    double * x = (double *) xkrt_memory_host_allocate(rt, HOST_DEVICE_GLOBAL_ID, bytes);
    CHECK(x);
    for (int i = 0; i < N; ++i) x[i] = h[i];
    xkrt_task_format_id_t fs = xkrt_task_format_put(rt, "scale");
    xkrt_task_format_set(rt, fs, XKRT_TASK_FORMAT_TARGET_CUDA, (xkrt_task_format_func_t) scale_body);
    for (int k = 0; k < 2; ++k)
    {
        xkrt_access_t a = segment(ACCESS_MODE_RW, x, x + N);
        xkrt_task_spawn_with_format_with_accesses(rt, 1, fs, NULL, 0, &a, 1);
    }
    xkrt_task_wait(rt);
    for (int i = 0; i < N; ++i) CHECK(x[i] == 9.0 * h[i]);
    xkrt_driver_module_unload(cu, mod);
    xkrt_driver_memory_host_deallocate(cu, 0, h, bytes);
    xkrt_driver_memory_host_deallocate(cu, 0, h2, bytes);

    /* runtime device memory */
    void * dm = xkrt_memory_device_allocate(rt, 1, 1 << 20);
    CHECK(dm);
    xkrt_memory_device_deallocate(rt, 1, dm);

    /* file I/O tasks: write a buffer in 5 slices, read it back in 7 into another buffer and
     * check it with a host task of the same batch (it waits for every read) */
    unsigned char * w = (unsigned char *) malloc(N), * r = (unsigned char *) malloc(N);
    CHECK(w && r);
    for (int i = 0; i < N; ++i) { w[i] = (unsigned char) (i * 7 + 1); r[i] = 0; }
    const int fd = open(argv[2], O_RDWR | O_CREAT | O_TRUNC, 0600);
    CHECK(fd >= 0);
    CHECK(xkrt_file_write_async(rt, fd, w, N, 5) == 0);
    xkrt_task_wait(rt);
    CHECK(xkrt_file_read_async(rt, fd, r, N, 7) == 0);
    xkrt_task_format_id_t fc = xkrt_task_format_put(rt, "check");
    xkrt_task_format_set(rt, fc, XKRT_TASK_FORMAT_TARGET_HOST, (xkrt_task_format_func_t) check_file);
    {
        xkrt_access_t a = segment(ACCESS_MODE_R, r, r + N);
        xkrt_task_spawn_with_format_with_accesses(rt, HOST_DEVICE_GLOBAL_ID, fc, NULL, 0, &a, 1);
    }
    xkrt_task_wait(rt);
    close(fd);
    CHECK(file_checked && memcmp(w, r, N) == 0);

    /* host registration, unified memory hints, the host driver's copies */
    CHECK(xkrt_driver_memory_host_register(cu, w, N) == 0 && xkrt_driver_memory_host_unregister(cu, w, N) == 0);
    double * u = (double *) xkrt_driver_memory_unified_allocate(cu, 0, bytes);
    CHECK(u);
    for (int i = 0; i < N; ++i) u[i] = i;
    CHECK(xkrt_driver_memory_unified_advise_device(cu, 0, u, bytes) == 0 && xkrt_driver_memory_unified_prefetch_device(cu, 0, u, bytes) == 0);
    CHECK(xkrt_driver_memory_unified_advise_host(cu, u, bytes) == 0 && xkrt_driver_memory_unified_prefetch_host(cu, u, bytes) == 0);
    CHECK(u[N - 1] == N - 1);
    xkrt_driver_memory_unified_deallocate(cu, 0, u, bytes);
    CHECK(xkrt_driver_transfer_h2d(host, r, w, 64) == 0);

    /* teams and the energy counter */
    CHECK(xkrt_team_driver_get(rt, XKRT_DRIVER_TYPE_HOST) && xkrt_team_driver_get_any(rt, 1u << XKRT_DRIVER_TYPE_HOST));
    xkrt_power_t pw;
    xkrt_driver_power_start(cu, 0, &pw);
    struct timespec ts = {0, 50 * 1000 * 1000};
    nanosleep(&ts, NULL);
    xkrt_driver_power_stop(cu, 0, &pw);
    CHECK(pw.dt >= 0.04 && pw.P >= 0);

    const int st = xkb_runtime_status(rt);
    CHECK(st == 0);
    CHECK(xkrt_deinit(rt) == 0);
    printf("{\"ok\": 1, \"power_w\": %.1f, \"info\": \"%s\"}\n", pw.P, info);
    free(bin); free(w); free(r);
    return 0;
}
