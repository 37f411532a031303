/* XKRT C API (task spawn / access / wait) implemented on libxkb200.
 *
 * The names, enum values, typedefs and the xkrt_access_t layout are those of the reference's C
 * API (api/c/include/xkrt/xkrt.h:61-566 and the headers it includes: memory/access/mode.h,
 * concurrency.h, scope.h, type.h, blas/matrix-storage.h, task/flag.h, task/format.h,
 * driver/driver-type.h, consts.h), so a C program written against that API compiles against
 * this header and links against libxkb200.so: runtime init/deinit, task formats, task spawn with
 * segment, matrix and handle accesses, task wait and completion, task argument/access accessors,
 * host / device / unified memory, asynchronous file I/O tasks, and the driver interface (queues,
 * transfers, modules, kernel launches) of the host and the GPU.
 *
 * Execution model: spawned tasks are resolved on the GPU (xkb_resolver) by a background worker
 * while the program keeps spawning, their data made coherent where they run (resident planner:
 * one device mirror per registered host region, H2D/D2H only for blocks the target lacks), and
 * run -- built-in device bodies on the device scheduler's persistent kernel, window by window
 * as soon as they are resolved while every task so far is one; otherwise, at xkrt_task_wait, as
 * a dataflow graph on a team of host threads, each with its own CUDA stream. xkrt_task_wait
 * returns when every task completed and host memory is coherent again. Handle accesses order tasks like the
 * reference's DependencyMap (they carry no data), concurrent-mode ones included: where the
 * reference's map inserts an extra empty writer task (dependency-map.hpp:93-137) the batch gets
 * one, a host task with no body spawned just before the task that needed it (it counts among
 * the batch's tasks). Two rare forms are ordered at least as strictly as the reference, not edge
 * for edge (xkb_handle_map_expand in xkrt_b200.h names them). Concurrent mode on a segment or
 * matrix access is rejected (XKB_EINVAL; the reference asserts it away) and user moldable tasks
 * are not supported. Functions that return void in the reference record failures instead; read
 * them with xkb_runtime_status().
 */
#ifndef XKRT_B200_CAPI_H
#define XKRT_B200_CAPI_H

#include <stddef.h>
#include <stdint.h>

#include "xkrt_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef void * xkrt_runtime_t;
typedef void * xkrt_task_t;
typedef void * xkrt_team_t;
typedef void * xkrt_driver_t;
typedef void * xkrt_device_t;
typedef void * xkrt_queue_t;
typedef void * xkrt_command_t;

typedef uint8_t  xkrt_device_global_id_t;
typedef uint8_t  xkrt_device_driver_id_t;
typedef uint16_t xkrt_task_wait_counter_type_t;
typedef uint16_t xkrt_task_access_counter_type_t;
typedef uint8_t  xkrt_task_flag_bitfield_t;
typedef uint8_t  xkrt_task_format_id_t;
typedef uint16_t xkrt_device_global_id_bitfield_t;
typedef uint8_t  xkrt_driver_type_bitfield_t;
typedef unsigned int xkrt_queue_command_list_counter_t;

#define HOST_DEVICE_GLOBAL_ID        ((xkrt_device_global_id_t) 0)
#define XKRT_DEVICES_MAX             (16)
#define UNSPECIFIED_DEVICE_GLOBAL_ID (XKRT_DEVICES_MAX)
#define TASK_MAX_ACCESSES            (1024)
#define UNSPECIFIED_TASK_ACCESS      ((xkrt_task_access_counter_type_t) TASK_MAX_ACCESSES)
#define XKRT_TASK_FORMAT_NULL        0

typedef enum xkrt_access_concurrency_t {
    ACCESS_CONCURRENCY_SEQUENTIAL  = 0x1,
    ACCESS_CONCURRENCY_COMMUTATIVE = 0x2,
    ACCESS_CONCURRENCY_CONCURRENT  = 0x4
} xkrt_access_concurrency_t;

typedef enum xkrt_access_mode_t {
    ACCESS_MODE_R  = 0x1,
    ACCESS_MODE_W  = 0x2,
    ACCESS_MODE_RW = 0x3,
    ACCESS_MODE_V  = 0x4,
    ACCESS_MODE_VW = 0x6,
    ACCESS_MODE_VR = 0x5,
    ACCESS_MODE_D  = 0x8
} xkrt_access_mode_t;

typedef enum xkrt_access_scope_t {
    ACCESS_SCOPE_NONUNIFIED = 0,
    ACCESS_SCOPE_UNIFIED    = 1
} xkrt_access_scope_t;

typedef enum xkrt_access_type_t {
    ACCESS_TYPE_HANDLE      = 0,
    ACCESS_TYPE_SEGMENT     = 1,
    ACCESS_TYPE_BLAS_MATRIX = 2,
    ACCESS_TYPE_NULL        = 3,
    ACCESS_TYPE_MAX         = 4
} xkrt_access_type_t;

typedef enum xkrt_matrix_storage_t {
    MATRIX_ROWMAJOR,
    MATRIX_COLMAJOR
} xkrt_matrix_storage_t;

typedef enum xkrt_task_flags_t {
    TASK_FLAG_ZERO       = 0,
    TASK_FLAG_DEPENDENT  = 1 << 0,
    TASK_FLAG_DETACHABLE = 1 << 1,
    TASK_FLAG_DEVICE     = 1 << 2,
    TASK_FLAG_DOMAIN     = 1 << 3,
    TASK_FLAG_MOLDABLE   = 1 << 4,
    TASK_FLAG_REQUEUE    = 1 << 7,
    TASK_FLAG_MAX        = 1 << 8
} xkrt_task_flags_t;

typedef enum xkrt_task_format_target_t {
    XKRT_TASK_FORMAT_TARGET_HOST = 0,
    XKRT_TASK_FORMAT_TARGET_CUDA = 1,
    XKRT_TASK_FORMAT_TARGET_ZE   = 2,
    XKRT_TASK_FORMAT_TARGET_CL   = 3,
    XKRT_TASK_FORMAT_TARGET_HIP  = 4,
    XKRT_TASK_FORMAT_TARGET_SYCL = 5,
    XKRT_TASK_FORMAT_TARGET_MAX  = 6
} xkrt_task_format_target_t;

typedef enum xkrt_driver_type_t {
    XKRT_DRIVER_TYPE_HOST = 0,
    XKRT_DRIVER_TYPE_CUDA = 1,
    XKRT_DRIVER_TYPE_ZE   = 2,
    XKRT_DRIVER_TYPE_CL   = 3,
    XKRT_DRIVER_TYPE_HIP  = 4,
    XKRT_DRIVER_TYPE_SYCL = 5,
    XKRT_DRIVER_TYPE_MAX  = 6
} xkrt_driver_type_t;

/* format bodies are called as f(runtime, device, task) (the reference's task_execute) */
typedef void (*xkrt_task_format_func_t)();
typedef void (*xkrt_task_func_t)(xkrt_runtime_t * runtime, xkrt_device_t * device, xkrt_task_t * task, void * user_data);

typedef struct xkrt_access_t {
    xkrt_access_concurrency_t concurrency;
    xkrt_access_mode_t        mode;
    xkrt_access_scope_t       scope;
    xkrt_access_type_t        type;
    union xkrt_region_t {
        struct xkrt_handle_t { void * addr; } handle;
        struct xkrt_segment_t { void * a; void * b; } segment;
        struct xkrt_matrix_t {
            xkrt_matrix_storage_t storage;
            void * addr;
            unsigned long ld;
            unsigned long offset_m;
            unsigned long offset_n;
            unsigned long m;
            unsigned long n;
            unsigned long sizeof_type;
        } matrix;
    } region;
} xkrt_access_t;

/* runtime (api/c/include/xkrt/xkrt.h:105-108) */
XKB_API int  xkrt_init(xkrt_runtime_t ** runtime);
XKB_API int  xkrt_deinit(xkrt_runtime_t * runtime);
XKB_API void xkrt_reset(xkrt_runtime_t * runtime);

/* memory (xkrt.h:110-124): host allocations and registrations are the regions that get device
 * mirrors; data a device task touches must lie in one of them */
XKB_API int    xkrt_memory_register(xkrt_runtime_t * runtime, void * ptr, size_t size);
XKB_API int    xkrt_memory_unregister(xkrt_runtime_t * runtime, void * ptr, size_t size);
XKB_API void * xkrt_memory_host_allocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, size_t size);
XKB_API void   xkrt_memory_host_deallocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, void * ptr, size_t size);

/* memory (xkrt.h:112-125): async registration is synchronous here; unified allocations are
 * used in place by device tasks (no copies) */
XKB_API int    xkrt_memory_register_async(xkrt_runtime_t * runtime, void * ptr, size_t size);
XKB_API int    xkrt_memory_unregister_async(xkrt_runtime_t * runtime, void * ptr, size_t size);
XKB_API void * xkrt_memory_unified_allocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, size_t size);
XKB_API void   xkrt_memory_unified_deallocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, void * ptr, size_t size);

/* drivers and devices (xkrt.h:128-135): the host is device 0, the GPU device 1; bodies receive
 * these device objects */
XKB_API xkrt_driver_t * xkrt_driver_get(xkrt_runtime_t * runtime, xkrt_driver_type_t type);
XKB_API xkrt_device_t * xkrt_device_get(xkrt_runtime_t * runtime, xkrt_device_global_id_t device);
XKB_API xkrt_driver_t * xkrt_device_driver_get(xkrt_runtime_t * runtime, xkrt_device_t * device);
XKB_API xkrt_device_driver_id_t xkrt_device_driver_id_get(xkrt_runtime_t * runtime, xkrt_device_t * device);
XKB_API unsigned int xkrt_get_ndevices(xkrt_runtime_t * runtime);
XKB_API unsigned int xkrt_get_ndevices_max(xkrt_runtime_t * runtime);

/* task completion (xkrt.h:138-144): a body may detach its task (incr) and complete it later
 * from any thread (decr back to 0, or complete); successors are released then, and no thread
 * waits for the detached task meanwhile. Tasks of this API
 * are committed and scheduled by the spawn calls and xkrt_task_wait: commit and enqueue record
 * XKB_EINVAL. */
XKB_API void xkrt_task_detachable_incr(xkrt_runtime_t * runtime, xkrt_task_t * task);
XKB_API void xkrt_task_detachable_decr(xkrt_runtime_t * runtime, xkrt_task_t * task);
XKB_API void xkrt_task_complete(xkrt_runtime_t * runtime, xkrt_task_t * task);
XKB_API void xkrt_task_commit(xkrt_runtime_t * runtime, xkrt_task_t * task);
XKB_API void xkrt_task_enqueue(xkrt_runtime_t * runtime, xkrt_task_t * task);
/* the task whose body runs on the calling thread (xkrt.h:156) */
XKB_API xkrt_task_t * xkrt_task_current(xkrt_runtime_t * runtime);

/* logger (xkrt.h:560-565): messages to stderr; fatal aborts, as in the reference */
XKB_API void xkrt_logger_info(const char * msg);
XKB_API void xkrt_logger_debug(const char * msg);
XKB_API void xkrt_logger_warn(const char * msg);
XKB_API void xkrt_logger_error(const char * msg);
XKB_API void xkrt_logger_fatal(const char * msg);

/* tasking (xkrt.h:138-163) */
XKB_API void xkrt_task_wait(xkrt_runtime_t * runtime);
XKB_API void * xkrt_task_args(xkrt_task_t * task);
XKB_API xkrt_access_t * xkrt_task_accesses(xkrt_task_t * task);
XKB_API xkrt_access_t * xkrt_task_access(xkrt_task_t * task, xkrt_task_access_counter_type_t access_id);
XKB_API void * xkrt_task_access_replica(xkrt_task_t * task, xkrt_task_access_counter_type_t access_id);

/* spawn (xkrt.h:160-196) */
XKB_API void xkrt_task_spawn_generic(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                     const xkrt_task_flag_bitfield_t flags, const xkrt_task_format_id_t fmtid,
                                     const void * args, const size_t args_size, const xkrt_access_t * accesses,
                                     const xkrt_task_access_counter_type_t naccesses,
                                     const xkrt_task_access_counter_type_t ocr_access,
                                     const xkrt_task_wait_counter_type_t detachable_counter_initial);
XKB_API void xkrt_task_spawn_with_format(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                         const xkrt_task_format_id_t fmtid, const void * args, const size_t args_size);
XKB_API void xkrt_task_spawn_with_format_with_accesses(xkrt_runtime_t * runtime, const xkrt_device_global_id_t device_global_id,
                                                       const xkrt_task_format_id_t fmtid, const void * args,
                                                       const size_t args_size, const xkrt_access_t * accesses,
                                                       const int naccesses);
XKB_API void xkrt_task_spawn(xkrt_runtime_t * runtime, xkrt_task_func_t func, void * user_data);

/* teams (xkrt.h:206-226): one host team */
XKB_API xkrt_team_t * xkrt_team_driver_device_get(xkrt_runtime_t * runtime, xkrt_driver_type_t type,
                                                  xkrt_device_driver_id_t device_driver_id);
XKB_API void xkrt_team_task_spawn(xkrt_runtime_t * runtime, xkrt_team_t * team, xkrt_task_func_t func, void * user_data);
XKB_API void xkrt_team_task_spawn_with_accesses(xkrt_runtime_t * runtime, xkrt_team_t * team, xkrt_task_func_t func,
                                                void * user_data, const xkrt_access_t * accesses, const int naccesses);

/* formats (xkrt.h:228-229) */
XKB_API xkrt_task_format_id_t xkrt_task_format_put(xkrt_runtime_t * runtime, const char * label);
XKB_API int xkrt_task_format_set(xkrt_runtime_t * runtime, xkrt_task_format_id_t fmtid, xkrt_task_format_target_t target,
                                 xkrt_task_format_func_t func);

/* device memory (xkrt.h:116-117): a plain device pointer (cudaMalloc) for the GPU, host memory
 * for device 0 -- the reference returns its allocator's chunk object instead */
XKB_API void * xkrt_memory_device_allocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, size_t size);
XKB_API void   xkrt_memory_device_deallocate(xkrt_runtime_t * runtime, xkrt_device_global_id_t device, void * chunk);

/* asynchronous file I/O (xkrt.h:114-115; src/file/readwrite.cc:104-170): spawns nchunks host
 * tasks, each with a virtual write (VW) segment access on its slice of the buffer, that read
 * (pread) or write (pwrite) that slice at the same offset of the file; they run at the next
 * xkrt_task_wait, and tasks that access the buffer after them wait for them. 0 or XKB_EINVAL. */
XKB_API int xkrt_file_read_async(xkrt_runtime_t * runtime, int fd, void * buffer, size_t n, unsigned int nchunks);
XKB_API int xkrt_file_write_async(xkrt_runtime_t * runtime, int fd, void * buffer, size_t n, unsigned int nchunks);

/* teams (xkrt.h:207-208) */
XKB_API xkrt_team_t * xkrt_team_driver_get(xkrt_runtime_t * runtime, xkrt_driver_type_t type);
XKB_API xkrt_team_t * xkrt_team_driver_get_any(xkrt_runtime_t * runtime, xkrt_driver_type_bitfield_t types);

/* ---- driver interface (xkrt.h:231-558; include/xkrt/driver/driver.h:62-232) ---------------- */
typedef enum xkrt_queue_type_t {
    XKRT_QUEUE_TYPE_H2D      = 0,
    XKRT_QUEUE_TYPE_D2H      = 1,
    XKRT_QUEUE_TYPE_D2D      = 2,
    XKRT_QUEUE_TYPE_KERN     = 3,
    XKRT_QUEUE_TYPE_FD_READ  = 4,
    XKRT_QUEUE_TYPE_FD_WRITE = 5,
    XKRT_QUEUE_TYPE_ALL
} xkrt_queue_type_t;

typedef enum xkrt_driver_module_format_t {
    XKRT_DRIVER_MODULE_FORMAT_SPIRV,
    XKRT_DRIVER_MODULE_FORMAT_NATIVE,
    XKRT_DRIVER_MODULE_FORMAT_UNKWN
} xkrt_driver_module_format_t;

typedef void * xkrt_driver_module_t;
typedef void * xkrt_driver_module_fn_t;

typedef struct xkrt_power_counter_t { uint64_t b1, b2, b3, b4; } xkrt_power_counter_t;
typedef struct xkrt_power_t {
    struct priv_t { uint64_t t1, t2; xkrt_power_counter_t c1, c2; } priv;
    double dt;   /* seconds between start and stop */
    double P;    /* mean power in W over that time (0 when the energy counter is unavailable) */
} xkrt_power_t;

/* A kernel launcher (include/xkrt/driver/kernel-launcher.h:44-51): called by
 * xkrt_task_kernel_launch with the queue the task's kernels go to and the command index to pass
 * on to xkrt_device_kernel_launch. */
typedef void (*xkrt_kernel_launcher_t)(void * runtime, void * device, void * task, void * queue, void * cmd,
                                       xkrt_queue_command_list_counter_t idx);

/* Inside a CUDA-target body: call launcher(runtime, device, task, queue, NULL, 0) with the queue of
 * the host thread running the body; the task completes once its kernels did (synchronous or
 * not). Outside a body: XKB_EINVAL (recorded). */
XKB_API void xkrt_task_kernel_launch(xkrt_runtime_t * runtime, xkrt_device_t * device, xkrt_task_t * task, int synchronous,
                                     xkrt_kernel_launcher_t launcher);
/* Launch fn (from xkrt_driver_module_get_fn) on the queue: args is the packed parameter buffer
 * of args_size bytes (the kernel's parameters at their natural alignment), as the reference's
 * CUDA driver passes it (src/driver/driver_cu.cc:1085-1131); records the queue's event idx when
 * the queue has one. 0 or an XKB_E* code. */
XKB_API int xkrt_device_kernel_launch(xkrt_runtime_t * runtime, xkrt_device_t * device, xkrt_queue_t * queue,
                                      xkrt_queue_command_list_counter_t idx, const xkrt_driver_module_fn_t * fn,
                                      const unsigned int gx, const unsigned int gy, const unsigned int gz,
                                      const unsigned int bx, const unsigned int by, const unsigned int bz,
                                      const unsigned int shared_memory_bytes, void * args, const size_t args_size);
XKB_API int xkrt_driver_kernel_launch(xkrt_driver_t * driver, xkrt_queue_t * queue, xkrt_queue_command_list_counter_t idx,
                                      const xkrt_driver_module_fn_t * fn, const unsigned int gx, const unsigned int gy,
                                      const unsigned int gz, const unsigned int bx, const unsigned int by,
                                      const unsigned int bz, const unsigned int shared_memory_bytes, void * args,
                                      const size_t args_size);

/* driver meta data and lifecycle: the runtime brings its drivers up in xkrt_init, so init returns
 * 0 and finalize does nothing */
XKB_API const char * xkrt_driver_get_name(xkrt_driver_t * driver);
XKB_API unsigned int xkrt_driver_get_ndevices_max(xkrt_driver_t * driver);
XKB_API int  xkrt_driver_init(xkrt_driver_t * driver, unsigned int ndevices, int use_p2p);
XKB_API void xkrt_driver_finalize(xkrt_driver_t * driver);

/* devices of a driver: the host driver has device 0, the CUDA driver the runtime's GPU as its
 * device 0; commit sets the device's own bit (global id) in affinity[0] */
XKB_API xkrt_device_t * xkrt_driver_device_create(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id);
XKB_API void xkrt_driver_device_init(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id);
XKB_API int  xkrt_driver_device_commit(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                       xkrt_device_global_id_bitfield_t * affinity);
XKB_API int  xkrt_driver_device_destroy(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id);
XKB_API void xkrt_driver_device_info(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, char * buffer,
                                     size_t size);

/* memory of a driver (area_idx is ignored: one area per device) */
XKB_API void * xkrt_driver_memory_device_allocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                  const size_t size, int area_idx);
XKB_API void   xkrt_driver_memory_device_deallocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                    void * ptr, const size_t size, int area_idx);
XKB_API void * xkrt_driver_memory_host_allocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                const size_t size);
XKB_API void   xkrt_driver_memory_host_deallocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                  void * mem, const size_t size);
XKB_API void * xkrt_driver_memory_unified_allocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                   const size_t size);
XKB_API void   xkrt_driver_memory_unified_deallocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                     void * mem, const size_t size);
XKB_API int xkrt_driver_memory_host_register(xkrt_driver_t * driver, void * mem, uint64_t size);
XKB_API int xkrt_driver_memory_host_unregister(xkrt_driver_t * driver, void * mem, uint64_t size);
XKB_API int xkrt_driver_memory_unified_advise_device(xkrt_driver_t * driver, const xkrt_device_driver_id_t device_global_id,
                                                     const void * addr, const size_t size);
XKB_API int xkrt_driver_memory_unified_advise_host(xkrt_driver_t * driver, const void * addr, const size_t size);
XKB_API int xkrt_driver_memory_unified_prefetch_device(xkrt_driver_t * driver, const xkrt_device_driver_id_t device_global_id,
                                                       const void * addr, const size_t size);
XKB_API int xkrt_driver_memory_unified_prefetch_host(xkrt_driver_t * driver, const void * addr, const size_t size);

/* transfers: synchronous ones complete before returning; asynchronous ones are ordered on the
 * queue (a host-driver queue copies synchronously) */
XKB_API int xkrt_driver_transfer_h2d(xkrt_driver_t * driver, void * dst, void * src, const size_t size);
XKB_API int xkrt_driver_transfer_d2h(xkrt_driver_t * driver, void * dst, void * src, const size_t size);
XKB_API int xkrt_driver_transfer_d2d(xkrt_driver_t * driver, void * dst, void * src, const size_t size);
XKB_API int xkrt_driver_transfer_h2d_async(xkrt_driver_t * driver, void * dst, void * src, const size_t size, xkrt_queue_t * queue);
XKB_API int xkrt_driver_transfer_d2h_async(xkrt_driver_t * driver, void * dst, void * src, const size_t size, xkrt_queue_t * queue);
XKB_API int xkrt_driver_transfer_d2d_async(xkrt_driver_t * driver, void * dst, void * src, const size_t size, xkrt_queue_t * queue);

/* queues: a CUDA queue is a non-blocking stream with `capacity` events, one per command index;
 * delete waits for the queue's work first */
XKB_API int xkrt_driver_queue_suggest(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, xkrt_queue_type_t qtype);
XKB_API xkrt_queue_t * xkrt_driver_queue_create(xkrt_driver_t * driver, xkrt_device_t * device, xkrt_queue_type_t qtype,
                                                xkrt_queue_command_list_counter_t capacity);
XKB_API void xkrt_driver_queue_delete(xkrt_driver_t * driver, xkrt_queue_t * queue);

/* modules: NATIVE images (cubin, fatbin or PTX for this GPU) loaded with the driver's module
 * loader; SPIR-V is refused (NULL) */
XKB_API xkrt_driver_module_t xkrt_driver_module_load(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                                     uint8_t * bin, size_t binsize, xkrt_driver_module_format_t format);
XKB_API void xkrt_driver_module_unload(xkrt_driver_t * driver, xkrt_driver_module_t module);
XKB_API xkrt_driver_module_fn_t xkrt_driver_module_get_fn(xkrt_driver_t * driver, xkrt_driver_module_t module, const char * name);

/* energy (driver.h power_start/stop): wall time between the two calls, and the GPU's mean power
 * from its energy counter (read through NVML when the library is present) */
XKB_API void xkrt_driver_power_start(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, xkrt_power_t * pwr);
XKB_API void xkrt_driver_power_stop(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, xkrt_power_t * pwr);

/* ---- additions of this library (no counterpart in the reference API) --------------------- */
/* A format whose device body is one of the library's built-in tile bodies (XKB_TASK_HEAT_F64,
 * XKB_TASK_HEAT_F32, XKB_TASK_AXPBY): the task's args are an xkb_task_desc_t whose grid / vector
 * pointers are HOST addresses inside registered regions; the runtime points them at the
 * device mirrors. Batches made only of such tasks run on the persistent scheduler. */
XKB_API xkrt_task_format_id_t xkb_task_format_builtin(xkrt_runtime_t * runtime, int kind);
/* First failure recorded since the last call (XKB_OK if none); clears it. */
XKB_API int xkb_runtime_status(xkrt_runtime_t * runtime);
/* The CUDA stream CUDA-target format bodies launch on (cudaStream_t as void *): inside a body,
 * the stream of the host thread running it (each thread of the team has its own). */
XKB_API void * xkb_runtime_stream(xkrt_runtime_t * runtime);
/* Counters of the last xkrt_task_wait: tasks run, unique edges, copies H2D / D2H, and whether the
 * persistent scheduler ran the batch (1) or the host team ran it as a dataflow graph (0). */
XKB_API int xkb_runtime_last_wait(xkrt_runtime_t * runtime, uint64_t * tasks, uint64_t * edges, uint64_t * h2d,
                                  uint64_t * d2h, int * fused);
/* Bytes the last xkrt_task_wait copied host -> device and device -> host. */
XKB_API int xkb_runtime_last_wait_bytes(xkrt_runtime_t * runtime, uint64_t * h2d_bytes, uint64_t * d2h_bytes);
/* Wall time of the phases of the last xkrt_task_wait, in ms: dependency resolution (records,
 * resolver batches, successor graph), coherency (planner fetches, H2D copies, descriptor upload;
 * fused batches only), execution, and the write-back of device-written blocks to the host. */
XKB_API int xkb_runtime_last_wait_times(xkrt_runtime_t * runtime, double * resolve_ms, double * coherency_ms, double * run_ms,
                                        double * writeback_ms);

#ifdef __cplusplus
}
#endif
#endif /* XKRT_B200_CAPI_H */
