// The driver interface of the XKRT C API (api/c/include/xkrt/xkrt.h:231-558, the function table
// of include/xkrt/driver/driver.h:62-232) for the two drivers of this runtime: the host and the
// CUDA GPU. CUDA calls go through the CUDA runtime; module loading and packed-argument kernel
// launches use the driver's module loader and cuLaunchKernel (as src/driver/driver_cu.cc:953-1131
// does), reached through cudaGetDriverEntryPointByVersion so the library does not link libcuda.
#include "capi_objects.h"
#include "common.cuh"
#include "../../include/xkrt_capi.h"

#include <cuda.h>
#include <dlfcn.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

using xkb_capi::Device;
using xkb_capi::Driver;
using xkb_capi::Queue;

namespace {

Driver * DRV(xkrt_driver_t * d) { return (Driver *) d; }
bool is_cuda(const Driver * d) { return d && d->type == XKRT_DRIVER_TYPE_CUDA; }
bool is_host(const Driver * d) { return d && d->type == XKRT_DRIVER_TYPE_HOST; }

// Driver entry points used here, resolved once.
struct CuFns {
    CUresult (*module_load)(CUmodule *, const void *) = nullptr;
    CUresult (*module_unload)(CUmodule) = nullptr;
    CUresult (*module_get_function)(CUfunction *, CUmodule, const char *) = nullptr;
    CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream, void **,
                       void **) = nullptr;
    bool ok = false;
};

const CuFns & cu()
{
    static CuFns f;
    static std::once_flag once;
    std::call_once(once, [] {
        auto get = [](const char * name, void ** p) {
            cudaDriverEntryPointQueryResult q;
            return cudaGetDriverEntryPointByVersion(name, p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess && *p;
        };
        f.ok = get("cuModuleLoadData", (void **) &f.module_load) && get("cuModuleUnload", (void **) &f.module_unload) &&
               get("cuModuleGetFunction", (void **) &f.module_get_function) && get("cuLaunchKernel", (void **) &f.launch);
        if (!f.ok) cudaGetLastError();
    });
    return f;
}

int set_device(const Driver * d)
{
    if (cudaSetDevice(d->ordinal) != cudaSuccess) return xkb_set_cuda_error(cudaGetLastError());
    return XKB_OK;
}

int copy_sync(Driver * d, void * dst, const void * src, size_t size, cudaMemcpyKind kind)
{
    if (!d) return xkb_set_error(XKB_EINVAL, "transfer: no driver");
    if (is_host(d)) { memcpy(dst, src, size); return XKB_OK; }
    if (int rc = set_device(d)) return rc;
    XKB_CUDA_TRY(cudaMemcpy(dst, src, size, kind));
    return XKB_OK;
}

int copy_async(Driver * d, void * dst, const void * src, size_t size, xkrt_queue_t * queue, cudaMemcpyKind kind)
{
    Queue * q = (Queue *) queue;
    if (!d) return xkb_set_error(XKB_EINVAL, "transfer: no driver");
    if (is_host(d) || !q || !q->stream) return copy_sync(d, dst, src, size, kind);
    XKB_CUDA_TRY(cudaMemcpyAsync(dst, src, size, kind, q->stream));
    return XKB_OK;
}

// NVML's energy counter (read only), found at run time.
struct Nvml {
    int (*init)() = nullptr;
    int (*by_pci)(const char *, void **) = nullptr;
    int (*energy)(void *, unsigned long long *) = nullptr;
    bool ok = false;
};

const Nvml & nvml()
{
    static Nvml n;
    static std::once_flag once;
    std::call_once(once, [] {
        void * h = dlopen("libnvidia-ml.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!h) return;
        n.init = (int (*)()) dlsym(h, "nvmlInit_v2");
        n.by_pci = (int (*)(const char *, void **)) dlsym(h, "nvmlDeviceGetHandleByPciBusId_v2");
        n.energy = (int (*)(void *, unsigned long long *)) dlsym(h, "nvmlDeviceGetTotalEnergyConsumption");
        n.ok = n.init && n.by_pci && n.energy && n.init() == 0;
    });
    return n;
}

// Energy of the GPU in mJ since its driver loaded, or 0 when it cannot be read.
uint64_t energy_mj(const Driver * d)
{
    if (!is_cuda(d) || !nvml().ok) return 0;
    char bus[64];
    if (cudaDeviceGetPCIBusId(bus, sizeof(bus), d->ordinal) != cudaSuccess) { cudaGetLastError(); return 0; }
    void * dev = nullptr;
    unsigned long long e = 0;
    if (nvml().by_pci(bus, &dev) != 0 || nvml().energy(dev, &e) != 0) return 0;
    return (uint64_t) e;
}

uint64_t now_ns()
{
    return (uint64_t) std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

} // namespace

// ---- meta data and lifecycle ----------------------------------------------------------------

extern "C" const char * xkrt_driver_get_name(xkrt_driver_t * driver)
{
    Driver * d = DRV(driver);
    return is_cuda(d) ? "CUDA" : is_host(d) ? "HOST" : nullptr;
}

extern "C" unsigned int xkrt_driver_get_ndevices_max(xkrt_driver_t * driver)
{
    Driver * d = DRV(driver);
    if (is_host(d)) return 1;
    int n = 0;
    if (!is_cuda(d) || cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
    return (unsigned) n;
}

extern "C" int xkrt_driver_init(xkrt_driver_t * driver, unsigned int ndevices, int use_p2p)
{
    (void) ndevices; (void) use_p2p;
    return DRV(driver) ? XKB_OK : xkb_set_error(XKB_EINVAL, "xkrt_driver_init: no driver");
}

extern "C" void xkrt_driver_finalize(xkrt_driver_t * driver) { (void) driver; }

// ---- devices --------------------------------------------------------------------------------

extern "C" xkrt_device_t * xkrt_driver_device_create(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id)
{
    Driver * d = DRV(driver);
    if (!d || device_driver_id != 0) { xkb_set_error(XKB_EINVAL, "xkrt_driver_device_create: no device %d", (int) device_driver_id); return nullptr; }
    return (xkrt_device_t *) d->device0;
}

extern "C" void xkrt_driver_device_init(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id)
{
    (void) driver; (void) device_driver_id;
}

extern "C" int xkrt_driver_device_commit(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id,
                                         xkrt_device_global_id_bitfield_t * affinity)
{
    Driver * d = DRV(driver);
    if (!d || device_driver_id != 0 || !affinity) return xkb_set_error(XKB_EINVAL, "xkrt_driver_device_commit: bad arguments");
    affinity[0] |= (xkrt_device_global_id_bitfield_t) (1u << d->device0->global_id);
    return XKB_OK;
}

extern "C" int xkrt_driver_device_destroy(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id)
{
    (void) driver; (void) device_driver_id;
    return XKB_OK;
}

// "<name>, cu device: <global id>, pci: <bus>:<device>, <memory> (GB)" as the reference's CUDA
// driver prints it (src/driver/driver_cu.cc:935-950).
extern "C" void xkrt_driver_device_info(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, char * buffer, size_t size)
{
    Driver * d = DRV(driver);
    if (!buffer || !size) return;
    buffer[0] = 0;
    if (is_host(d)) { snprintf(buffer, size, "host, device: 0"); return; }
    cudaDeviceProp p;
    if (!is_cuda(d) || device_driver_id != 0 || cudaGetDeviceProperties(&p, d->ordinal) != cudaSuccess) { cudaGetLastError(); return; }
    snprintf(buffer, size, "%s, cu device: %i, pci: %02x:%02x, %.2f (GB)", p.name, d->device0->global_id, p.pciBusID, p.pciDeviceID,
             (double) p.totalGlobalMem / 1e9);
}

// ---- memory ---------------------------------------------------------------------------------

extern "C" void * xkrt_driver_memory_device_allocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, const size_t size,
                                                     int area_idx)
{
    (void) area_idx;
    Driver * d = DRV(driver);
    if (!d || device_driver_id != 0) { xkb_set_error(XKB_EINVAL, "memory_device_allocate: no device %d", (int) device_driver_id); return nullptr; }
    if (is_host(d)) return malloc(size);
    void * p = nullptr;
    if (set_device(d) || cudaMalloc(&p, size) != cudaSuccess) { xkb_set_cuda_error(cudaGetLastError()); return nullptr; }
    return p;
}

extern "C" void xkrt_driver_memory_device_deallocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, void * ptr,
                                                     const size_t size, int area_idx)
{
    (void) device_driver_id; (void) size; (void) area_idx;
    Driver * d = DRV(driver);
    if (is_host(d)) free(ptr);
    else if (is_cuda(d) && ptr && cudaFree(ptr) != cudaSuccess) xkb_set_cuda_error(cudaGetLastError());
}

extern "C" void * xkrt_driver_memory_host_allocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, const size_t size)
{
    (void) device_driver_id;
    Driver * d = DRV(driver);
    if (is_host(d)) return malloc(size);
    void * p = nullptr;
    if (!is_cuda(d) || set_device(d) || cudaHostAlloc(&p, size, cudaHostAllocPortable) != cudaSuccess)
    { xkb_set_error(XKB_ENOMEM, "memory_host_allocate: %zu bytes", (size_t) size); cudaGetLastError(); return nullptr; }
    return p;
}

extern "C" void xkrt_driver_memory_host_deallocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, void * mem,
                                                   const size_t size)
{
    (void) device_driver_id; (void) size;
    Driver * d = DRV(driver);
    if (is_host(d)) free(mem);
    else if (is_cuda(d) && mem && cudaFreeHost(mem) != cudaSuccess) xkb_set_cuda_error(cudaGetLastError());
}

extern "C" void * xkrt_driver_memory_unified_allocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, const size_t size)
{
    (void) device_driver_id;
    Driver * d = DRV(driver);
    if (is_host(d)) return malloc(size);
    void * p = nullptr;
    if (!is_cuda(d) || set_device(d) || cudaMallocManaged(&p, size) != cudaSuccess)
    { xkb_set_error(XKB_ENOMEM, "memory_unified_allocate: %zu bytes", (size_t) size); cudaGetLastError(); return nullptr; }
    return p;
}

extern "C" void xkrt_driver_memory_unified_deallocate(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, void * mem,
                                                      const size_t size)
{
    (void) device_driver_id; (void) size;
    Driver * d = DRV(driver);
    if (is_host(d)) free(mem);
    else if (is_cuda(d) && mem && cudaFree(mem) != cudaSuccess) xkb_set_cuda_error(cudaGetLastError());
}

extern "C" int xkrt_driver_memory_host_register(xkrt_driver_t * driver, void * mem, uint64_t size)
{
    Driver * d = DRV(driver);
    if (is_host(d)) return XKB_OK;
    if (!is_cuda(d)) return xkb_set_error(XKB_EINVAL, "memory_host_register: no driver");
    if (int rc = set_device(d)) return rc;
    XKB_CUDA_TRY(cudaHostRegister(mem, size, cudaHostRegisterPortable));
    return XKB_OK;
}

extern "C" int xkrt_driver_memory_host_unregister(xkrt_driver_t * driver, void * mem, uint64_t size)
{
    (void) size;
    Driver * d = DRV(driver);
    if (is_host(d)) return XKB_OK;
    if (!is_cuda(d)) return xkb_set_error(XKB_EINVAL, "memory_host_unregister: no driver");
    XKB_CUDA_TRY(cudaHostUnregister(mem));
    return XKB_OK;
}

// Preferred location of a unified range: the GPU or the host (src/driver/driver_cu.cc:1137-1165).
static int advise(Driver * d, cudaMemLocation loc, const void * addr, size_t size)
{
    if (is_host(d)) return XKB_OK;
    if (!is_cuda(d)) return xkb_set_error(XKB_EINVAL, "memory_unified_advise: no driver");
    XKB_CUDA_TRY(cudaMemAdvise_v2(addr, size, cudaMemAdviseSetPreferredLocation, loc));
    return XKB_OK;
}

extern "C" int xkrt_driver_memory_unified_advise_device(xkrt_driver_t * driver, const xkrt_device_driver_id_t device_global_id,
                                                        const void * addr, const size_t size)
{
    (void) device_global_id;
    Driver * d = DRV(driver);
    cudaMemLocation loc;
    loc.type = cudaMemLocationTypeDevice; loc.id = d ? d->ordinal : 0;
    return advise(d, loc, addr, size);
}

extern "C" int xkrt_driver_memory_unified_advise_host(xkrt_driver_t * driver, const void * addr, const size_t size)
{
    cudaMemLocation loc;
    loc.type = cudaMemLocationTypeHost; loc.id = 0;
    return advise(DRV(driver), loc, addr, size);
}

static int prefetch(Driver * d, cudaMemLocation loc, const void * addr, size_t size)
{
    if (is_host(d)) return XKB_OK;
    if (!is_cuda(d)) return xkb_set_error(XKB_EINVAL, "memory_unified_prefetch: no driver");
    if (int rc = set_device(d)) return rc;
    XKB_CUDA_TRY(cudaMemPrefetchAsync_v2(addr, size, loc, 0, 0));
    XKB_CUDA_TRY(cudaStreamSynchronize(0));
    return XKB_OK;
}

extern "C" int xkrt_driver_memory_unified_prefetch_device(xkrt_driver_t * driver, const xkrt_device_driver_id_t device_global_id,
                                                          const void * addr, const size_t size)
{
    (void) device_global_id;
    Driver * d = DRV(driver);
    cudaMemLocation loc;
    loc.type = cudaMemLocationTypeDevice; loc.id = d ? d->ordinal : 0;
    return prefetch(d, loc, addr, size);
}

extern "C" int xkrt_driver_memory_unified_prefetch_host(xkrt_driver_t * driver, const void * addr, const size_t size)
{
    cudaMemLocation loc;
    loc.type = cudaMemLocationTypeHost; loc.id = 0;
    return prefetch(DRV(driver), loc, addr, size);
}

// ---- transfers ------------------------------------------------------------------------------

extern "C" int xkrt_driver_transfer_h2d(xkrt_driver_t * driver, void * dst, void * src, const size_t size)
{ return copy_sync(DRV(driver), dst, src, size, cudaMemcpyHostToDevice); }
extern "C" int xkrt_driver_transfer_d2h(xkrt_driver_t * driver, void * dst, void * src, const size_t size)
{ return copy_sync(DRV(driver), dst, src, size, cudaMemcpyDeviceToHost); }
extern "C" int xkrt_driver_transfer_d2d(xkrt_driver_t * driver, void * dst, void * src, const size_t size)
{ return copy_sync(DRV(driver), dst, src, size, cudaMemcpyDeviceToDevice); }
extern "C" int xkrt_driver_transfer_h2d_async(xkrt_driver_t * driver, void * dst, void * src, const size_t size, xkrt_queue_t * queue)
{ return copy_async(DRV(driver), dst, src, size, queue, cudaMemcpyHostToDevice); }
extern "C" int xkrt_driver_transfer_d2h_async(xkrt_driver_t * driver, void * dst, void * src, const size_t size, xkrt_queue_t * queue)
{ return copy_async(DRV(driver), dst, src, size, queue, cudaMemcpyDeviceToHost); }
extern "C" int xkrt_driver_transfer_d2d_async(xkrt_driver_t * driver, void * dst, void * src, const size_t size, xkrt_queue_t * queue)
{ return copy_async(DRV(driver), dst, src, size, queue, cudaMemcpyDeviceToDevice); }

// ---- queues ---------------------------------------------------------------------------------

// Queues per device and type the reference's CUDA driver suggests (src/driver/driver_cu.cc:601-614).
extern "C" int xkrt_driver_queue_suggest(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, xkrt_queue_type_t qtype)
{
    (void) device_driver_id;
    Driver * d = DRV(driver);
    if (is_host(d)) return 1;
    return qtype == XKRT_QUEUE_TYPE_KERN ? 8 : 4;
}

extern "C" xkrt_queue_t * xkrt_driver_queue_create(xkrt_driver_t * driver, xkrt_device_t * device, xkrt_queue_type_t qtype,
                                                   xkrt_queue_command_list_counter_t capacity)
{
    (void) device;
    Driver * d = DRV(driver);
    if (!d) { xkb_set_error(XKB_EINVAL, "queue_create: no driver"); return nullptr; }
    Queue * q = new Queue{d->type, (int) qtype, d->ordinal, nullptr, true, 0, nullptr};
    if (is_cuda(d))
    {
        if (set_device(d) || cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking) != cudaSuccess)
        { xkb_set_cuda_error(cudaGetLastError()); delete q; return nullptr; }
        q->events = capacity ? new cudaEvent_t[capacity]() : nullptr;
        for (unsigned i = 0; i < capacity; ++i, ++q->capacity)
            if (cudaEventCreateWithFlags(&q->events[i], cudaEventDisableTiming) != cudaSuccess)
            {
                xkb_set_cuda_error(cudaGetLastError());
                xkrt_driver_queue_delete(driver, (xkrt_queue_t *) q);
                return nullptr;
            }
    }
    return (xkrt_queue_t *) q;
}

extern "C" void xkrt_driver_queue_delete(xkrt_driver_t * driver, xkrt_queue_t * queue)
{
    (void) driver;
    Queue * q = (Queue *) queue;
    if (!q || !q->owned) return;
    if (q->stream) cudaStreamSynchronize(q->stream);
    for (unsigned i = 0; i < q->capacity; ++i) cudaEventDestroy(q->events[i]);
    delete[] q->events;
    if (q->stream) cudaStreamDestroy(q->stream);
    delete q;
}

// ---- modules and kernel launches ------------------------------------------------------------

extern "C" xkrt_driver_module_t xkrt_driver_module_load(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, uint8_t * bin,
                                                        size_t binsize, xkrt_driver_module_format_t format)
{
    (void) binsize;
    Driver * d = DRV(driver);
    if (!is_cuda(d) || device_driver_id != 0 || format != XKRT_DRIVER_MODULE_FORMAT_NATIVE || !bin)
    { xkb_set_error(XKB_EINVAL, "module_load: a NATIVE image for the CUDA driver's device 0 is expected"); return nullptr; }
    if (!cu().ok) { xkb_set_error(XKB_ENODEV, "module_load: the CUDA driver's module loader is unavailable"); return nullptr; }
    CUmodule m = nullptr;
    if (set_device(d) || cudaFree(nullptr) != cudaSuccess) { xkb_set_cuda_error(cudaGetLastError()); return nullptr; }  // context current
    const CUresult r = cu().module_load(&m, bin);
    if (r != CUDA_SUCCESS) { xkb_set_error(XKB_ECUDA, "module_load: driver error %d", (int) r); return nullptr; }
    return (xkrt_driver_module_t) m;
}

extern "C" void xkrt_driver_module_unload(xkrt_driver_t * driver, xkrt_driver_module_t module)
{
    (void) driver;
    if (module && cu().ok) cu().module_unload((CUmodule) module);
}

extern "C" xkrt_driver_module_fn_t xkrt_driver_module_get_fn(xkrt_driver_t * driver, xkrt_driver_module_t module, const char * name)
{
    (void) driver;
    CUfunction f = nullptr;
    if (!module || !name || !cu().ok) { xkb_set_error(XKB_EINVAL, "module_get_fn: no module"); return nullptr; }
    const CUresult r = cu().module_get_function(&f, (CUmodule) module, name);
    if (r != CUDA_SUCCESS) { xkb_set_error(XKB_EINVAL, "module_get_fn: no function %s (driver error %d)", name, (int) r); return nullptr; }
    return (xkrt_driver_module_fn_t) f;
}

// fn is the function handle itself, passed as a pointer as in the reference
// (src/driver/driver_cu.cc:1113-1124: `(CUfunction) fn`).
extern "C" int xkrt_driver_kernel_launch(xkrt_driver_t * driver, xkrt_queue_t * queue, xkrt_queue_command_list_counter_t idx,
                                         const xkrt_driver_module_fn_t * fn, const unsigned int gx, const unsigned int gy,
                                         const unsigned int gz, const unsigned int bx, const unsigned int by, const unsigned int bz,
                                         const unsigned int shared_memory_bytes, void * args, const size_t args_size)
{
    Driver * d = DRV(driver);
    Queue * q = (Queue *) queue;
    if (!is_cuda(d) || !q || !q->stream || !fn) return xkb_set_error(XKB_EINVAL, "kernel_launch: a CUDA queue and a function are expected");
    if (!cu().ok) return xkb_set_error(XKB_ENODEV, "kernel_launch: cuLaunchKernel is unavailable");
    size_t sz = args_size;
    void * conf[] = {CU_LAUNCH_PARAM_BUFFER_POINTER, args, CU_LAUNCH_PARAM_BUFFER_SIZE, &sz, CU_LAUNCH_PARAM_END};
    const CUresult r = cu().launch((CUfunction) fn, gx, gy, gz, bx, by, bz, shared_memory_bytes, (CUstream) q->stream, nullptr,
                                   args_size ? conf : nullptr);
    if (r != CUDA_SUCCESS) return xkb_set_error(XKB_ECUDA, "kernel_launch: driver error %d", (int) r);
    if (idx < q->capacity) XKB_CUDA_TRY(cudaEventRecord(q->events[idx], q->stream));
    return XKB_OK;
}

// ---- energy ---------------------------------------------------------------------------------

extern "C" void xkrt_driver_power_start(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, xkrt_power_t * pwr)
{
    (void) device_driver_id;
    if (!pwr) return;
    memset(pwr, 0, sizeof(*pwr));
    pwr->priv.c1.b1 = energy_mj(DRV(driver));
    pwr->priv.t1 = now_ns();
}

extern "C" void xkrt_driver_power_stop(xkrt_driver_t * driver, xkrt_device_driver_id_t device_driver_id, xkrt_power_t * pwr)
{
    (void) device_driver_id;
    if (!pwr) return;
    pwr->priv.t2 = now_ns();
    pwr->priv.c2.b1 = energy_mj(DRV(driver));
    pwr->dt = (double) (pwr->priv.t2 - pwr->priv.t1) * 1e-9;
    pwr->P = (pwr->priv.c1.b1 && pwr->priv.c2.b1 >= pwr->priv.c1.b1 && pwr->dt > 0)
           ? (double) (pwr->priv.c2.b1 - pwr->priv.c1.b1) * 1e-3 / pwr->dt : 0.0;
}
