// Link-seam definitions for the reference-backed oracle binaries (test infrastructure only).
//
// src/task/task.cc pulls in the reference's memory-coherency tree, which calls into the
// runtime (copies, device allocation, task execution). The oracle links the reference's
// trees WITHOUT the reference's runtime and drivers, so these out-of-line members are
// defined here. Each forwards to a hook the harness installs; a harness that never
// reaches them (the dependency oracle) leaves the hooks null and the call aborts.
#include <xkrt/runtime.h>

#include <cstdio>
#include <cstdlib>

#include "seams.h"

XKRT_NAMESPACE_BEGIN

xk_seam_hooks_t xk_seam_hooks = {};

static void seam_missing(const char * what)
{
    fprintf(stderr, "oracle seam `%s` reached without a hook\n", what);
    abort();
}

void runtime_t::copy(
    const device_global_id_t device_global_id,
    const memory_view_t & host_view,
    const device_global_id_t dst_device_global_id,
    const memory_replica_view_t & dst_device_view,
    const device_global_id_t src_device_global_id,
    const memory_replica_view_t & src_device_view,
    const callback_t & callback)
{
    if (!xk_seam_hooks.copy2d) seam_missing("runtime_t::copy(2d)");
    xk_seam_hooks.copy2d(this, device_global_id, host_view, dst_device_global_id, dst_device_view,
                                src_device_global_id, src_device_view, callback);
}

void runtime_t::copy(
    const device_global_id_t device_global_id,
    const size_t size,
    const device_global_id_t dst_device_global_id,
    const uintptr_t dst_device_addr,
    const device_global_id_t src_device_global_id,
    const uintptr_t src_device_addr,
    const callback_t & callback)
{
    if (!xk_seam_hooks.copy1d) seam_missing("runtime_t::copy(1d)");
    xk_seam_hooks.copy1d(this, device_global_id, size, dst_device_global_id, dst_device_addr,
                                src_device_global_id, src_device_addr, callback);
}

device_t * runtime_t::device_get(const device_global_id_t device_global_id)
{
    if (!xk_seam_hooks.device_get) seam_missing("runtime_t::device_get");
    return xk_seam_hooks.device_get(this, device_global_id);
}

area_chunk_t * runtime_t::memory_device_allocate(const device_global_id_t device_global_id, const size_t size)
{
    if (!xk_seam_hooks.allocate) seam_missing("runtime_t::memory_device_allocate");
    return xk_seam_hooks.allocate(this, device_global_id, size);
}

void runtime_t::memory_device_deallocate(const device_global_id_t device_global_id, area_chunk_t * chunk)
{
    if (!xk_seam_hooks.deallocate) seam_missing("runtime_t::memory_device_deallocate");
    xk_seam_hooks.deallocate(this, device_global_id, chunk);
}

int runtime_t::memory_unified_advise(const device_global_id_t, const void *, const size_t) { return 0; }
int runtime_t::memory_unified_prefetch(const device_global_id_t, const void *, const size_t) { return 0; }

void task_execute(runtime_t * runtime, device_t * device, task_t * task)
{
    if (!xk_seam_hooks.execute) seam_missing("task_execute");
    xk_seam_hooks.execute(runtime, device, task);
}

thread_t * thread_t::get_tls(void) { seam_missing("thread_t::get_tls"); return nullptr; }
task_t * thread_t::allocate_task(const size_t) { seam_missing("thread_t::allocate_task"); return nullptr; }

XKRT_NAMESPACE_END
