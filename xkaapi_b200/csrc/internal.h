// Library-internal entry points shared between translation units (not exported).
#pragma once
#include <cuda_runtime.h>

#include "../../include/xkrt_b200.h"

// Launch one task descriptor as its own kernel (the plain per-task form) on `stream`.
int xkb_internal_launch_task(const xkb_task_desc_t * d, cudaStream_t stream);

// Set a scheduler's descriptors on the device only (persistent forms only; no host copy).
// checked: the caller validated every descriptor with xkb_internal_task_valid.
int xkb_internal_sched_set_tasks_device(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks, bool checked);

// The descriptor checks of xkb_sched_set_tasks: a known kind with a well-formed tile or range.
static inline bool xkb_internal_task_valid(const xkb_task_desc_t & d)
{
    if (d.kind == XKB_TASK_HEAT_F64 || d.kind == XKB_TASK_HEAT_F32)
    {
        const auto & h = d.u.heat;
        return h.src && h.dst && h.src != h.dst && h.ld >= h.nx && h.nx >= 0 && h.ny >= 0 && h.x0 <= h.x1 && h.y0 <= h.y1;
    }
    if (d.kind == XKB_TASK_AXPBY)
    {
        const auto & a = d.u.axpby;
        return a.lo >= 0 && a.lo <= a.hi && (a.hi == a.lo || (a.x && a.y));
    }
    return d.kind == XKB_TASK_NOOP;
}

// Reset a resolver to no tasks, keeping its device buffers for the next graph.
int xkb_internal_resolver_reset(xkb_resolver_t * R);
