// Library-internal entry points shared between translation units (not exported).
#pragma once
#include <cuda_runtime.h>

#include "../../include/xkrt_b200.h"

// Launch one task descriptor as its own kernel (the plain per-task form) on `stream`.
int xkb_internal_launch_task(const xkb_task_desc_t * d, cudaStream_t stream);

// Set a scheduler's descriptors on the device only (persistent forms only; no host copy).
int xkb_internal_sched_set_tasks_device(xkb_sched_t * S, const xkb_task_desc_t * tasks, size_t ntasks);

// Reset a resolver to no tasks, keeping its device buffers for the next graph.
int xkb_internal_resolver_reset(xkb_resolver_t * R);
