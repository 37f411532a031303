// Objects of the XKRT C API that the runtime (xkrt_capi.cc) and the driver interface
// (xkrt_driver.cc) both hand out as opaque pointers.
#pragma once

#include <cuda_runtime.h>

namespace xkb_capi {

// A device of the runtime: global id 0 is the host, 1 the GPU (include/xkrt/consts.h
// HOST_DEVICE_GLOBAL_ID = 0; drivers' devices follow it).
struct Device { int global_id; };

// A driver (XKRT_DRIVER_TYPE_HOST or _CUDA): the CUDA device it drives (-1 for the host) and its
// device 0.
struct Driver { int type; int ordinal; Device * device0; };

// A queue of commands (include/xkrt/driver/queue.h:137-229): for the CUDA driver a stream, and
// one event per command index, recorded when a kernel of that index is launched. A host queue
// has no stream (its transfers are synchronous).
struct Queue {
    int driver_type;
    int qtype;
    int ordinal;
    cudaStream_t stream;
    bool owned;                 // stream and events created by xkrt_driver_queue_create
    unsigned capacity;
    cudaEvent_t * events;
};

} // namespace xkb_capi
