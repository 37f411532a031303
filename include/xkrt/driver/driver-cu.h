/* The CUDA queue a kernel launcher receives (include/xkrt/driver/driver-cu.h of the reference,
 * queue_cu_t): cu.handle.high is the stream to launch on, cu.events.buffer[idx] an event the
 * launcher may record after its kernels. */
#ifndef XKRT_B200_DRIVER_CU_H
#define XKRT_B200_DRIVER_CU_H
#include <cuda_runtime.h>
#include "../b200/api.hpp"

XKRT_NAMESPACE_BEGIN

typedef struct command_t command_t;

typedef struct queue_cu_t {
    int driver_type;                  /* XKRT_DRIVER_TYPE_CUDA */
    int qtype;                        /* XKRT_QUEUE_TYPE_KERN */
    struct {
        struct { cudaStream_t high, low; } handle;
        struct { cudaEvent_t * buffer; unsigned int capacity; } events;
    } cu;
} queue_cu_t;

XKRT_NAMESPACE_END
#endif
