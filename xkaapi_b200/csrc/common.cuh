// Shared definitions for the sm_100a kernels of libxkb200.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/xkrt_b200.h"

#define XKB_CUDA_TRY(expr)                                  \
    do {                                                    \
        cudaError_t _e = (expr);                            \
        if (_e != cudaSuccess) return xkb_set_cuda_error(_e); \
    } while (0)

// Records the CUDA error string and the source line that met it for xkb_last_error() and returns
// XKB_ECUDA (XKB_ENODEV / XKB_ENOMEM for a missing device / device memory).
int xkb_set_cuda_error_at(cudaError_t e, const char * file, int line);
#define xkb_set_cuda_error(e) xkb_set_cuda_error_at((e), __FILE__, __LINE__)
int xkb_set_error(int code, const char * fmt, ...);

static inline cudaStream_t xkb_stream(void * s) { return (cudaStream_t) s; }

__device__ __forceinline__ uint64_t xkb_globaltimer()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ int xkb_ld_acquire(const int * p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void xkb_st_release(int * p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" :: "l"(p), "r"(v) : "memory");
}
