// Error reporting and version for the libxkb200 C ABI.
#include "common.cuh"

#include <cstdarg>
#include <cstdio>

static thread_local char g_last_error[512] = "";

int xkb_set_error(int code, const char * fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

int xkb_set_cuda_error(cudaError_t e)
{
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver)
        return xkb_set_error(XKB_ENODEV, "CUDA: %s", cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation)
        return xkb_set_error(XKB_ENOMEM, "CUDA: %s", cudaGetErrorString(e));
    return xkb_set_error(XKB_ECUDA, "CUDA: %s", cudaGetErrorString(e));
}

extern "C" const char * xkb_last_error(void) { return g_last_error; }
extern "C" const char * xkb_version(void) { return "libxkb200 0.1 sm_100a"; }
