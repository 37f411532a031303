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

int xkb_set_cuda_error_at(cudaError_t e, const char * file, int line)
{
    const char * base = file;
    for (const char * p = file; *p; ++p) if (*p == '/') base = p + 1;
    const int code = (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? XKB_ENODEV
                   : e == cudaErrorMemoryAllocation ? XKB_ENOMEM : XKB_ECUDA;
    return xkb_set_error(code, "CUDA: %s (%s:%d)", cudaGetErrorString(e), base, line);
}

extern "C" const char * xkb_last_error(void) { return g_last_error; }
extern "C" const char * xkb_version(void) { return "libxkb200 0.1 sm_100a"; }
