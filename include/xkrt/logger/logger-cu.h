/* CUDA driver-call check of the XKRT C++ source API (include/xkrt/logger/logger-cu.h of the
 * reference): a failed call is fatal. */
#ifndef XKRT_B200_LOGGER_CU_H
#define XKRT_B200_LOGGER_CU_H
#include <cuda.h>
#include "logger.h"
#define CU_SAFE_CALL(X)                                                                  \
    do {                                                                                 \
        CUresult xkb_r_ = (X);                                                           \
        if (xkb_r_ != CUDA_SUCCESS)                                                      \
        {                                                                                \
            const char * xkb_s_ = "?";                                                   \
            cuGetErrorString(xkb_r_, &xkb_s_);                                           \
            LOGGER_FATAL("`%s` failed with `%s` (%d)", #X, xkb_s_, (int) xkb_r_);        \
        }                                                                                \
    } while (0)
#endif
