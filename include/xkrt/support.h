/* Build options a program may test (include/xkrt/support.h.in of the reference): this library
 * drives the host and one CUDA GPU, with no debug build fields. */
#ifndef XKRT_B200_SUPPORT_H
#define XKRT_B200_SUPPORT_H
#define XKRT_SUPPORT_CUDA              1
#define XKRT_SUPPORT_HIP               0
#define XKRT_SUPPORT_ZE                0
#define XKRT_SUPPORT_ZE_SYCL_INTEROP   0
#define XKRT_SUPPORT_SYCL              0
#define XKRT_SUPPORT_CL                0
#define XKRT_SUPPORT_STATS             0
#define XKRT_SUPPORT_CAIRO             0
#define XKRT_SUPPORT_NVML              0
#define XKRT_SUPPORT_ZES               0
#define XKRT_SUPPORT_RSMI              0
#define XKRT_SUPPORT_JULIA             0
#define XKRT_SUPPORT_DEBUG             0
#define XKRT_MEMORY_REGISTER_OVERFLOW_PROTECTION 0
#define XKRT_MEMORY_REGISTER_PAGE      0
#define XKRT_MEMORY_REGISTER_ASSISTED  0
#endif
