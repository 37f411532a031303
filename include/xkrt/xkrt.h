/* The XKRT C API under the reference's include path (api/c/include/xkrt/xkrt.h): a C program
 * that includes <xkrt/xkrt.h> compiles against this library with -I<repo>/include. */
#ifndef XKRT_B200_XKRT_H
#define XKRT_B200_XKRT_H
#include "../xkrt_capi.h"
#endif
