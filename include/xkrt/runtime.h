/* XKRT C++ source API: the runtime (include/xkrt/runtime.h of the reference). */
#ifndef XKRT_B200_RUNTIME_H
#define XKRT_B200_RUNTIME_H
#include "b200/api.hpp"
#endif
