/* XKRT C++ source API: half-open intervals (include/xkrt/memory/access/common/interval.hpp of the reference). */
#ifndef XKRT_B200_MEMORY_ACCESS_COMMON_INTERVAL_HPP
#define XKRT_B200_MEMORY_ACCESS_COMMON_INTERVAL_HPP
#include "../../../b200/api.hpp"
#endif
