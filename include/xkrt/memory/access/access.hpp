/* XKRT C++ source API: accesses (include/xkrt/memory/access/access.hpp of the reference). */
#ifndef XKRT_B200_MEMORY_ACCESS_ACCESS_HPP
#define XKRT_B200_MEMORY_ACCESS_ACCESS_HPP
#include "../../b200/api.hpp"
#endif
