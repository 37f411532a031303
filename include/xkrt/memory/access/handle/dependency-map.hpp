/* XKRT C++ source API: handle accesses. The reference's dependency map lives here; in this library handle dependencies are resolved by the runtime, so the header only brings the access types. */
#ifndef XKRT_B200_MEMORY_ACCESS_HANDLE_DEPENDENCY_MAP_HPP
#define XKRT_B200_MEMORY_ACCESS_HANDLE_DEPENDENCY_MAP_HPP
#include "../../../b200/api.hpp"
#endif
