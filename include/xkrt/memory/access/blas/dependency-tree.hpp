/* XKRT C++ source API: matrix accesses. The reference's dependency tree lives here; in this library dependencies are resolved on the GPU, so the header only brings the access types. */
#ifndef XKRT_B200_MEMORY_ACCESS_BLAS_DEPENDENCY_TREE_HPP
#define XKRT_B200_MEMORY_ACCESS_BLAS_DEPENDENCY_TREE_HPP
#include "../../../b200/api.hpp"
#endif
