/* XKRT C++ source API: task formats (include/xkrt/task/format.h of the reference). */
#ifndef XKRT_B200_TASK_FORMAT_H
#define XKRT_B200_TASK_FORMAT_H
#include "../b200/api.hpp"
#endif
