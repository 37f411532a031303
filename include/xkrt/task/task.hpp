/* XKRT C++ source API: tasks and their layout (include/xkrt/task/task.hpp of the reference). */
#ifndef XKRT_B200_TASK_TASK_HPP
#define XKRT_B200_TASK_TASK_HPP
#include "../b200/api.hpp"
#endif
