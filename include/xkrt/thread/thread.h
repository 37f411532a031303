/* XKRT C++ source API: threads: task memory, resolve, commit (include/xkrt/thread/thread.h of the reference). */
#ifndef XKRT_B200_THREAD_THREAD_H
#define XKRT_B200_THREAD_THREAD_H
#include "../b200/api.hpp"
#endif
