/* Monotonic clock in nanoseconds (include/xkrt/logger/metric.h of the reference). */
#ifndef XKRT_B200_METRIC_H
#define XKRT_B200_METRIC_H
#include <stdint.h>
#include <time.h>
static inline uint64_t get_nanotime(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (uint64_t) ts.tv_sec * 1000000000ull + (uint64_t) ts.tv_nsec;
}
#endif
