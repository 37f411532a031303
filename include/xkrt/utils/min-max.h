/* MIN / MAX of the XKRT C++ source API (include/xkrt/utils/min-max.h of the reference). */
#ifndef XKRT_B200_MIN_MAX_H
#define XKRT_B200_MIN_MAX_H
#ifndef MIN
#define MIN(X, Y) ((Y) < (X) ? (Y) : (X))
#endif
#ifndef MAX
#define MAX(X, Y) ((X) < (Y) ? (Y) : (X))
#endif
#endif
