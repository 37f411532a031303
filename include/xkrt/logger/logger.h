/* Logging macros of the XKRT C++ source API (include/xkrt/logger/logger.h of the reference):
 * messages to stderr, LOGGER_FATAL aborts. */
#ifndef XKRT_B200_LOGGER_H
#define XKRT_B200_LOGGER_H
#include <cstdio>
#include <cstdlib>
#define XKB_LOGGER_PRINT(level, ...) do { fprintf(stderr, "[xkrt] %s: ", level); fprintf(stderr, __VA_ARGS__); fputc('\n', stderr); } while (0)
#define LOGGER_INFO(...)  XKB_LOGGER_PRINT("info", __VA_ARGS__)
#define LOGGER_WARN(...)  XKB_LOGGER_PRINT("warn", __VA_ARGS__)
#define LOGGER_ERROR(...) XKB_LOGGER_PRINT("error", __VA_ARGS__)
#if XKRT_SUPPORT_DEBUG
#define LOGGER_DEBUG(...) XKB_LOGGER_PRINT("debug", __VA_ARGS__)
#else
#define LOGGER_DEBUG(...)
#endif
#define LOGGER_FATAL(...) do { XKB_LOGGER_PRINT("fatal", __VA_ARGS__); abort(); } while (0)
#endif
