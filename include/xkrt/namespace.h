/* Namespace of the XKRT C++ source API (include/xkrt/namespace.h of the reference). */
#ifndef XKRT_B200_NAMESPACE_H
#define XKRT_B200_NAMESPACE_H
#define XKRT_NAMESPACE         xkrt
#define XKRT_NAMESPACE_BEGIN   namespace XKRT_NAMESPACE {
#define XKRT_NAMESPACE_END     }
#define XKRT_NAMESPACE_USE     using namespace XKRT_NAMESPACE
#endif
