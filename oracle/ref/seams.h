// Hooks behind the oracle's link-seam definitions (oracle/ref/seams.cc); test infrastructure only.
#ifndef XK_ORACLE_SEAMS_H
#define XK_ORACLE_SEAMS_H
#include <xkrt/runtime.h>

XKRT_NAMESPACE_BEGIN
typedef struct xk_seam_hooks_t {
    void (*copy2d)(runtime_t *, device_global_id_t, const memory_view_t &, device_global_id_t,
                   const memory_replica_view_t &, device_global_id_t, const memory_replica_view_t &,
                   const callback_t &);
    void (*copy1d)(runtime_t *, device_global_id_t, size_t, device_global_id_t, uintptr_t,
                   device_global_id_t, uintptr_t, const callback_t &);
    device_t * (*device_get)(runtime_t *, device_global_id_t);
    area_chunk_t * (*allocate)(runtime_t *, device_global_id_t, size_t);
    void (*deallocate)(runtime_t *, device_global_id_t, area_chunk_t *);
    void (*execute)(runtime_t *, device_t *, task_t *);
} xk_seam_hooks_t;
extern xk_seam_hooks_t xk_seam_hooks;
XKRT_NAMESPACE_END
#endif
