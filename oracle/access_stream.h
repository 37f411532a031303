/* Access-stream file format shared by the oracle programs (test infrastructure only).
 *
 * A stream is the sequence of accesses that tasks declare, in spawn order, each task's
 * accesses in declaration order -- the order in which the reference's spawning thread
 * hands them to task_dependency_resolve() (src/task/task.cc:285-299).
 *
 * File: 16-byte header { uint64 magic = XK_STREAM_MAGIC, uint64 count } then `count`
 * 64-byte little-endian records. Task ids are dense and non-decreasing from 0.
 *
 *   matrix access  (ACCESS_TYPE_BLAS_MATRIX = 2): addr = storage base, ld (elements),
 *                  offset_m/offset_n (elements/columns), m x n tile, sizeof_type --
 *                  the arguments of access_t's matrix constructor (access.hpp:539-574).
 *   segment access (ACCESS_TYPE_SEGMENT = 1): byte interval [addr, ld) -- the two
 *                  addresses of access_t's segment constructor (access.hpp:479-514).
 *   handle access  (ACCESS_TYPE_HANDLE = 0): addr = the handle (access_t's handle constructor).
 *   mode: xkrt_access_mode_t bits (R=1, W=2, V=4, D=8; include/xkrt/memory/access/mode.h:54-66).
 */
#ifndef XK_ORACLE_ACCESS_STREAM_H
#define XK_ORACLE_ACCESS_STREAM_H

#include <stdint.h>
#include <stdio.h>

#define XK_STREAM_MAGIC   0x314d525453424b58ull   /* "XKBSTRM1" */
#define XK_STREAM_HANDLE  0
#define XK_STREAM_SEGMENT 1
#define XK_STREAM_MATRIX  2

typedef struct xk_stream_rec_t {
    uint32_t task;
    uint8_t  type;
    uint8_t  mode;
    uint16_t reserved;
    uint64_t addr;
    uint64_t ld;
    uint64_t offset_m;
    uint64_t offset_n;
    uint64_t m;
    uint64_t n;
    uint64_t sizeof_type;
} xk_stream_rec_t;

#ifdef __cplusplus
#include <vector>
static inline int xk_stream_read(const char * path, std::vector<xk_stream_rec_t> & out)
{
    static_assert(sizeof(xk_stream_rec_t) == 64, "stream record must be 64 bytes");
    FILE * f = fopen(path, "rb");
    if (!f) return -1;
    uint64_t hdr[2];
    if (fread(hdr, 8, 2, f) != 2 || hdr[0] != XK_STREAM_MAGIC) { fclose(f); return -1; }
    out.resize(hdr[1]);
    if (hdr[1] && fread(out.data(), sizeof(xk_stream_rec_t), hdr[1], f) != hdr[1]) { fclose(f); return -1; }
    fclose(f);
    return 0;
}
#endif

#endif
