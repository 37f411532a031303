// Library entry for concurrent-mode handle accesses: expands an access stream into the form the
// resolver takes (extra writer tasks inserted, CNC-W resolved as reads; handles.h states the rule
// and the reference code it follows).
#include "common.cuh"
#include "handles.h"

#include <cstring>
#include <new>
#include <vector>

struct xkb_handle_map {
    xkb_handles::Map map;
    uint64_t inserted = 0;                  // extra tasks inserted so far (shifts the task ids)
    std::vector<xkb_handles::Access> acc;
    std::vector<uint64_t> extra;
};

extern "C" int xkb_handle_map_create(xkb_handle_map_t ** map)
{
    if (!map) return xkb_set_error(XKB_EINVAL, "xkb_handle_map_create: null output");
    *map = new (std::nothrow) xkb_handle_map();
    return *map ? XKB_OK : xkb_set_error(XKB_ENOMEM, "xkb_handle_map_create: out of memory");
}

extern "C" int xkb_handle_map_destroy(xkb_handle_map_t * map)
{
    delete map;
    return XKB_OK;
}

extern "C" int xkb_handle_map_expand(xkb_handle_map_t * M, const xkb_access_rec_t * in, size_t n, xkb_access_rec_t * out,
                                     size_t cap, size_t * nout)
{
    if (!M || (n && (!in || !out)) || !nout) return xkb_set_error(XKB_EINVAL, "xkb_handle_map_expand: null argument");
    *nout = 0;
    size_t k = 0;
    for (size_t i = 0; i < n;)
    {
        size_t j = i;
        while (j < n && in[j].task == in[i].task) ++j;
        M->acc.clear(); M->extra.clear();
        for (size_t a = i; a < j; ++a)
        {
            const int conc = in[a].reserved >> 8;
            if (in[a].type == XKB_ACCESS_TYPE_HANDLE) M->acc.push_back({in[a].addr, in[a].mode, conc});
            else if (conc == xkb_handles::CONCURRENT)
                return xkb_set_error(XKB_EINVAL, "access %zu: concurrent mode applies to handle accesses only", a);
        }
        if (k + (j - i) + M->acc.size() > cap)
            return xkb_set_error(XKB_ERANGE, "xkb_handle_map_expand: output capacity %zu is too small", cap);
        const char * why = "";
        if (!M->acc.empty() && M->map.task(M->acc.data(), M->acc.size(), true, M->extra, &why))
            return xkb_set_error(XKB_EINVAL, "task %u: %s", in[i].task, why);
        for (uint64_t h : M->extra)
        {
            xkb_access_rec_t & e = out[k++];
            memset(&e, 0, sizeof(e));
            e.task = (uint32_t) (in[i].task + M->inserted++);
            e.type = XKB_ACCESS_TYPE_HANDLE; e.mode = xkb_handles::MODE_VW; e.addr = h;
        }
        for (size_t a = i; a < j; ++a)
        {
            xkb_access_rec_t & r = out[k++];
            r = in[a];
            r.task = (uint32_t) (in[a].task + M->inserted);
            if (r.type == XKB_ACCESS_TYPE_HANDLE) r.mode = xkb_handles::resolve_mode(r.mode, r.reserved >> 8);
            r.reserved &= 0xff;
        }
        i = j;
    }
    *nout = k;
    return XKB_OK;
}
