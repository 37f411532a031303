// The C API's handle-map decisions (xkaapi_b200/csrc/handles.h) in the two forms it takes with an
// order at least as strict as the reference's (exact = false), and their refusal with exact = true.
#include "../../xkaapi_b200/csrc/handles.h"

#include <cstdio>

using xkb_handles::Access;
using xkb_handles::Map;

static int fails = 0;
#define CHECK(c) do { if (!(c)) { std::fprintf(stderr, "line %d: %s\n", __LINE__, #c); ++fails; } } while (0)

int main()
{
    const uint64_t h = 0x5000, g = 0x6000;
    const char * why = "";
    std::vector<uint64_t> extra;
    {
        // a task listing h twice, the second access needing an extra writer (reads pending)
        Map m;
        Access r{h, 1, 1}, w{h, 2, 4};
        CHECK(m.task(&r, 1, true, extra, &why) == 0 && extra.empty());
        Access t[2] = {{h, 1, 1}, {h, 2, 4}};
        CHECK(m.task(t, 2, true, extra, &why) == -22 && extra.empty());
        CHECK(m.task(t, 2, false, extra, &why) == 0 && extra.size() == 1 && extra[0] == h);
        // after it: a CNC-W (t[1]) pending and a read (t[0]) -> the next sequential read needs one
        extra.clear();
        CHECK(m.task(&r, 1, true, extra, &why) == 0 && extra.size() == 1);
        (void) w;
    }
    {
        // a concurrent read while concurrent writes of an earlier task are pending
        Map m;
        Access cw{h, 2, 4}, cr{h, 1, 4}, sw{h, 2, 1};
        extra.clear();
        CHECK(m.task(&cw, 1, true, extra, &why) == 0 && extra.empty());
        CHECK(m.task(&cr, 1, true, extra, &why) == -22);
        CHECK(m.task(&cr, 1, false, extra, &why) == 0 && extra.empty());
        // the read dropped the concurrent writes from the map: a sequential write needs no extra task
        CHECK(m.task(&sw, 1, true, extra, &why) == 0 && extra.empty());
    }
    {
        // extra writers for two handles in one task, in access order; a refused task changes nothing
        Map m;
        Access rr[2] = {{h, 1, 1}, {g, 1, 1}};
        extra.clear();
        CHECK(m.task(rr, 2, true, extra, &why) == 0);
        Access cc[2] = {{g, 2, 4}, {h, 2, 4}};
        CHECK(m.task(cc, 2, true, extra, &why) == 0 && extra.size() == 2 && extra[0] == g && extra[1] == h);
        Access bad[2] = {{h, 2, 4}, {h, 1, 1}};                                // CNC-W, then a read needing an extra writer
        extra.clear();
        CHECK(m.task(bad, 2, true, extra, &why) == -22 && extra.empty());
        Access one{h, 1, 1};
        CHECK(m.task(&one, 1, true, extra, &why) == 0 && extra.size() == 1); // state unchanged by the refusal
    }
    if (fails) return 1;
    std::printf("ok\n");
    return 0;
}
