// PoolArray (xkaapi_b200/csrc/pool.h): fixed reservations, growth, and the parking of released
// fixed reservations for the next reservation of the same size in the process.
#include "../../xkaapi_b200/csrc/pool.h"

#include <cstdio>
#include <cstdlib>

#define CHECK(c) do { if (!(c)) { std::fprintf(stderr, "line %d: %s\n", __LINE__, #c); return 1; } } while (0)

struct Rec { long a, b; };

int main()
{
    const size_t N = size_t(1) << 20;
    void * first = nullptr;
    {
        xkb::PoolArray<Rec> p;
        CHECK(p.reserve_fixed(N));
        CHECK(p.fixed());
        for (size_t i = 0; i < 1000; ++i) CHECK(p.push_back(Rec{(long) i, -(long) i}));
        CHECK(p.size() == 1000 && p[999].a == 999 && p[999].b == -999);
        CHECK(!p.resize(N + 1));                         // a fixed reservation never grows past its size
        CHECK(p.size() == 1000);
        first = p.data();
    }                                                    // released: parked
    {
        xkb::PoolArray<Rec> q;
        CHECK(q.reserve_fixed(N));
        CHECK(q.data() == first);                        // the parked reservation, reused
        CHECK(q.size() == 0);                            // empty again; old contents are not elements
        CHECK(q.push_back(Rec{7, 8}) && q[0].a == 7);
        xkb::PoolArray<Rec> r;
        CHECK(r.reserve_fixed(N));                       // none parked now: a new mapping
        CHECK(r.data() != first);
        xkb::PoolArray<Rec> s;
        CHECK(s.reserve_fixed(N / 2));                   // another size never takes a parked one
    }
    {
        xkb::PoolArray<Rec> g;                           // growable (not fixed): mremap growth keeps contents
        for (size_t i = 0; i < 3 * N; ++i) CHECK(g.push_back(Rec{(long) i, 0}));
        CHECK(g[3 * N - 1].a == (long) (3 * N - 1) && g[12345].a == 12345);
        g.release();
        CHECK(g.size() == 0 && g.data() == nullptr);
    }
    std::printf("ok\n");
    return 0;
}
