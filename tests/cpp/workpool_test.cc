// WorkPool (xkaapi_b200/csrc/workpool.h): every member runs the function once per run(), runs
// follow one another, a one-member pool runs on the caller, destruction joins the members.
#include "../../xkaapi_b200/csrc/workpool.h"

#include <atomic>
#include <cstdio>
#include <vector>

int main()
{
    for (unsigned n : {1u, 2u, 7u, 16u})
    {
        xkb::WorkPool pool(n);
        if (pool.size() != n) { std::fprintf(stderr, "size %u != %u\n", pool.size(), n); return 1; }
        std::vector<int> hits(n, 0);
        std::atomic<long> sum(0);
        for (int round = 0; round < 200; ++round)
            pool.run([&](unsigned k) { hits[k] += 1; sum += (long) k + round; });
        long want = 0;
        for (int round = 0; round < 200; ++round)
            for (unsigned k = 0; k < n; ++k) want += (long) k + round;
        for (unsigned k = 0; k < n; ++k)
            if (hits[k] != 200) { std::fprintf(stderr, "member %u ran %d times\n", k, hits[k]); return 1; }
        if (sum != want) { std::fprintf(stderr, "sum %ld != %ld\n", (long) sum, want); return 1; }
    }
    std::printf("ok\n");
    return 0;
}
