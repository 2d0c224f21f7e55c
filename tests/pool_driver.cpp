// Test driver for clwilson_b200/csrc/wl_pool.h (the serving row pool), used by
// tests/test_row_pool.py: random allocations and releases against a row map,
// checking after every operation that allocated ranges do not overlap, that the
// free ranges are disjoint, fully coalesced and cover exactly the unused rows,
// and that first fit returns the lowest range with room.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include "wl_pool.h"

static int fail(const char* what, long op) {
    printf("FAIL %s at operation %ld\n", what, op);
    return 1;
}

int main(int argc, char** argv) {
    const uint32_t cap = argc > 1 ? (uint32_t)atoi(argv[1]) : 5000;
    const long ops = argc > 2 ? atol(argv[2]) : 200000;
    std::mt19937_64 rng(argc > 3 ? atoi(argv[3]) : 1);
    RowPool pool;
    pool.reset(cap);
    std::vector<int> owner(cap, -1);                      // row -> allocation id
    std::vector<std::pair<uint32_t, uint32_t>> live;      // (r0, n)
    long fits = 0, misses = 0;
    for (long op = 0; op < ops; ++op) {
        if (live.empty() || rng() % 100 < 55) {
            const uint32_t n = 1 + (uint32_t)(rng() % (rng() % 8 == 0 ? cap / 2 : 64));
            // the lowest start of a free run of n rows
            long want = -1;
            for (uint32_t r = 0, run = 0; r < cap; ++r) {
                run = owner[r] < 0 ? run + 1 : 0;
                if (run == n) { want = (long)r + 1 - n; break; }
            }
            uint32_t r0 = 0;
            const bool ok = pool.alloc(n, &r0);
            if (ok != (want >= 0)) return fail("alloc result", op);
            if (!ok) { ++misses; continue; }
            if ((long)r0 != want) return fail("first fit", op);
            for (uint32_t r = r0; r < r0 + n; ++r) owner[r] = (int)op;
            live.push_back({ r0, n });
            ++fits;
        } else {
            const size_t k = rng() % live.size();
            const auto a = live[k];
            live[k] = live.back();
            live.pop_back();
            for (uint32_t r = a.first; r < a.first + a.second; ++r) {
                if (owner[r] < 0) return fail("double free", op);
                owner[r] = -1;
            }
            pool.release(a.first, a.second);
        }
        // invariants
        uint32_t used = 0;
        for (uint32_t r = 0; r < cap; ++r) used += owner[r] >= 0;
        if (used != pool.used) return fail("used count", op);
        uint32_t prev_end = 0, free_rows = 0;
        bool first = true;
        for (const auto& f : pool.free) {
            if (f.second == 0) return fail("empty free range", op);
            if (!first && f.first <= prev_end) return fail("free ranges overlap or touch", op);
            for (uint32_t r = f.first; r < f.first + f.second; ++r)
                if (owner[r] >= 0) return fail("free range over used rows", op);
            free_rows += f.second;
            prev_end = f.first + f.second;
            first = false;
        }
        if (free_rows + used != cap) return fail("free + used != capacity", op);
    }
    printf("ok %ld allocations, %ld without room\n", fits, misses);
    return 0;
}
