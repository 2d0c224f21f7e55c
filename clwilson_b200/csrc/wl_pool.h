// wl_pool.h -- the serving session's row pool: first-fit allocation of
// contiguous row ranges, with freed ranges coalesced with their neighbours.
// Host code only (no CUDA).
#pragma once
#include <cstdint>
#include <iterator>
#include <map>

struct RowPool {
    uint32_t cap = 0, used = 0;
    std::map<uint32_t, uint32_t> free;   // first row of a free range -> its length

    void reset(uint32_t rows) {
        cap = rows;
        used = 0;
        free.clear();
        if (rows) free[0] = rows;
    }

    // The lowest free range of at least n rows; false when none has room.
    bool alloc(uint32_t n, uint32_t* r0) {
        if (n == 0) return false;
        for (auto it = free.begin(); it != free.end(); ++it) {
            if (it->second < n) continue;
            *r0 = it->first;
            const uint32_t rest = it->second - n, start = it->first + n;
            free.erase(it);
            if (rest) free[start] = rest;
            used += n;
            return true;
        }
        return false;
    }

    // Return rows [r0, r0 + n), merged with the free ranges next to them.
    void release(uint32_t r0, uint32_t n) {
        if (n == 0) return;
        used -= n;
        auto it = free.emplace(r0, n).first;
        auto nx = std::next(it);
        if (nx != free.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free.erase(nx);
        }
        if (it != free.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free.erase(it);
            }
        }
    }
};
