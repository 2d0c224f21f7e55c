// wl_host.h -- host-side internals shared by the engine (wl_engine.cu) and the
// serving session (wl_serve.cu): device buffers, error macros, the context.
#pragma once
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include <cuda_runtime.h>

#include "wilson.h"
#include "wl_internal.h"

// A growable device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

inline int ensure(DevBuf& b, size_t bytes) {
    if (bytes <= b.cap && b.p) return 0;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t nb = std::max<size_t>(bytes, 256);
    if (cudaMalloc(&b.p, nb) != cudaSuccess) {
        cudaGetLastError();
        return WL_ERR_NOMEM;
    }
    b.cap = nb;
    return 0;
}

template <class T> inline T* as(DevBuf& b) { return reinterpret_cast<T*>(b.p); }

// Rows per thread of the prefix-fold sweep for a bucket of nrows rows, given
// the tuned choice (1, 2 or 4): one row below 512 rows, at most two below 1,024.
inline int sparse_rpt_for(int tuned, uint32_t nrows) {
    if (nrows < 512) return 1;
    if (tuned == 4 && nrows < 1024) return 2;
    return tuned;
}

// Row tiles of a bucket's n rows for the sweep kernels (256-thread CTAs).
// Full tiles of 256 * rpt rows (one split per CTA), then tiles of 256 rows,
// then the last rows in one tile whose group width is the rest rounded up to
// a power of two (at least min_tps) up to 32 rows and to a multiple of 32
// above: several splits share a CTA when the width is below 256, and few
// lanes carry no row (a power-of-two width for the rest would leave up to
// half of them empty).
// same_groups: every tile of the bucket runs the same number of splits per
// CTA -- the dense sweep stages a CTA's columns in chunks shared by its
// groups, and the power of two that a split's product drops depends on the
// chunk length, so all rows of a split must see the same chunks.  Then a
// bucket of 256 * rpt rows or more keeps full tiles, one split per CTA, and
// its last rows go in one tile of the rest's width that also runs one split
// per CTA (groups = 1; the CTA's threads past it idle); a smaller bucket is
// one tile.
struct RowTile {
    uint32_t row0, tps;
    int rpt;
    uint32_t groups = 0;     // splits per CTA; 0: 256 / tps
};
inline uint32_t group_width(uint32_t lanes, uint32_t min_tps) {
    uint32_t t = min_tps;
    if (lanes <= 32) { while (t < lanes) t <<= 1; }
    else t = (lanes + 31) / 32 * 32;
    return t;
}
inline void row_tiles(uint32_t n, int rpt, uint32_t min_tps, std::vector<RowTile>& out, bool same_groups = false) {
    out.clear();
    uint32_t r0 = 0;
    const uint32_t full = 256u * (uint32_t)rpt;
    while (n - r0 >= full) { out.push_back({ r0, 256u, rpt }); r0 += full; }
    if (same_groups && r0 > 0) {
        const uint32_t rest = n - r0;
        if (rest) out.push_back({ r0, group_width((rest + rpt - 1) / rpt, min_tps), rpt, 1u });
        return;
    }
    while (n - r0 >= 256u) { out.push_back({ r0, 256u, 1 }); r0 += 256u; }
    const uint32_t rest = n - r0;
    if (!rest) return;
    out.push_back({ r0, group_width(rest, min_tps), 1 });
}
// Splits one item of the tile runs.
inline uint32_t tile_groups(const RowTile& t) { return t.groups ? t.groups : 256u / t.tps; }
// The sweep items of one tile: one per split for full-width tiles, else one
// per tile_groups consecutive splits.
template <class Push>
inline void tile_items(const RowTile& t, uint32_t s_begin, uint32_t s_end, Push push) {
    const uint32_t per = tile_groups(t);
    const uint32_t code = t.groups ? (t.tps | (t.groups << 16)) : t.tps;
    for (uint32_t s = s_begin; s < s_end; s += per) push(t.row0, s, code);
}

// Limb width of residues mod p^2 for primes up to pmax_incl.
inline int limb_width(uint64_t pmax_incl) {
    if (pmax_incl < (1ull << 31)) return 2;
    if (pmax_incl < (1ull << 47)) return 3;
    return 4;
}

#define CK(x)                                                        \
    do {                                                             \
        cudaError_t e_ = (x);                                        \
        if (e_ != cudaSuccess) {                                     \
            fprintf(stderr, "wilson: CUDA error %s at %s:%d\n",      \
                    cudaGetErrorString(e_), __FILE__, __LINE__);     \
            return WL_ERR_CUDA;                                      \
        }                                                            \
    } while (0)

#define RC(x)                      \
    do {                           \
        int r_ = (x);              \
        if (r_) return r_;         \
    } while (0)

struct wl_ctx {
    int device = 0;
    int sms = 148;
    int cell_variant = 1;   // formulation of the sweep's cell step (see wl_kernels.cu cellv)
    wl_tuning tune = {};     // sweep kernel choices per limb width (wl_autotune)
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;   // dense sweep, overlapped with the sparse sweep
    cudaEvent_t ev[8] = {};
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t big0 = nullptr, big1 = nullptr;
    cudaEvent_t rows_ready = nullptr;   // row tables uploaded and k_setup_rows done (main stream)
    double ms_big = 0;
    DevBuf base;            // odd primes < 65536 (sieving primes of the column sieve)
    uint32_t nbase = 0;
    DevBuf cols;            // column cache: all primes < col_limit, ascending, u32
    uint64_t ncols = 0, col_limit = 0;
    DevBuf gprod, gk;       // exact products of its aligned groups of COL_GROUP columns
    uint64_t ngroups = 0;
    DevBuf bitmap, segcount, offsets;
    DevBuf tp, keys, counts, buckets, rowinfo, rowmod, items, part, ipart, defs, rowout, dsplit;
    // columns above 2^32
    cudaStream_t st3 = nullptr;
    DevBuf bbitmap, bsegcount, boffsets, boffs, wcols, wbuckets, witems, wpart, wdefs, bacc, bdef, wkeys, wcounts;
    DevBuf uacc, udef;   // columns below 2^32: per-row product of all splits, per-bucket deficit
    DevBuf prod;         // wl_rows_product: moduli, partial products, products
    DevBuf windesc, seglo;   // test-prime windows of all ranges, their segment starts
    uint32_t launches = 0;
    uint64_t h2d = 0, d2h = 0;
    double ms_sieve = 0;
    uint64_t sieve_ints = 0, sieve_bytes = 0;
    DevBuf work;         // dense sweep work counters: column cells, window cells, products
};

// The column groups of the resident table for the prefix-fold sweep
// (WL_COL_GROUPS=0 in the environment turns them off, for comparisons).
inline wl::ColGroups col_groups(wl_ctx* c) {
    static const bool off = getenv("WL_COL_GROUPS") && atoi(getenv("WL_COL_GROUPS")) == 0;
    wl::ColGroups g;
    if (off || !c->ngroups) return g;
    g.gprod = as<uint32_t>(c->gprod);
    g.gk = as<uint8_t>(c->gk);
    g.ngroups = c->ngroups;
    return g;
}

// A range's window of test primes and its classes.
struct RangeState {
    uint64_t pmin, pmax, lo0;
    uint32_t nseg;
    uint64_t word_off, seg_off;
    uint64_t tp_off = 0, ntp = 0;
    uint64_t T[3] = { 0, 0, 0 };
    uint64_t per_class[3] = { 0, 0, 0 };
};

// Every prime below `limit` (<= 2^32) in the context's resident column table.
int ensure_columns(wl_ctx* c, uint64_t limit);
// Test primes of each range, ascending (deterministic Miller-Rabin on the
// device); with allow_empty a range without primes is not an error.
int gen_test_primes(wl_ctx* c, const wl_range* ranges, size_t nr, std::vector<RangeState>& rs,
                    std::vector<uint64_t>& tps, bool allow_empty = false);
// results.txt value of one row (cl_wilson.cpp:872-898): 1 if it is a result line.
int result_of(const wl_row& r, int32_t* value);
