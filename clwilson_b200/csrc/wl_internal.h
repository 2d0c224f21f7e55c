// wl_internal.h -- data layout shared by the CUDA kernels and the host engine.
#pragma once
#include <stdint.h>
#include <stdlib.h>
#include <cuda_runtime.h>

namespace wl {

// Sieve geometry: one CTA sieves SEG_SPAN consecutive integers, odd ones only,
// as a SEG_WORDS x 32-bit bitmap in shared memory.
constexpr uint32_t SEG_SPAN = 1u << 18;
constexpr uint32_t SEG_BITS = SEG_SPAN / 2;
constexpr uint32_t SEG_WORDS = SEG_BITS / 32;

// Per-row modulus constants.  Only the first L limbs of n are meaningful.
struct __align__(32) RowMod {
    uint32_t n[4];     // n = p^2, little-endian 32-bit limbs
    uint32_t ninv;     // -n^-1 mod 2^32
    uint32_t pad;
    uint64_t p;
};

// A bucket: the test primes of one (range, residue class).  All rows of a
// bucket share the class target T and so the column set (sieving primes
// q <= T, q < q_cap) and the Legendre exponents v_q(T!).
struct Bucket {
    uint64_t T;          // shared class target (cl_wilson.cpp:1557-1579)
    uint64_t part_base;  // partial products: part[part_base + s*nrows + r]
    uint32_t ncols;      // columns used: cols[0 .. ncols)
    uint32_t row_begin;  // first row (global index) of this bucket
    uint32_t nrows;
    uint32_t nsplit;     // column splits
    uint32_t def_base;   // split deficits: defs[def_base + s]
    uint32_t L;          // limb width (2, 3, 4)
    uint32_t type;       // 0: p = 1 mod 3, 1: p = 5 mod 12, 2: p = 11 mod 12
    uint32_t range;      // index of the range this bucket belongs to
    uint32_t cdense;     // columns [0, cdense) take the dense sweep (exponent changes at
                         // nearly every column), [cdense, ncols) the prefix-fold sweep
    uint32_t ndense;     // splits 0 .. ndense-1 cover the dense columns, the rest the others
    uint32_t dstart;     // dense split s covers columns [dsplit[dstart+s], dsplit[dstart+s+1])
    uint32_t cbase;      // column offset: split ranges are relative to cols + cbase (a serving
                         // step sweeps the chunk [cbase, cbase + ncols) of the bucket's columns)
};

// Column range [c0, c1) of split s of a bucket.  Dense splits have explicit
// boundaries (dsplit, balanced by estimated cost); the others are equal.
__host__ __device__ inline void split_range(const Bucket& b, uint32_t s, uint64_t* c0, uint64_t* c1,
                                            const uint32_t* dsplit = nullptr) {
    if (s < b.ndense) {
        if (dsplit) {
            *c0 = dsplit[b.dstart + s];
            *c1 = dsplit[b.dstart + s + 1];
        } else {
            *c0 = (uint64_t)b.cdense * s / b.ndense;
            *c1 = (uint64_t)b.cdense * (s + 1) / b.ndense;
        }
    } else {
        const uint64_t n = b.ncols - b.cdense, k = b.nsplit - b.ndense, j = s - b.ndense;
        *c0 = b.cdense + n * j / k;
        *c1 = b.cdense + n * (j + 1) / k;
    }
    *c0 += b.cbase;
    *c1 += b.cbase;
}

// Shape of the dense sweep for a bucket of nrows rows: rows per thread (1; 2
// with WL_DENSE_RPT=2) and threads per split (256, or the power of two >= 8
// that covers the rows of a small bucket).
inline void dense_shape(uint32_t nrows, int* rpt, uint32_t* tps) {
    static const int env_rpt = getenv("WL_DENSE_RPT") ? atoi(getenv("WL_DENSE_RPT")) : 0;
    const int r = (env_rpt == 2 && nrows >= 64) ? 2 : 1;
    uint32_t t = 256;
    if (nrows < 256u * (uint32_t)r) {
        t = 8;   // at most 32 splits per CTA
        while (t * (uint32_t)r < nrows) t <<= 1;
    }
    *rpt = r;
    *tps = t;
}

// One CTA of the column sweep: threads [k*tps, (k+1)*tps) work on split
// split0 + k; thread i of a group takes rows row0 + i + j*tps, j < RPT.
// The CTA runs 256 / tps splits, except that a dense-sweep item may set its
// count in the high half of `tps` (item_tps / item_groups): the last,
// partly filled row tile of a bucket runs one split in a narrower group, with
// the chunk length of the bucket's full tiles.
struct SweepItem {
    uint32_t bucket, row0, split0, tps;
};
__host__ __device__ inline uint32_t item_tps(const SweepItem& it) { return it.tps & 0xFFFFu; }
__host__ __device__ inline uint32_t item_groups(const SweepItem& it) {
    return (it.tps >> 16) ? (it.tps >> 16) : 256u / (it.tps & 0xFFFFu);
}

// Per-row state beyond the modulus.
struct RowInfo {
    uint64_t p;
    uint64_t Tp;         // own target (p-1)/6, /4 or /2
    uint32_t bucket;
    uint32_t it_begin;   // tail items [it_begin, it_begin + it_count): item k multiplies
    uint32_t it_count;   // N = T+1+k*K .. min(T+(k+1)*K, Tp), K uniform per call
    uint32_t type;
};

// Per-row output.
struct RowOut {
    uint64_t s0, s1;     // digits of T_p! mod p^2 (or of the capped partial product)
    uint64_t rem, quot;  // ((p-1)! + 1) mod p^2 = rem + p*quot
    uint32_t status;     // 0 ok, 1 rem != 0, 2 no representation found
    uint32_t pad;
};

struct Deficit { uint64_t lo, hi; };

// Sieve geometry above 2^32: 2^21 integers per segment (odd ones: 2^20 bits,
// a 128 KB shared-memory bitmap), several consecutive segments per CTA.
constexpr uint32_t BIG_SPAN = 1u << 21;
constexpr uint32_t BIG_BITS = BIG_SPAN / 2;
constexpr uint32_t BIG_WORDS = BIG_BITS / 32;
constexpr uint32_t BIG_PRESIEVE = 17;   // odd primes 3..61 are removed by mask tables

// Launch wrappers (wl_kernels.cu).  All are asynchronous on `st`.
void launch_sieve_segments(uint32_t seg0, uint32_t nseg, uint64_t limit, const uint32_t* base,
                           uint32_t nbase, uint32_t* bitmap, uint32_t* seg_count, cudaStream_t st);
void launch_scan_counts(const uint32_t* counts, uint32_t n, uint64_t first, uint64_t* offsets,
                        cudaStream_t st);
void launch_compact(uint32_t nseg, uint64_t lo0, const uint32_t* bitmap, const uint64_t* offsets,
                    uint32_t* out32, uint64_t* out64, cudaStream_t st);
// One range's window of test primes: odd numbers lo0 + 2i + 1 tested in [lo, hi);
// bitmap words from word_off, segment counts from seg_off, blocks from block0.
struct WinDesc {
    uint64_t lo0, lo, hi;
    uint64_t word_off, seg_off;
    uint32_t block0, pad;
};
void launch_window_primes_multi(const WinDesc* d, uint32_t nr, uint32_t nblocks, uint32_t* bitmap,
                                uint32_t* seg_count, cudaStream_t st);
void launch_compact_multi(uint32_t nseg, const uint64_t* seg_lo, const uint32_t* bitmap, const uint64_t* offsets,
                          uint64_t* out64, cudaStream_t st);
void launch_count_leq(const uint32_t* cols, uint64_t ncols, const uint64_t* keys, uint32_t nkeys,
                      uint64_t* out, cudaStream_t st);
void launch_setup_rows(const RowInfo* info, uint32_t nrows, RowMod* mods, cudaStream_t st);
// Column groups: the resident column table in aligned groups of COL_GROUP
// primes, each group's exact product as little-endian 32-bit limbs
// (gprod[COL_GROUP*g ..], gk[g] limbs, at most COL_GROUP).  ColGroups{} (no
// table) makes the prefix-fold sweep take every column as one cell.
constexpr uint32_t COL_GROUP = 32;
struct ColGroups {
    const uint32_t* gprod = nullptr;
    const uint8_t* gk = nullptr;
    uint64_t ngroups = 0;
};
void launch_group_products(const uint32_t* cols, uint64_t ngroups, uint32_t* gprod, uint8_t* gk, cudaStream_t st);
// cols: the column table whose index 0 the groups are aligned to
void launch_sweep(int variant, int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                  const RowMod* mods, const uint32_t* cols, uint4* part, Deficit* defs, cudaStream_t st,
                  ColGroups groups = ColGroups());
// dense sweep kernels: digit-sorted windows (3-bit at 3 CTAs/SM, 4-bit at
// 2 CTAs/SM, 3-bit at 2 CTAs/SM with every value in registers), a per-column
// bucket switch (3- and 4-bit), or digit-sorted windows with the buckets in
// shared memory (3-bit at 4 CTAs/SM, 4-bit at 2)
enum { DENSE_SORTED_W3 = 0, DENSE_SORTED_W4 = 1, DENSE_SWITCH_W3 = 2, DENSE_SWITCH_W4 = 3, DENSE_SMEM_W3 = 4,
       DENSE_SMEM_W4 = 5, DENSE_SORTED_W3_2CTA = 6 };
// work (may be null): adds the launch's column cells, window cells and full products, summed over rows
void launch_sweep_dense(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                        const RowMod* mods, const uint32_t* cols, const uint32_t* dsplit, uint4* part, Deficit* defs,
                        cudaStream_t st, int kernel, uint32_t hstep, unsigned long long* work = nullptr);
void launch_sieve_big(uint64_t lo, uint64_t hi, uint32_t nseg, uint32_t segs_per_cta, const uint32_t* base,
                      uint32_t nbase, uint32_t* offsets, uint32_t* bitmap, uint32_t* seg_count, cudaStream_t st);
void launch_compact_big(uint32_t nseg, uint64_t lo0, const uint32_t* bitmap, const uint64_t* offsets, uint64_t* out,
                        cudaStream_t st);
void launch_count_leq64(const uint64_t* cols, uint64_t ncols, const uint64_t* keys, uint32_t nkeys, uint64_t* out,
                        cudaStream_t st);
void launch_sweep64(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items, const RowMod* mods,
                    const uint64_t* cols, uint4* part, Deficit* defs, cudaStream_t st);
// los (may be null): per-bucket bitmap regions, bucket b's at word cbase holding los[b] + 64w + 1 + 2i
void launch_sweep_bits(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                       const RowMod* mods, const uint32_t* bitmap, uint64_t lo, const uint64_t* keys, uint4* part,
                       Deficit* defs, cudaStream_t st, const uint64_t* los = nullptr);
void launch_count_bits(const uint32_t* bitmap, uint64_t lo, uint64_t nwords, uint64_t key, unsigned long long* out,
                       cudaStream_t st);
void launch_merge(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* part,
                  const Deficit* defs, uint32_t row_begin, uint32_t nrows, uint4* acc, Deficit* bdef, cudaStream_t st);
void launch_acc_init(uint32_t nrows, uint32_t nbuckets, uint4* acc, Deficit* bdef, cudaStream_t st);
void launch_clear_below(uint32_t* bitmap, uint64_t lo, uint64_t q_lo, uint64_t nwords, cudaStream_t st);
void launch_clear_tail(RowInfo* info, uint32_t row_begin, uint32_t nrows, cudaStream_t st);
void launch_tail_merge(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* ipart,
                       uint64_t K, uint32_t row_begin, uint32_t nrows, uint4* acc, Deficit* bdef, cudaStream_t st);
void launch_merge_cta(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* part,
                      const Deficit* defs, uint32_t row_begin, uint32_t nrows, uint4* acc, Deficit* bdef,
                      cudaStream_t st);
void launch_iterate(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, uint32_t row_begin,
                    uint32_t nrows, uint32_t item_begin, uint32_t nitems, uint64_t K, uint4* out, cudaStream_t st);
void launch_finish(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods,
                   const uint4* part, const Deficit* defs, uint64_t K, const uint4* ipart,
                   uint32_t row_begin, uint32_t nrows, int full, RowOut* out, cudaStream_t st,
                   const uint4* acc1 = nullptr, const Deficit* def1 = nullptr,
                   const uint4* acc2 = nullptr, const Deficit* def2 = nullptr);
// out = row-wise product of nparts partial products (digits s0, s1 per row)
void launch_rows_product(const uint64_t* ps, uint64_t n_rows, const uint64_t* parts, uint32_t nparts, uint64_t* out,
                         cudaStream_t st);

}  // namespace wl
