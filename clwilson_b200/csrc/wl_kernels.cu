// wl_kernels.cu -- sm_100a kernels of the Wilson-prime engine.
//
//   k_sieve_segments / k_compact   sieving primes q < 2^32 (the columns)
//   k_window_primes_multi          test primes in [pmin, pmax) of every range (the rows)
//   k_setup_rows                   per-row modulus constants (setup.cl)
//   k_sweep<L,RPT>                 prod_{q <= T} q^{v_q(T!)} over a column split
//                                  (mulsmall.cl / mullarge.cl / reduce.cl)
//   k_iterate<L>                   prod of consecutive integers (iterate.cl)
//   k_finish<L>                    combine splits + tail, class lift, quotient
//                                  (cl_wilson.cpp:691-900, find.cl)
#include <cstdlib>

#include "wl_internal.h"
#include "wl_arith.cuh"

namespace wl {

// ===========================================================================
// Column sieve: all primes below `limit` (limit <= 2^32), odd-only segmented
// sieve of Eratosthenes with the bitmap in shared memory.
// ===========================================================================

constexpr uint32_t SIEVE_THREADS = 512;
constexpr uint32_t SMALL_PRIME_COOP = 1024;   // primes below this are marked cooperatively

__global__ void __launch_bounds__(SIEVE_THREADS)
k_sieve_segments(uint32_t seg0, uint64_t limit, const uint32_t* __restrict__ base, uint32_t nbase,
                 uint32_t* __restrict__ bitmap, uint32_t* __restrict__ seg_count) {
    __shared__ uint32_t marks[SEG_WORDS];
    __shared__ uint32_t warp_sum[SIEVE_THREADS / 32];
    const uint32_t seg = seg0 + blockIdx.x;
    const uint64_t lo = (uint64_t)seg * SEG_SPAN;
    const uint64_t hi = lo + SEG_SPAN;
    for (uint32_t i = threadIdx.x; i < SEG_WORDS; i += blockDim.x) marks[i] = 0;
    __syncthreads();

    // base primes are odd primes in ascending order; stop once b^2 >= hi
    uint32_t k = 0;
    // cooperative marking for small primes: thread t marks multiples t, t+T, ...
    for (; k < nbase; ++k) {
        const uint64_t b = base[k];
        if (b >= SMALL_PRIME_COOP || b * b >= hi) break;
        uint64_t m = (lo + b - 1) / b * b;
        if (m < b * b) m = b * b;
        if (!(m & 1)) m += b;
        if (m >= hi) continue;
        const uint32_t i0 = (uint32_t)((m - lo) >> 1);
        for (uint32_t i = i0 + threadIdx.x * (uint32_t)b; i < SEG_BITS; i += blockDim.x * (uint32_t)b)
            atomicOr(&marks[i >> 5], 1u << (i & 31));
    }
    // one larger prime per thread
    for (uint32_t kk = k + threadIdx.x; kk < nbase; kk += blockDim.x) {
        const uint64_t b = base[kk];
        if (b * b >= hi) break;
        uint64_t m = (lo + b - 1) / b * b;
        if (m < b * b) m = b * b;
        if (!(m & 1)) m += b;
        for (uint64_t i = (m - lo) >> 1; i < SEG_BITS; i += b)
            atomicOr(&marks[i >> 5], 1u << (i & 31));
    }
    __syncthreads();

    uint32_t cnt = 0;
    for (uint32_t w = threadIdx.x; w < SEG_WORDS; w += blockDim.x) {
        uint32_t prime_bits = ~marks[w];
        const uint64_t first = lo + (uint64_t)w * 64 + 1;           // number of bit 0
        if (first + 62 >= limit) {                                   // clip to < limit
            uint32_t keep = 0;
            for (int bI = 0; bI < 32; ++bI)
                if (first + 2 * (uint64_t)bI < limit) keep |= 1u << bI;
            prime_bits &= keep;
        }
        if (seg == 0 && w == 0) prime_bits &= ~1u;                  // 1 is not prime
        bitmap[(uint64_t)blockIdx.x * SEG_WORDS + w] = prime_bits;
        cnt += __popc(prime_bits);
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (uint32_t i = 0; i < blockDim.x / 32; ++i) s += warp_sum[i];
        seg_count[blockIdx.x] = s;
    }
}

// Exclusive scan of per-segment counts (single CTA), offsets[i] = first + sum_{j<i} counts[j];
// offsets[n] = total.
__global__ void __launch_bounds__(1024)
k_scan_counts(const uint32_t* __restrict__ counts, uint32_t n, uint64_t first, uint64_t* __restrict__ offsets) {
    __shared__ uint64_t part[1024];
    const uint32_t per = (n + blockDim.x - 1) / blockDim.x;
    const uint32_t b = threadIdx.x * per, e = min(n, b + per);
    uint64_t s = 0;
    for (uint32_t i = b; i < e; ++i) s += counts[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
        uint64_t v = (threadIdx.x >= off) ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint64_t run = first + (threadIdx.x ? part[threadIdx.x - 1] : 0);
    for (uint32_t i = b; i < e; ++i) { offsets[i] = run; run += counts[i]; }
    if (threadIdx.x == blockDim.x - 1) offsets[n] = first + part[blockDim.x - 1];
}

// Ordered write-out of the numbers whose bit is set: segment s covers odd
// numbers lo + 2i + 1 with lo = seg_lo[s], or lo0 + s*span without seg_lo.
// Writes 32-bit or 64-bit values.
constexpr uint32_t COMPACT_THREADS = 256;
__global__ void __launch_bounds__(COMPACT_THREADS)
k_compact(uint64_t lo0, uint32_t span, const uint32_t* __restrict__ bitmap, const uint64_t* __restrict__ offsets,
          uint32_t* __restrict__ out32, uint64_t* __restrict__ out64, const uint64_t* __restrict__ seg_lo) {
    __shared__ uint32_t wsum[COMPACT_THREADS / 32];
    constexpr uint32_t WPT = SEG_WORDS / COMPACT_THREADS;   // words per thread
    const uint32_t seg = blockIdx.x;
    const uint32_t* bm = bitmap + (uint64_t)seg * SEG_WORDS + threadIdx.x * WPT;
    uint32_t words[WPT];
    uint32_t cnt = 0;
#pragma unroll
    for (uint32_t i = 0; i < WPT; ++i) { words[i] = bm[i]; cnt += __popc(words[i]); }
    // block exclusive scan of cnt
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (uint32_t i = 0; i < wid; ++i) wbase += wsum[i];
    uint64_t pos = offsets[seg] + wbase + incl - cnt;
    const uint64_t lo = seg_lo ? seg_lo[seg] : lo0 + (uint64_t)seg * span;
#pragma unroll
    for (uint32_t i = 0; i < WPT; ++i) {
        uint32_t w = words[i];
        const uint64_t base_n = lo + (uint64_t)(threadIdx.x * WPT + i) * 64 + 1;
        while (w) {
            const int bI = __ffs(w) - 1;
            w &= w - 1;
            const uint64_t v = base_n + 2 * (uint64_t)bI;
            if (out32) out32[pos] = (uint32_t)v;
            else out64[pos] = v;
            ++pos;
        }
    }
}

// ===========================================================================
// Test primes: deterministic Miller-Rabin on every odd n in [lo, hi).
// Bitmap layout as the sieve: segment s covers odd numbers lo0 + s*SEG_SPAN + 2i + 1.
// ===========================================================================

__device__ bool is_prime64(uint64_t n) {
    if (n < 2) return false;
    const uint32_t small[] = { 2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61, 67, 71 };
#pragma unroll
    for (int i = 0; i < 20; ++i) {
        if (n == small[i]) return true;
        if (n % small[i] == 0) return false;
    }
    Mod64 M;
    M.init(n);
    uint64_t d = n - 1;
    int s = __ffsll((long long)d) - 1;
    d >>= s;
    const uint64_t minus1 = M.to(n - 1);
    // bases of J. Sinclair: deterministic for n < 2^64
    const uint64_t bases[7] = { 2, 325, 9375, 28178, 450775, 9780504, 1795265022 };
    for (int i = 0; i < 7; ++i) {
        const uint64_t a = bases[i] % n;
        if (a == 0) continue;
        uint64_t x = red64(M.pow(M.to(a), d), n);
        if (x == M.one % n || x == minus1 % n) continue;
        bool ok = false;
        for (int r = 1; r < s; ++r) {
            x = red64(M.mul(x, x), n);
            if (x == minus1 % n) { ok = true; break; }
        }
        if (!ok) return false;
    }
    return true;
}

// All ranges in one launch: range r owns blocks [d[r].block0, d[r].block0 +
// ceil((hi - lo0) / 512)), one thread per odd number from its lo0, so only the
// range's own integers are tested; its bitmap words and segment counts start
// at d[r].word_off and d[r].seg_off (bitmap zeroed beforehand).
__global__ void __launch_bounds__(256)
k_window_primes_multi(const WinDesc* __restrict__ d, uint32_t nr, uint32_t* __restrict__ bitmap,
                      uint32_t* __restrict__ seg_count) {
    uint32_t a = 0, b = nr - 1;          // the last range with block0 <= blockIdx.x
    while (a < b) {
        const uint32_t m = (a + b + 1) >> 1;
        if (d[m].block0 <= blockIdx.x) a = m; else b = m - 1;
    }
    const WinDesc w = d[a];
    const uint64_t bit = (uint64_t)(blockIdx.x - w.block0) * blockDim.x + threadIdx.x;
    const uint64_t nval = w.lo0 + 2 * bit + 1;
    const bool pr = (nval >= w.lo && nval < w.hi) ? is_prime64(nval) : false;
    const uint32_t word = __ballot_sync(0xffffffffu, pr);
    if ((threadIdx.x & 31) == 0) {
        bitmap[w.word_off + (bit >> 5)] = word;
        if (word) atomicAdd(&seg_count[w.seg_off + bit / SEG_BITS], (uint32_t)__popc(word));
    }
}

// ===========================================================================
// Count of columns <= key (binary search over the sorted column array).
// ===========================================================================

// Exact product of each aligned group of COL_GROUP resident columns (one
// thread per group): little-endian 32-bit limbs gprod[COL_GROUP*g ..], gk[g]
// of them with the top one nonzero.  Each prime adds at most one limb, so a
// group takes at most COL_GROUP limbs.
__global__ void __launch_bounds__(128) k_group_products(const uint32_t* __restrict__ cols, uint64_t ngroups,
                                                        uint32_t* __restrict__ gprod, uint8_t* __restrict__ gk) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups) return;
    uint32_t acc[COL_GROUP];
    uint32_t len = 1;
    acc[0] = 1;
    const uint32_t* q = cols + g * COL_GROUP;
    for (uint32_t i = 0; i < COL_GROUP; ++i) {
        const uint32_t v = q[i];
        uint32_t carry = 0;
        for (uint32_t k = 0; k < len; ++k) {
            const uint64_t x = (uint64_t)acc[k] * v + carry;
            acc[k] = (uint32_t)x;
            carry = (uint32_t)(x >> 32);
        }
        if (carry && len < COL_GROUP) acc[len++] = carry;
    }
    for (uint32_t k = 0; k < len; ++k) gprod[g * COL_GROUP + k] = acc[k];
    gk[g] = (uint8_t)len;
}

__global__ void k_count_leq(const uint32_t* __restrict__ cols, uint64_t ncols, const uint64_t* __restrict__ keys,
                            uint32_t nkeys, uint64_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nkeys) return;
    const uint64_t key = keys[i];
    uint64_t a = 0, b = ncols;          // first index with cols[idx] > key
    while (a < b) {
        uint64_t m = (a + b) >> 1;
        if ((uint64_t)cols[m] <= key) a = m + 1; else b = m;
    }
    out[i] = a;
}

// ===========================================================================
// Row setup: n = p^2 and -n^-1 mod 2^32 (setup.cl:18-45 computes the
// reference's own per-prime constants; these are this engine's).
// ===========================================================================

__global__ void k_setup_rows(const RowInfo* __restrict__ info, uint32_t nrows, RowMod* __restrict__ mods) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const uint64_t p = info[i].p;
    const u128 n = (u128)p * p;
    RowMod r;
    r.n[0] = (uint32_t)n;
    r.n[1] = (uint32_t)(n >> 32);
    r.n[2] = (uint32_t)(n >> 64);
    r.n[3] = (uint32_t)(n >> 96);
    uint32_t x = r.n[0];                // n^-1 mod 2^32 by Newton
    for (int k = 0; k < 5; ++k) x *= 2u - r.n[0] * x;
    r.ninv = 0u - x;
    r.pad = 0;
    r.p = p;
    mods[i] = r;
}

// ===========================================================================
// Column sweep.  For the bucket's target T and a split [c0, c1) of the
// ascending column array (primes q <= T), each row computes
//     C = prod_{c0 <= i < c1} q_i^{e_i},   e_i = v_{q_i}(T!)  (Legendre),
// by the prefix-product identity: with P_i = q_c0 ... q_i and the exponents
// non-increasing, C = prod_{i: e_i > e_{i+1}} P_i^{e_i - e_{i+1}} (e_{c1} = 0).
// Each prime therefore costs one cell; a fold A *= P^d happens only where the
// exponent drops, which for q > sqrt(T) is once per distinct floor(T/q).
// An aligned group of COL_GROUP columns with one exponent costs less: P is
// multiplied by the group's exact product, one Montgomery limb step per 32
// bits (limb_step), 27 to 29 steps for 32 primes of 27 to 29 bits.
// Fold points depend on T only, so all rows of the bucket fold together.
// Every cell or limb step drops a factor 2^32 and every full product
// 2^(32L); the total ("deficit") is identical for all rows of a split and
// stored once per split.
// ===========================================================================

template <int L>
__device__ __forceinline__ void fold_pow(Res<L>& A, const Res<L>& P, uint64_t d, const uint32_t* n, uint32_t ninv) {
    Res<L> Y = P;
    const int top = 63 - __clzll((long long)d);
    for (int b = top - 1; b >= 0; --b) {
        Y = mont_mul<L>(Y, Y, n, ninv);
        if ((d >> b) & 1) Y = mont_mul<L>(Y, P, n, ninv);
    }
    A = mont_mul<L>(A, Y, n, ninv);
}

__device__ __forceinline__ uint32_t sat32(uint64_t v) { return v > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)v; }

// cell step in formulation V (0: carry-flag PTX chain, 1: wide products,
// 2: wide products with a high-half first reduction); all are exact
template <int L, int V>
__device__ __forceinline__ void cellv(Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    if (V == 0) cell(x, q, n, ninv);
    else if (V == 1) cell_w<L>(x, q, n, ninv);
    else cell_h<L>(x, q, n, ninv);
}
template <int L, int V>
__device__ __forceinline__ void cell_wide_v(Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    cellv<L, V>(x, q, n, ninv);
    cond_sub_chain(x, n);
}

// The cell of row j of a thread's RPT rows.  V = 3 mixes formulations: the
// wide-product cell on rows 0 .. RPT-2 and the carry-chain cell on the last
// row, whose instruction streams overlap in part on B200 (register-only: 3
// wide + 1 carry-chain rows run 5% / 3% / 2% faster than wide rows alone at
// L = 2 / 3 / 4).  j is a compile-time index after unrolling.
template <int L, int V, int RPT>
__device__ __forceinline__ void cellr(int j, Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    if (V == 3) {
        if (RPT > 1 && j == RPT - 1) cell(x, q, n, ninv);
        else cell_w<L>(x, q, n, ninv);
    } else {
        cellv<L, V>(x, q, n, ninv);
    }
}
template <int L, int V, int RPT>
__device__ __forceinline__ void cell_wide_r(int j, Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    cellr<L, V, RPT>(j, x, q, n, ninv);
    cond_sub_chain(x, n);
}

template <int L, int RPT, int V>
__global__ void __launch_bounds__(256)
k_sweep(const Bucket* __restrict__ buckets, const SweepItem* __restrict__ items, const RowMod* __restrict__ mods,
        const uint32_t* __restrict__ cols, uint4* __restrict__ part, Deficit* __restrict__ defs, ColGroups grp) {
    const SweepItem it = items[blockIdx.x];
    if (threadIdx.x >= (256 / it.tps) * it.tps) return;   // lanes past the CTA's last whole group
    const Bucket bk = buckets[it.bucket];
    const uint32_t s = it.split0 + threadIdx.x / it.tps;
    if (s >= bk.nsplit) return;
    const uint32_t rl = it.row0 + threadIdx.x % it.tps;

    uint32_t n[RPT][L];
    uint32_t ninv[RPT];
    bool live[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        const uint32_t r = rl + j * it.tps;
        live[j] = r < bk.nrows;
        const RowMod m = mods[bk.row_begin + (live[j] ? r : 0)];
#pragma unroll
        for (int k = 0; k < L; ++k) n[j][k] = m.n[k];
        ninv[j] = m.ninv;
    }

    const uint64_t T = bk.T;
    uint64_t c0, c1;
    split_range(bk, s, &c0, &c1);

    Res<L> P[RPT], A[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) { set_small<L>(P[j], 1); set_small<L>(A[j], 1); }
    u128 def = 0;

    if (c0 < c1) {
        const uint32_t qf = cols[c0];
        uint64_t e_cur = legendre(T, qf);
        // columns q <= thr share the exponent e_cur (valid above sqrt(T));
        // below sqrt(T) thr is the current column, so every column is checked
        uint32_t thr = sat32(((uint64_t)qf * qf > T) ? T / e_cur : qf);
        uint32_t cells = 0;
        const uint32_t* cp = cols + c0;
        const uint32_t* const ce = cols + c1;
        while (cp < ce) {
            // a whole aligned group of columns with the current exponent: its
            // exact product, limb by limb (gk limbs for COL_GROUP columns)
            if (grp.gprod != nullptr && ((uint64_t)(cp - cols) & (COL_GROUP - 1)) == 0 && cp + COL_GROUP <= ce &&
                (uint64_t)(cp - cols) / COL_GROUP < grp.ngroups && __ldg(cp + COL_GROUP - 1) <= thr) {
                const uint64_t gi = (uint64_t)(cp - cols) / COL_GROUP;
                const uint32_t k = grp.gk[gi];
                const uint32_t* gw = grp.gprod + gi * COL_GROUP;
                uint32_t t[RPT][L];
#pragma unroll
                for (int j = 0; j < RPT; ++j)
#pragma unroll
                    for (int l = 0; l < L; ++l) t[j][l] = 0;
#pragma unroll 4
                for (uint32_t i = 0; i < k; ++i) {
                    const uint32_t w = __ldg(gw + i);
#pragma unroll
                    for (int j = 0; j < RPT; ++j) limb_step<L>(t[j], P[j], w, n[j], ninv[j]);
                }
#pragma unroll
                for (int j = 0; j < RPT; ++j) {
#pragma unroll
                    for (int l = 0; l < L; ++l) P[j].w[l] = t[j][l];
                    cond_sub_chain(P[j], n[j]);
                }
                cp += COL_GROUP;
                cells += k;
                continue;
            }
            if ((((uintptr_t)cp) & 31) == 0 && cp + 8 <= ce) {
                const uint4 g0 = __ldg(reinterpret_cast<const uint4*>(cp));
                const uint4 g1 = __ldg(reinterpret_cast<const uint4*>(cp) + 1);
                if (g1.w <= thr) {
                    if (L == 2 || g1.w < 0x80000000u) {
#pragma unroll
                        for (int j = 0; j < RPT; ++j) {
                            cellr<L, V, RPT>(j, P[j], g0.x, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g0.y, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g0.z, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g0.w, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g1.x, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g1.y, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g1.z, n[j], ninv[j]);
                            cellr<L, V, RPT>(j, P[j], g1.w, n[j], ninv[j]);
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < RPT; ++j) {
                            cell_wide_r<L, V, RPT>(j, P[j], g0.x, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g0.y, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g0.z, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g0.w, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g1.x, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g1.y, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g1.z, n[j], ninv[j]);
                            cell_wide_r<L, V, RPT>(j, P[j], g1.w, n[j], ninv[j]);
                        }
                    }
                    cp += 8;
                    cells += 8;
                    continue;
                }
            }
            const uint32_t q = __ldg(cp);
            if (q > thr) {
                const uint64_t e_new = legendre(T, q);
                const uint64_t d = e_cur - e_new;
                if (d) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], d, n[j], ninv[j]);
                    def += (u128)d * (32ull * cells + 32 * L);
                }
                e_cur = e_new;
                thr = sat32(((uint64_t)q * q > T) ? T / e_new : q);
            }
            if (L == 2 || q < 0x80000000u) {
#pragma unroll
                for (int j = 0; j < RPT; ++j) cellr<L, V, RPT>(j, P[j], q, n[j], ninv[j]);
            } else {
#pragma unroll
                for (int j = 0; j < RPT; ++j) cell_wide_r<L, V, RPT>(j, P[j], q, n[j], ninv[j]);
            }
            ++cp;
            ++cells;
        }
#pragma unroll
        for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], e_cur, n[j], ninv[j]);
        def += (u128)e_cur * (32ull * cells + 32 * L);
    }

#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        if (!live[j]) continue;
        const uint32_t r = rl + j * it.tps;
        uint4 o;
        o.x = A[j].w[0];
        o.y = A[j].w[1];
        o.z = L > 2 ? A[j].w[2 < L ? 2 : 0] : 0;
        o.w = L > 3 ? A[j].w[3 < L ? 3 : 0] : 0;
        part[bk.part_base + (uint64_t)s * bk.nrows + r] = o;
    }
    if (it.row0 == 0 && threadIdx.x % it.tps == 0) {
        Deficit dd;
        dd.lo = (uint64_t)def;
        dd.hi = (uint64_t)(def >> 64);
        defs[bk.def_base + s] = dd;
    }
}

// ===========================================================================
// Dense column sweep: the same product prod q_i^{e_i} over a split, for columns
// where e_i = v_{q_i}(T!) changes at nearly every column (q^2 < ~32 T ln T),
// so that prefix folding would pay an exponentiation per column.
//
// Each exponent is split as e = H*2^s + l with l < 2^s, s chosen per split so
// that H changes about once per `hstep` columns (8 by default):
//     prod q^e = (prod q^H)^(2^s) * prod q^l.
// The first factor is the prefix-fold product on H (cheap folds, one cell per
// column), raised to 2^s by s squarings.  The second is a windowed product
// over DW-bit digits of l (3 or 4): for window j, column q goes into bucket
// B[digit_j(l)] (one cell), and prod_d B_d^d is formed with two running
// products.  Windows are combined from the top (Horner).  Cost: about
// 1 + (s/DW)(1 - 2^-DW) cells per column, plus the folds and the per-split
// combination products.
//
// The exponents are the same for every row of the bucket, so they are
// computed once per CTA per chunk of columns into shared memory.  Each CTA
// holds item_groups(it) splits (groups of tps threads), each group staging
// its own chunk.  Deficits (powers of two dropped by Montgomery steps) are uniform per
// split and tracked exactly as in k_sweep.
// ===========================================================================

constexpr int DENSE_CHUNK = 1024;    // staged columns per CTA and pass

// cell on bucket d (1 .. NB) of a window for each of the thread's RPT rows; d
// is the same for every thread of a split group (the rows of a bucket share
// their exponents), so the switch is a uniform branch and the RPT cells of a
// case are independent chains the compiler interleaves
template <int L, int NB, int RPT>
__device__ __forceinline__ void bucket_cell(Res<L> (&B)[RPT][NB], uint32_t d, uint32_t q,
                                            const uint32_t (&n)[RPT][L], const uint32_t (&ninv)[RPT], bool wide) {
    switch (d) {
#define WL_BC(k) case k: if (k <= NB) {                                                   \
            _Pragma("unroll") for (int j = 0; j < RPT; ++j) {                             \
                cell_w<L>(B[j][(k <= NB ? k : 1) - 1], q, n[j], ninv[j]);                 \
                if (wide) cond_sub_chain(B[j][(k <= NB ? k : 1) - 1], n[j]);              \
            } } break;
        WL_BC(1) WL_BC(2) WL_BC(3) WL_BC(4) WL_BC(5) WL_BC(6) WL_BC(7) WL_BC(8)
        WL_BC(9) WL_BC(10) WL_BC(11) WL_BC(12) WL_BC(13) WL_BC(14) WL_BC(15)
#undef WL_BC
        default: break;
    }
}

// One CTA: 256/tps splits of one bucket (groups of tps threads, tps >= 8);
// thread lt of a group takes rows row0 + lt + j*tps, j < RPT.  H changes about
// once per `hstep` columns of a split.
//
// SORT = 1: each staged chunk of a window pass is counting-sorted by digit in
// shared memory, and the cells of digit d run as a straight loop into bucket d
// (no per-column branch), alternating between the bucket and a second chain X
// that is folded into the bucket at the end of the digit's run (one Montgomery
// product when the run has two or more columns).
constexpr uint32_t DENSE_GMAX = 32;   // splits per CTA at most (tps >= 8)

// SMB = 1 (with SORT = 1, RPT = 1): the window buckets live in dynamic shared
// memory (bucket d of thread t at sbk[d * 256 + t]); a digit's run loads its
// bucket once, runs its cells in registers and stores it back.  That frees the
// bucket registers (more CTAs per SM, or wider windows).
//
// work (optional): the launch's work summed over rows -- work[0] += cells of
// the exponent's high part (one per column), work[1] += cells of the window
// digits, work[2] += full Montgomery products (about L cells each).  Every
// thread of a group runs the same sequence, so its first thread adds the
// group's counts times its rows.
template <int L, int MINB, int DW, int RPT, int SORT, int SMB = 0>
__global__ void __launch_bounds__(256, MINB)
k_sweep_dense(const Bucket* __restrict__ buckets, const SweepItem* __restrict__ items,
              const RowMod* __restrict__ mods, const uint32_t* __restrict__ cols, const uint32_t* __restrict__ dsplit,
              uint4* __restrict__ part, Deficit* __restrict__ defs, uint32_t hstep,
              unsigned long long* __restrict__ work) {
    __shared__ uint32_t sq[DENSE_CHUNK];
    __shared__ uint64_t sm[DENSE_CHUNK];
    __shared__ uint32_t ss[SORT ? DENSE_CHUNK : 1];       // chunk sorted by digit
    constexpr int NBK = (1 << DW) - 1;          // buckets per window
    __shared__ uint32_t scnt[DENSE_GMAX][NBK + 1];        // deficit of bucket d, in units of 32 bits
    __shared__ uint32_t scur[SORT ? DENSE_GMAX : 1][NBK + 1];
    extern __shared__ uint4 sbk[];                         // SMB: NBK x 256 buckets
    static_assert(!SMB || (SORT && RPT == 1), "shared-memory buckets need the sorted kernel, one row per thread");
    const SweepItem it = items[blockIdx.x];
    const Bucket bk = buckets[it.bucket];
    const uint32_t tps = item_tps(it);
    const uint32_t G = item_groups(it);           // splits in this CTA
    // per-group tables hold DENSE_GMAX groups (the host plans tps >= 8)
    if (tps < 8 || tps > 256 || G == 0 || G > DENSE_GMAX || G * tps > 256) return;
    const uint32_t g = threadIdx.x / tps, lt = threadIdx.x % tps;
    const uint32_t KG = DENSE_CHUNK / G;          // staged columns per split and chunk
    const uint32_t s = it.split0 + g;
    // threads past the CTA's last group (G * tps may be below 256) take no
    // split; they still pass every barrier, and g = threadIdx.x / tps <= 31 <
    // DENSE_GMAX keeps their per-group table rows in bounds
    const bool has_split = g < G && s < bk.ndense;
    const uint64_t T = bk.T;

    uint32_t n[RPT][L];
    uint32_t ninv[RPT];
    bool live[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        const uint32_t r = it.row0 + lt + j * tps;
        live[j] = has_split && r < bk.nrows;
        const RowMod m = mods[bk.row_begin + (r < bk.nrows ? r : 0)];
#pragma unroll
        for (int k = 0; k < L; ++k) n[j][k] = m.n[k];
        ninv[j] = m.ninv;
    }
    uint64_t c0 = 0, c1 = 0;
    if (has_split) split_range(bk, s, &c0, &c1, dsplit);
    // all groups of the CTA run the same number of chunks so that barriers match
    uint64_t maxlen = 0;
    for (uint32_t k = 0; k < G; ++k) {
        if (it.split0 + k >= bk.ndense) break;
        uint64_t a0, a1;
        split_range(bk, it.split0 + k, &a0, &a1, dsplit);
        if (a1 - a0 > maxlen) maxlen = a1 - a0;
    }
    const uint32_t nchunks = (uint32_t)((maxlen + KG - 1) / KG);

    // exponent split e = H*2^sb + l: H changes about once per hstep columns
    uint32_t sb = 0;
    uint64_t e_first = 0;
    if (c1 > c0) {
        e_first = legendre(T, cols[c0]);
        const uint64_t e_last = legendre(T, cols[c1 - 1]);
        const uint64_t span = e_first - e_last;
        const uint64_t per = (c1 - c0) / hstep + 1;
        const uint64_t want = span / per;         // H steps wanted: span / 2^sb <= per
        while (sb < 63 && (want >> sb) != 0) ++sb;
        const uint32_t top = 64 - __clzll((long long)e_first);
        if (sb > top) sb = top;
    }
    const uint64_t lmask = sb >= 64 ? ~0ull : ((1ull << sb) - 1);
    const uint32_t nwin = (sb + DW - 1) / DW;
    const uint32_t base = g * KG;

    // ---- pass 0: prefix product on H ----
    Res<L> P[RPT], A[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) { set_small<L>(P[j], 1); set_small<L>(A[j], 1); }
    u128 defA = 0;
    uint64_t h_cur = e_first >> sb;
    uint32_t cells = 0;
    uint64_t nprod = 0, nbucket = 0;   // work counters (full products; window cells)
    for (uint32_t ch = 0; ch < nchunks; ++ch) {
        __syncthreads();
        const uint64_t cb = c0 + (uint64_t)ch * KG;
        for (uint32_t k = lt; k < KG; k += tps) {
            if (has_split && cb + k < c1) {
                const uint32_t q = cols[cb + k];
                sq[base + k] = q;
                sm[base + k] = legendre(T, q) >> sb;
            }
        }
        __syncthreads();
        const uint32_t nh = (has_split && cb < c1) ? (uint32_t)(c1 - cb < KG ? c1 - cb : KG) : 0;
        for (uint32_t k = 0; k < nh; ++k) {
            const uint64_t h = sm[base + k];
            if (h != h_cur) {
                const uint64_t d = h_cur - h;
#pragma unroll
                for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], d, n[j], ninv[j]);
                defA += (u128)d * (32ull * cells + 32 * L);
                nprod += (uint64_t)(63 - __clzll((long long)d)) + __popcll(d);
                h_cur = h;
            }
            const uint32_t q = sq[base + k];
            const bool wide = L != 2 && q >= 0x80000000u;
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
                cell_w<L>(P[j], q, n[j], ninv[j]);
                if (wide) cond_sub_chain(P[j], n[j]);
            }
            ++cells;
        }
    }
    if (h_cur) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], h_cur, n[j], ninv[j]);
        defA += (u128)h_cur * (32ull * cells + 32 * L);
        nprod += (uint64_t)(63 - __clzll((long long)h_cur)) + __popcll(h_cur);
    }
    for (uint32_t k = 0; k < sb; ++k) {               // A^(2^sb)
#pragma unroll
        for (int j = 0; j < RPT; ++j) A[j] = mont_mul<L>(A[j], A[j], n[j], ninv[j]);
        defA = 2 * defA + 32 * L;
    }
    nprod += sb;

    // ---- windows over the low bits, top window first ----
    Res<L> acc[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) set_small<L>(acc[j], 1);
    u128 defacc = 0;
    for (int w = (int)nwin - 1; w >= 0; --w) {
        Res<L> B[SMB ? 1 : RPT][SMB ? 1 : NBK];
        if (SMB) {
#pragma unroll
            for (int d = 0; d < NBK; ++d) sbk[d * 256 + threadIdx.x] = make_uint4(1, 0, 0, 0);
        } else {
#pragma unroll
            for (int j = 0; j < RPT; ++j)
#pragma unroll
                for (int d = 0; d < NBK; ++d) set_small<L>(B[j][d], 1);
        }
        __syncthreads();
        for (uint32_t k = lt; k <= NBK; k += tps) scnt[g][k] = 0;
        for (uint32_t ch = 0; ch < nchunks; ++ch) {
            __syncthreads();
            const uint64_t cb = c0 + (uint64_t)ch * KG;
            const uint32_t nh = (has_split && cb < c1) ? (uint32_t)(c1 - cb < KG ? c1 - cb : KG) : 0;
            if (SORT) {
                for (uint32_t k = lt; k <= NBK; k += tps) scur[g][k] = 0;
                __syncthreads();
            }
            for (uint32_t k = lt; k < KG; k += tps) {
                if (has_split && cb + k < c1) {
                    const uint32_t q = cols[cb + k];
                    const uint32_t dg = (uint32_t)(((legendre(T, q) & lmask) >> (DW * w)) & NBK);
                    sq[base + k] = q;
                    sm[base + k] = dg;
                    atomicAdd(SORT ? &scur[g][dg] : &scnt[g][dg], 1u);
                }
            }
            __syncthreads();
            if (SORT) {
                // exclusive prefix of the digit counts (the scatter cursors), and
                // the deficit of each bucket's run: 32 per cell, 32L for the fold of X
                if (lt == 0) {
                    uint32_t o = 0;
                    for (int d = 0; d <= NBK; ++d) {
                        const uint32_t c = scur[g][d];
                        scur[g][d] = o;
                        o += c;
                        scnt[g][d] += c + (c >= 2 ? (uint32_t)L : 0u);
                    }
                }
                __syncthreads();
                for (uint32_t k = lt; k < nh; k += tps) {
                    const uint32_t dg = (uint32_t)sm[base + k];
                    ss[base + atomicAdd(&scur[g][dg], 1u)] = sq[base + k];
                }
                __syncthreads();
                // after the scatter scur[d] is the end of digit d's run
                Res<L> X[RPT];
#pragma unroll
                for (int j = 0; j < RPT; ++j) set_small<L>(X[j], 1);
#pragma unroll
                for (int d = 1; d <= NBK; ++d) {
                    const uint32_t k0 = scur[g][d - 1], k1 = scur[g][d];
                    nbucket += k1 - k0;
                    nprod += (k1 - k0 >= 2) ? 1u : 0u;
                    if (SMB) {
                        if (k1 == k0) continue;
                        const uint4 v = sbk[(d - 1) * 256 + threadIdx.x];
                        Res<L>& b = B[0][0];
                        b.w[0] = v.x; b.w[1] = v.y;
                        if (L > 2) b.w[2 < L ? 2 : 0] = v.z;
                        if (L > 3) b.w[3 < L ? 3 : 0] = v.w;
                    }
                    uint32_t k = k0;
                    for (; k + 1 < k1; k += 2) {
                        const uint32_t qa = ss[base + k], qb = ss[base + k + 1];
#pragma unroll
                        for (int j = 0; j < RPT; ++j) {
                            cell_w<L>(B[j][SMB ? 0 : d - 1], qa, n[j], ninv[j]);
                            cell_w<L>(X[j], qb, n[j], ninv[j]);
                            if (L != 2 && qa >= 0x80000000u) cond_sub_chain(B[j][SMB ? 0 : d - 1], n[j]);
                            if (L != 2 && qb >= 0x80000000u) cond_sub_chain(X[j], n[j]);
                        }
                    }
                    if (k < k1) {
                        const uint32_t qa = ss[base + k];
#pragma unroll
                        for (int j = 0; j < RPT; ++j) {
                            cell_w<L>(B[j][SMB ? 0 : d - 1], qa, n[j], ninv[j]);
                            if (L != 2 && qa >= 0x80000000u) cond_sub_chain(B[j][SMB ? 0 : d - 1], n[j]);
                        }
                    }
                    if (k1 - k0 >= 2) {
#pragma unroll
                        for (int j = 0; j < RPT; ++j) {
                            B[j][SMB ? 0 : d - 1] = mont_mul<L>(B[j][SMB ? 0 : d - 1], X[j], n[j], ninv[j]);
                            set_small<L>(X[j], 1);
                        }
                    }
                    if (SMB) {
                        const Res<L>& b = B[0][0];
                        sbk[(d - 1) * 256 + threadIdx.x] =
                            make_uint4(b.w[0], b.w[1], L > 2 ? b.w[2 < L ? 2 : 0] : 0, L > 3 ? b.w[3 < L ? 3 : 0] : 0);
                    }
                }
            } else {
                for (uint32_t k = 0; k < nh; ++k) {
                    const uint32_t d = (uint32_t)sm[base + k];
                    const uint32_t q = sq[base + k];
                    if constexpr (!SMB) {
                        if (d) bucket_cell<L, NBK, RPT>(B, d, q, n, ninv, L != 2 && q >= 0x80000000u);
                    }
                    nbucket += d ? 1u : 0u;
                }
            }
        }
        // R = prod_d B_d^d by running products from the top bucket down
        __syncthreads();
        u128 defS = (u128)32 * scnt[g][NBK], defR = defS;
#pragma unroll
        for (int d = NBK - 2; d >= 0; --d) {
            defS += (u128)32 * scnt[g][d + 1] + 32 * L;
            defR += defS + 32 * L;
        }
#pragma unroll
        for (int j = 0; j < RPT; ++j) {
            auto bucket = [&](int d) -> Res<L> {
                if (!SMB) return B[j][SMB ? 0 : d];
                const uint4 v = sbk[d * 256 + threadIdx.x];
                Res<L> b;
                b.w[0] = v.x; b.w[1] = v.y;
                if (L > 2) b.w[2 < L ? 2 : 0] = v.z;
                if (L > 3) b.w[3 < L ? 3 : 0] = v.w;
                return b;
            };
            Res<L> S = bucket(NBK - 1), R = S;
#pragma unroll
            for (int d = NBK - 2; d >= 0; --d) {
                S = mont_mul<L>(S, bucket(d), n[j], ninv[j]);
                R = mont_mul<L>(R, S, n[j], ninv[j]);
            }
            if (w == (int)nwin - 1) {
                acc[j] = R;
            } else {
                for (int k = 0; k < DW; ++k) acc[j] = mont_mul<L>(acc[j], acc[j], n[j], ninv[j]);
                acc[j] = mont_mul<L>(acc[j], R, n[j], ninv[j]);
            }
        }
        if (w == (int)nwin - 1) {
            defacc = defR;
        } else {
            for (int k = 0; k < DW; ++k) defacc = 2 * defacc + 32 * L;
            defacc += defR + 32 * L;
        }
        nprod += 2 * (NBK - 1) + (w == (int)nwin - 1 ? 0 : DW + 1);
    }
    u128 def = defA;
    if (nwin) def = defA + defacc + 32 * L;
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        Res<L> res = A[j];
        if (nwin) res = mont_mul<L>(A[j], acc[j], n[j], ninv[j]);
        if (live[j]) {
            uint4 o;
            o.x = res.w[0];
            o.y = res.w[1];
            o.z = L > 2 ? res.w[2 < L ? 2 : 0] : 0;
            o.w = L > 3 ? res.w[3 < L ? 3 : 0] : 0;
            part[bk.part_base + (uint64_t)s * bk.nrows + it.row0 + lt + j * tps] = o;
        }
    }
    if (has_split && it.row0 == 0 && lt == 0) {
        Deficit dd;
        dd.lo = (uint64_t)def;
        dd.hi = (uint64_t)(def >> 64);
        defs[bk.def_base + s] = dd;
    }
    if (work && has_split && lt == 0) {
        const uint32_t left = bk.nrows > it.row0 ? bk.nrows - it.row0 : 0u;
        const uint64_t rows = left < tps * RPT ? left : tps * RPT;
        if (nwin) ++nprod;                              // A * acc
        atomicAdd(&work[0], (unsigned long long)(cells * rows));
        atomicAdd(&work[1], (unsigned long long)(nbucket * rows));
        atomicAdd(&work[2], (unsigned long long)(nprod * rows));
    }
}

// ===========================================================================
// Consecutive-integer tail: prod_{N = start}^{start+len-1} N  (iterate.cl:30-43)
// ===========================================================================

// Tail item idx belongs to the row r with the largest it_begin <= idx (rows
// with no tail share it_begin with the next row); it covers
// N = T + 1 + k*K .. min(T + (k+1)*K, Tp) with k = idx - it_begin.
__device__ __forceinline__ uint32_t tail_row(const RowInfo* __restrict__ info, uint32_t lo, uint32_t hi, uint32_t idx) {
    // largest r in [lo, hi) with info[r].it_begin <= idx
    while (hi - lo > 1) {
        const uint32_t m = (lo + hi) >> 1;
        if (info[m].it_begin <= idx) lo = m; else hi = m;
    }
    return lo;
}

template <int L>
__global__ void __launch_bounds__(256)
k_iterate(const Bucket* __restrict__ buckets, const RowInfo* __restrict__ info, const RowMod* __restrict__ mods,
          uint32_t row_begin, uint32_t nrows, uint32_t item_begin, uint32_t nitems, uint64_t K, uint4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nitems) return;
    const uint32_t idx = item_begin + i;
    const uint32_t row = tail_row(info, row_begin, row_begin + nrows, idx);
    const RowInfo ri = info[row];
    const uint64_t T = buckets[ri.bucket].T;
    const uint64_t k = idx - ri.it_begin;
    const uint64_t start = T + 1 + k * K;
    const uint64_t rest = ri.Tp - T - k * K;
    const uint32_t len = (uint32_t)(rest < K ? rest : K);
    const RowMod m = mods[row];
    uint32_t n[L];
#pragma unroll
    for (int q = 0; q < L; ++q) n[q] = m.n[q];
    Res<L> acc;
    set_small<L>(acc, 1);
    const uint64_t last = start + len - 1;
    if (last < 0x80000000ull) {
        uint32_t N = (uint32_t)start;
        uint32_t j = 0;
        for (; j + 4 <= len; j += 4, N += 4) {
            cell_w<L>(acc, N, n, m.ninv);
            cell_w<L>(acc, N + 1, n, m.ninv);
            cell_w<L>(acc, N + 2, n, m.ninv);
            cell_w<L>(acc, N + 3, n, m.ninv);
        }
        for (; j < len; ++j, ++N) cell_w<L>(acc, N, n, m.ninv);
    } else {
        uint64_t N = start;
        for (uint32_t j = 0; j < len; ++j, ++N) cell64<L>(acc, N, n, m.ninv);
    }
    uint4 o;
    o.x = acc.w[0];
    o.y = acc.w[1];
    o.z = L > 2 ? acc.w[2 < L ? 2 : 0] : 0;
    o.w = L > 3 ? acc.w[3 < L ? 3 : 0] : 0;
    out[idx] = o;
}

// ===========================================================================
// Finish: combine the split partials and the tail, restore the tracked
// power of two, and (full search) lift T_p! to (p-1)! with the class formula
// (cl_wilson.cpp:731-870), add 1, and split into rem + p*quot.
// ===========================================================================

// digits of v < p^2 in base p: v = d0 + p*d1
template <int L>
__device__ void digits_base_p(const Res<L>& v, uint64_t p, uint64_t* d0, uint64_t* d1) {
    // remainder by bit-serial long division (runs once per row)
    uint64_t r = 0;
    for (int i = 32 * L - 1; i >= 0; --i) {
        const uint32_t bitv = (v.w[i >> 5] >> (i & 31)) & 1u;
        // r < p < 2^62, so 2r + 1 fits
        r = (r << 1) | bitv;
        if (r >= p) r -= p;
    }
    // exact quotient (v - r) / p modulo 2^64; the true quotient is < p < 2^64
    uint64_t vlo = (uint64_t)v.w[0] | ((uint64_t)v.w[1] << 32);
    const uint64_t pinv = inv64(p);
    *d0 = r;
    *d1 = (vlo - r) * pinv;
}

// Cornacchia: x^2 + d*y^2 = p given r0^2 = -d (mod p)
__device__ bool cornacchia(uint64_t p, uint64_t d, uint64_t r0, uint64_t* x, uint64_t* y) {
    if (r0 <= p / 2) r0 = p - r0;
    uint64_t a = p, b = r0;
    const uint64_t lim = isqrt64(p);
    while (b > lim) { uint64_t t = a % b; a = b; b = t; }
    const uint64_t rest = p - b * b;
    if (rest % d) return false;
    const uint64_t yy = rest / d, yr = isqrt64(yy);
    if (yr * yr != yy) return false;
    *x = b;
    *y = yr;
    return true;
}

// The search for a non-residue g (quadratic for find_a, cubic for find_cu)
// runs to this bound, then reports "no representation".  Under the
// generalised Riemann hypothesis the least non-residue of either kind is
// below 3 (ln p)^2 < 6,000 for p < 2^62 (Bach's explicit bound); among the
// primes below 1e8 the largest least cubic non-residue is 41 (p = 65139031).
// For type 1 (p = 5 mod 12) the quadratic search ends at g = 2 or 3, since
// (3/p) = (p/3) = -1 there.
constexpr uint64_t NONRESIDUE_LIMIT = 1ull << 16;

// a with p = a^2 + b^2 (a odd, sign a = 1 mod 4: find.cl:52-58, only a^2 is used)
__device__ bool find_a(uint64_t p, int64_t* out) {
    Mod64 M;
    M.init(p);
    const uint64_t minus1 = p - 1;
    for (uint64_t g = 2; g < NONRESIDUE_LIMIT && g < p; ++g) {
        if (M.from(M.pow(M.to(g), (p - 1) / 2)) != minus1) continue;
        const uint64_t r = M.from(M.pow(M.to(g), (p - 1) / 4));
        uint64_t x, y;
        if (!cornacchia(p, 1, r, &x, &y)) return false;
        const uint64_t a = (x & 1) ? x : y;
        *out = (a % 4 == 3) ? -(int64_t)a : (int64_t)a;
        return true;
    }
    return false;
}

// c with 4p = c^2 + 27d^2 (c = 1 mod 3) and u with 4p = u^2 + 3v^2 (u = umod mod 3),
// the sign rules of find.cl:77-83, 101-107 and cl_wilson.cpp:634
__device__ bool find_cu(uint64_t p, int64_t* c_out, int64_t* u_out) {
    Mod64 M;
    M.init(p);
    for (uint64_t g = 2; g < NONRESIDUE_LIMIT && g < p; ++g) {
        const uint64_t w = M.from(M.pow(M.to(g), (p - 1) / 3));
        if (w == 1) continue;
        const uint64_t r = (2 * w + 1) % p;            // sqrt(-3) mod p
        uint64_t x, y;
        if (!cornacchia(p, 3, r, &x, &y)) return false;
        const int64_t X = (int64_t)x, Y = (int64_t)y;
        const int64_t us[3] = { 2 * X, X + 3 * Y, X - 3 * Y };
        const int64_t vs[3] = { 2 * Y, X - Y, X + Y };
        const uint32_t umod = (((p - 1) / 6) % 2 == 0) ? 1 : 2;
        const uint64_t u = (uint64_t)(us[0] < 0 ? -us[0] : us[0]);
        *u_out = (u % 3 == umod) ? (int64_t)u : -(int64_t)u;
        for (int k = 0; k < 3; ++k) {
            const int64_t v = vs[k] < 0 ? -vs[k] : vs[k];
            if (v % 3 == 0) {
                const uint64_t c = (uint64_t)(us[k] < 0 ? -us[k] : us[k]);
                *c_out = (c % 3 == 2) ? -(int64_t)c : (int64_t)c;
                return true;
            }
        }
        return false;
    }
    return false;
}

template <int L>
__device__ __forceinline__ Res<L> mont_of_signed(int64_t v, const Res<L>& R2, const uint32_t* n, uint32_t ninv) {
    Res<L> x;
    set_small<L>(x, (uint64_t)(v < 0 ? -v : v));
    x = mont_mul<L>(x, R2, n, ninv);
    if (v < 0) {
        Res<L> z;
        set_small<L>(z, 0);
        x = sub_mod2n<L>(z, x, n);
    }
    return x;
}

template <int L>
__global__ void __launch_bounds__(128)
k_finish(const Bucket* __restrict__ buckets, const RowInfo* __restrict__ info, const RowMod* __restrict__ mods,
         const uint4* __restrict__ part, const Deficit* __restrict__ defs, uint64_t K,
         const uint4* __restrict__ ipart, uint32_t row_begin, uint32_t nrows, int full,
         RowOut* __restrict__ out, const uint4* __restrict__ acc1, const Deficit* __restrict__ def1,
         const uint4* __restrict__ acc2, const Deficit* __restrict__ def2, int merged) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const uint32_t row = row_begin + i;
    const RowInfo ri = info[row];
    const Bucket bk = buckets[ri.bucket];
    const RowMod m = mods[row];
    uint32_t n[L];
#pragma unroll
    for (int k = 0; k < L; ++k) n[k] = m.n[k];
    const uint32_t ninv = m.ninv;
    const uint32_t rl = row - bk.row_begin;

    // combine split partials
    Res<L> X;
    set_small<L>(X, 1);
    u128 def = 0;
    for (uint32_t s = 0; s < (merged ? 0u : bk.nsplit); ++s) {
        const uint4 v = part[bk.part_base + (uint64_t)s * bk.nrows + rl];
        Res<L> y;
        y.w[0] = v.x; y.w[1] = v.y;
        if (L > 2) y.w[2 < L ? 2 : 0] = v.z;
        if (L > 3) y.w[3 < L ? 3 : 0] = v.w;
        X = mont_mul<L>(X, y, n, ninv);
        const Deficit d = defs[bk.def_base + s];
        def += ((u128)d.hi << 64 | d.lo) + 32 * L;
    }
    // the consecutive-integer tail
    for (uint32_t k = 0; k < ri.it_count; ++k) {
        const uint32_t idx = ri.it_begin + k;
        const uint4 v = ipart[idx];
        const uint64_t start = bk.T + 1 + (uint64_t)k * K;
        const uint64_t rest = ri.Tp - bk.T - (uint64_t)k * K;
        const uint64_t len = rest < K ? rest : K;
        Res<L> y;
        y.w[0] = v.x; y.w[1] = v.y;
        if (L > 2) y.w[2 < L ? 2 : 0] = v.z;
        if (L > 3) y.w[3 < L ? 3 : 0] = v.w;
        X = mont_mul<L>(X, y, n, ninv);
        const bool small = start + len - 1 < 0x80000000ull;
        def += (u128)len * (small ? 32 : 64) + 32 * L;
    }
    // split partials merged into per-row accumulators (k_merge*): columns
    // below 2^32 and, when used, the windows above
    for (int a = 0; a < 2; ++a) {
        const uint4* acc = a ? acc2 : acc1;
        const Deficit* dd = a ? def2 : def1;
        if (!acc) continue;
        const uint4 v = acc[row];
        Res<L> y;
        y.w[0] = v.x; y.w[1] = v.y;
        if (L > 2) y.w[2 < L ? 2 : 0] = v.z;
        if (L > 3) y.w[3 < L ? 3 : 0] = v.w;
        X = mont_mul<L>(X, y, n, ninv);
        const Deficit d = dd[ri.bucket];
        def += (((u128)d.hi << 64) | d.lo) + 32 * L;
    }
    // R mod n (Montgomery one), 2R mod n, R^2 mod n by doubling
    Res<L> one;
    set_small<L>(one, 1);
    for (int k = 0; k < 32 * L; ++k) dbl_mod<L>(one, n);
    Res<L> two = one;
    dbl_mod<L>(two, n);
    Res<L> R2 = one;
    for (int k = 0; k < 32 * L; ++k) dbl_mod<L>(R2, n);
    // X * 2^def: multiply by Mont(2^def) = (2R)^def in the Montgomery domain
    const Res<L> Z = mont_pow<L>(two, def, one, n, ninv);
    Res<L> V = mont_mul<L>(X, Z, n, ninv);
    reduce_full<L>(V, n);                                   // V = value mod n

    RowOut o;
    o.pad = 0;
    digits_base_p<L>(V, ri.p, &o.s0, &o.s1);
    o.rem = 0;
    o.quot = 0;
    o.status = 0;
    if (full) {
        const uint64_t p = ri.p;
        const Res<L> M = mont_mul<L>(V, R2, n, ninv);     // Montgomery form of T_p!
        Res<L> mp;
        set_small<L>(mp, p);
        mp = mont_mul<L>(mp, R2, n, ninv);
        const Res<L> two_p = mont_pow<L>(two, (u128)p, one, n, ninv);   // 2^p
        Res<L> W;
        bool ok = true;
        if (ri.type == 0) {
            int64_t cc = 0, uu = 0;
            ok = find_cu(p, &cc, &uu);
            const Res<L> mu = mont_of_signed<L>(uu, R2, n, ninv);
            const Res<L> mc = mont_of_signed<L>(cc, R2, n, ninv);
            W = mont_pow<L>(M, 6, one, n, ninv);                           // T!^6
            Res<L> a = sub_mod2n<L>(two_p, one, n);                         // 2^p - 1
            Res<L> u3 = mont_mul<L>(mont_mul<L>(mu, mu, n, ninv), mu, n, ninv);
            Res<L> z;
            set_small<L>(z, 0);
            Res<L> b = sub_mod2n<L>(z, u3, n);                              // -u^3
            a = mont_mul<L>(b, a, n, ninv);
            Res<L> three;
            set_small<L>(three, 3);
            three = mont_mul<L>(three, R2, n, ninv);
            b = mont_mul<L>(three, mont_mul<L>(mp, mu, n, ninv), n, ninv);  // 3pu
            a = add_mod2n<L>(a, b, n);
            W = mont_mul<L>(W, a, n, ninv);
            // p/c - c with c^-1 = c^(p(p-1)-1) mod p^2
            const u128 einv = (u128)p * (p - 1) - 1;
            const Res<L> ci = mont_pow<L>(mc, einv, one, n, ninv);
            a = sub_mod2n<L>(mont_mul<L>(mp, ci, n, ninv), mc, n);
            W = mont_mul<L>(W, a, n, ninv);
            // (3^p - 1)/2
            a = sub_mod2n<L>(mont_pow<L>(three, (u128)p, one, n, ninv), one, n);
            const Res<L> two_inv = mont_pow<L>(two, einv, one, n, ninv);
            a = mont_mul<L>(a, two_inv, n, ninv);
            W = mont_mul<L>(W, a, n, ninv);
        } else if (ri.type == 1) {
            int64_t aa = 0;
            ok = find_a(p, &aa);
            const Res<L> ma = mont_of_signed<L>(aa, R2, n, ninv);
            W = mont_pow<L>(M, 4, one, n, ninv);                           // T!^4
            Res<L> three, four;
            set_small<L>(three, 3);
            set_small<L>(four, 4);
            three = mont_mul<L>(three, R2, n, ninv);
            four = mont_mul<L>(four, R2, n, ninv);
            Res<L> a = sub_mod2n<L>(mont_mul<L>(three, two_p, n, ninv), four, n);   // 3*2^p - 4
            W = mont_mul<L>(W, a, n, ninv);
            a = sub_mod2n<L>(mont_mul<L>(two, mont_mul<L>(ma, ma, n, ninv), n, ninv), mp, n);  // 2a^2 - p
            W = mont_mul<L>(W, a, n, ninv);
        } else {
            W = mont_mul<L>(M, M, n, ninv);                                 // T!^2
            W = mont_mul<L>(W, sub_mod2n<L>(one, two_p, n), n, ninv);      // (1 - 2^p)
        }
        Res<L> rawone;
        set_small<L>(rawone, 1);
        Res<L> Wv = mont_mul<L>(W, rawone, n, ninv);                       // out of Montgomery form
        reduce_full<L>(Wv, n);
        // + 1 mod n
        add_limbs<L>(Wv, rawone.w);
        if (geq<L>(Wv, n)) sub_limbs<L>(Wv, n);
        uint64_t rem, quot;
        digits_base_p<L>(Wv, p, &rem, &quot);
        o.rem = rem;
        o.quot = quot;
        if (!ok) o.status = 2;              // representation not found
        else if (rem != 0) o.status = 1;    // Wilson quotient check failed
    }
    out[row] = o;
}

// ===========================================================================
// Row-wise product of partial column products.  When the column interval of
// one range is split between GPUs, each returns per-row partial products as
// values s0 + p*s1 < p^2; their product is the running product over the union
// of the pieces (the role of reduce.cl:11-44, which folds work-group partials
// into a residue, one level up).  parts[k * 2n + 2i + {0, 1}] = digits of row
// i's k-th partial; out[2i + {0, 1}] = digits of the product.
// ===========================================================================

template <int L>
__device__ void rows_product_one(uint64_t p, const uint64_t* __restrict__ parts, uint64_t n_rows, uint32_t nparts,
                                 uint64_t i, uint64_t* d0, uint64_t* d1) {
    const u128 nn = (u128)p * p;
    uint32_t n[L];
#pragma unroll
    for (int k = 0; k < L; ++k) n[k] = k < 4 ? (uint32_t)(nn >> (32 * k)) : 0u;
    uint32_t x = n[0];                  // n^-1 mod 2^32 by Newton
    for (int k = 0; k < 5; ++k) x *= 2u - n[0] * x;
    const uint32_t ninv = 0u - x;
    Res<L> R2;                          // R^2 mod n by doubling 1 (64L times)
    set_small<L>(R2, 1);
    for (int k = 0; k < 64 * L; ++k) dbl_mod<L>(R2, n);
    Res<L> X;                           // running product, Montgomery form
    for (uint32_t k = 0; k < nparts; ++k) {
        const uint64_t* d = parts + (uint64_t)k * 2 * n_rows + 2 * i;
        const u128 v = (u128)d[1] * p + d[0];
        Res<L> y;
#pragma unroll
        for (int w = 0; w < L; ++w) y.w[w] = w < 4 ? (uint32_t)(v >> (32 * w)) : 0u;
        y = mont_mul<L>(y, R2, n, ninv);                  // v * R
        X = k ? mont_mul<L>(X, y, n, ninv) : y;
    }
    Res<L> one;
    set_small<L>(one, 1);
    Res<L> V = mont_mul<L>(X, one, n, ninv);               // out of Montgomery form
    reduce_full<L>(V, n);
    digits_base_p<L>(V, p, d0, d1);
}

__global__ void __launch_bounds__(128)
k_rows_product(const uint64_t* __restrict__ ps, uint64_t n_rows, const uint64_t* __restrict__ parts, uint32_t nparts,
               uint64_t* __restrict__ out) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows) return;
    const uint64_t p = ps[i];
    uint64_t d0, d1;
    if (p < (1ull << 31)) rows_product_one<2>(p, parts, n_rows, nparts, i, &d0, &d1);
    else if (p < (1ull << 47)) rows_product_one<3>(p, parts, n_rows, nparts, i, &d0, &d1);
    else rows_product_one<4>(p, parts, n_rows, nparts, i, &d0, &d1);
    out[2 * i] = d0;
    out[2 * i + 1] = d1;
}

// ===========================================================================
// Columns above 2^32.  A window [lo, hi) is sieved by CTAs that each own
// `spc` consecutive segments of BIG_SPAN integers.  Odd primes 3..61 are
// removed by OR-ing precomputed 32-bit masks (one table per prime, indexed by
// the residue of the word's first number); every larger sieving prime keeps
// its next bit offset in global memory between the CTA's segments, so its
// starting point is divided out only once per CTA.
// ===========================================================================

constexpr uint32_t BIG_THREADS = 1024;
__constant__ uint32_t c_pre[BIG_PRESIEVE] = { 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53, 59, 61 };
__constant__ uint32_t c_preoff[BIG_PRESIEVE] = { 0, 3, 8, 15, 26, 39, 56, 75, 98, 127, 158, 195, 236, 279, 326, 379, 438 };
constexpr uint32_t PRE_TABLE = 499;          // 3 + 5 + ... + 61
constexpr uint32_t OFF_NONE = 0xFFFFFFFFu;   // prime does not reach this CTA's range

__global__ void __launch_bounds__(BIG_THREADS)
k_sieve_big(uint64_t lo, uint64_t hi, uint32_t nseg, uint32_t spc, const uint32_t* __restrict__ base, uint32_t nbase,
            uint32_t ncoop, uint32_t* __restrict__ offs, uint32_t* __restrict__ bitmap, uint32_t* __restrict__ seg_count) {
    extern __shared__ uint32_t smem[];
    uint32_t* bm = smem;                  // BIG_WORDS words
    uint32_t* tab = smem + BIG_WORDS;     // PRE_TABLE masks
    __shared__ uint32_t wsum[BIG_THREADS / 32];
    __shared__ uint32_t sres[BIG_PRESIEVE], sinc[BIG_PRESIEVE];
    __shared__ uint32_t s_coop[2][160];
    if (threadIdx.x < BIG_PRESIEVE) sinc[threadIdx.x] = (64u * blockDim.x) % c_pre[threadIdx.x];
    for (uint32_t i = threadIdx.x; i < PRE_TABLE; i += blockDim.x) {
        uint32_t j = 0;
        while (j + 1 < BIG_PRESIEVE && c_preoff[j + 1] <= i) ++j;
        const uint32_t p = c_pre[j], r = i - c_preoff[j];
        uint32_t m = 0;
        for (uint32_t b = 0; b < 32; ++b)
            if ((r + 2 * b) % p == 0) m |= 1u << b;    // number = (r mod p) + 2b
        tab[i] = m;
    }
    const uint32_t seg0 = blockIdx.x * spc;
    const uint64_t cta_lo = lo + (uint64_t)seg0 * BIG_SPAN;
    const uint64_t range_bits = (uint64_t)spc * BIG_BITS;
    uint32_t* off = offs + (uint64_t)blockIdx.x * nbase;
    for (uint32_t k = threadIdx.x; k < nbase; k += blockDim.x) {
        const uint64_t p = base[k];
        uint64_t m = (cta_lo + p - 1) / p * p;
        if (m < p * p) m = p * p;
        if (!(m & 1)) m += p;
        const uint64_t o = (m - cta_lo - 1) / 2;       // number = cta_lo + 2o + 1
        off[k] = o < range_bits ? (uint32_t)o : OFF_NONE;
        if (k < ncoop) s_coop[0][k] = off[k];
    }
    __syncthreads();
    uint32_t cur = 0;
    for (uint32_t j = 0; j < spc; ++j) {
        const uint32_t seg = seg0 + j;
        if (seg >= nseg) break;                          // uniform across the CTA
        const uint64_t slo = cta_lo + (uint64_t)j * BIG_SPAN;
        // residues of the thread's first word start, then stepped by
        // blockDim.x words (64 * blockDim.x integers) with an add and a subtract
        if (threadIdx.x < BIG_PRESIEVE) sres[threadIdx.x] = (uint32_t)(slo % c_pre[threadIdx.x]);
        __syncthreads();
        uint32_t rr[BIG_PRESIEVE];
#pragma unroll
        for (uint32_t q = 0; q < BIG_PRESIEVE; ++q) {
            const uint32_t p = c_pre[q];
            rr[q] = (sres[q] + (64u * threadIdx.x + 1u) % p) % p;
        }
        for (uint32_t w = threadIdx.x; w < BIG_WORDS; w += blockDim.x) {
            uint32_t word = 0;
#pragma unroll
            for (uint32_t q = 0; q < BIG_PRESIEVE; ++q) {
                word |= tab[c_preoff[q] + rr[q]];
                rr[q] += sinc[q];
                if (rr[q] >= c_pre[q]) rr[q] -= c_pre[q];
            }
            bm[w] = word;
        }
        __syncthreads();
        // primes below 1024: all threads stride over one prime's multiples; the
        // offsets live in shared memory, read from one half and the next
        // segment's written to the other
        for (uint32_t k = 0; k < ncoop; ++k) {
            const uint32_t o = s_coop[cur][k];
            if (o == OFF_NONE) continue;
            const uint32_t p = base[k];
            for (uint32_t i = o + threadIdx.x * p; i < BIG_BITS; i += blockDim.x * p)
                atomicOr(&bm[i >> 5], 1u << (i & 31));
            if (threadIdx.x == 0) s_coop[cur ^ 1][k] = o + ((BIG_BITS - 1 - o) / p + 1) * p - BIG_BITS;
        }
        // larger primes: one per thread, offsets carried to the next segment
        for (uint32_t k = ncoop + threadIdx.x; k < nbase; k += blockDim.x) {
            uint32_t o = off[k];
            if (o == OFF_NONE) continue;
            const uint32_t p = base[k];
            for (; o < BIG_BITS; o += p) atomicOr(&bm[o >> 5], 1u << (o & 31));
            off[k] = o - BIG_BITS;
        }
        __syncthreads();
        uint32_t cnt = 0;
        for (uint32_t w = threadIdx.x; w < BIG_WORDS; w += blockDim.x) {
            uint32_t pb = ~bm[w];
            const uint64_t first = slo + 64ull * w + 1;
            if (first + 62 >= hi) {
                uint32_t keep = 0;
                for (uint32_t b = 0; b < 32; ++b)
                    if (first + 2ull * b < hi) keep |= 1u << b;
                pb &= keep;
            }
            bitmap[(uint64_t)seg * BIG_WORDS + w] = pb;
            cnt += __popc(pb);
        }
        for (int o2 = 16; o2 > 0; o2 >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o2);
        if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t t = 0;
            for (uint32_t i = 0; i < blockDim.x / 32; ++i) t += wsum[i];
            seg_count[seg] = t;
        }
        __syncthreads();
        cur ^= 1;
    }
}

// ordered u64 write-out of a big window's bitmap (segment s: odd numbers lo0 + s*BIG_SPAN + 2i + 1)
__global__ void __launch_bounds__(1024)
k_compact_big(uint64_t lo0, const uint32_t* __restrict__ bitmap, const uint64_t* __restrict__ offsets,
              uint64_t* __restrict__ out) {
    __shared__ uint32_t wsum[32];
    constexpr uint32_t WPT = BIG_WORDS / 1024;
    const uint32_t seg = blockIdx.x;
    const uint32_t* bm = bitmap + (uint64_t)seg * BIG_WORDS + threadIdx.x * WPT;
    uint32_t cnt = 0;
    for (uint32_t i = 0; i < WPT; ++i) cnt += __popc(bm[i]);
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += v;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (uint32_t i = 0; i < wid; ++i) wbase += wsum[i];
    uint64_t pos = offsets[seg] + wbase + incl - cnt;
    const uint64_t lo = lo0 + (uint64_t)seg * BIG_SPAN;
    for (uint32_t i = 0; i < WPT; ++i) {
        uint32_t w = bm[i];
        const uint64_t base_n = lo + (uint64_t)(threadIdx.x * WPT + i) * 64 + 1;
        while (w) {
            const int b = __ffs(w) - 1;
            w &= w - 1;
            out[pos++] = base_n + 2ull * b;
        }
    }
}

__global__ void k_count_leq64(const uint64_t* __restrict__ cols, uint64_t ncols, const uint64_t* __restrict__ keys,
                              uint32_t nkeys, uint64_t* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nkeys) return;
    const uint64_t key = keys[i];
    uint64_t a = 0, b = ncols;
    while (a < b) {
        const uint64_t m = (a + b) >> 1;
        if (cols[m] <= key) a = m + 1; else b = m;
    }
    out[i] = a;
}

// Sweep over 64-bit columns q > 2^32 > sqrt(T): exponent floor(T/q), prefix
// folding as in k_sweep, each cell a two-round 64-bit Montgomery step.
template <int L, int RPT>
__global__ void __launch_bounds__(256)
k_sweep64(const Bucket* __restrict__ buckets, const SweepItem* __restrict__ items, const RowMod* __restrict__ mods,
          const uint64_t* __restrict__ cols, uint4* __restrict__ part, Deficit* __restrict__ defs) {
    const SweepItem it = items[blockIdx.x];
    if (threadIdx.x >= (256 / it.tps) * it.tps) return;   // lanes past the CTA's last whole group
    const Bucket bk = buckets[it.bucket];
    const uint32_t s = it.split0 + threadIdx.x / it.tps;
    if (s >= bk.nsplit) return;
    const uint32_t rl = it.row0 + threadIdx.x % it.tps;
    uint32_t n[RPT][L];
    uint32_t ninv[RPT];
    bool live[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        const uint32_t r = rl + j * it.tps;
        live[j] = r < bk.nrows;
        const RowMod m = mods[bk.row_begin + (live[j] ? r : 0)];
#pragma unroll
        for (int k = 0; k < L; ++k) n[j][k] = m.n[k];
        ninv[j] = m.ninv;
    }
    const uint64_t T = bk.T;
    uint64_t c0, c1;
    split_range(bk, s, &c0, &c1);
    Res<L> P[RPT], A[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) { set_small<L>(P[j], 1); set_small<L>(A[j], 1); }
    u128 def = 0;
    if (c0 < c1) {
        uint64_t e_cur = T / cols[c0];
        uint64_t thr = T / e_cur;
        uint64_t cells = 0;
        const uint64_t* cp = cols + c0;
        const uint64_t* const ce = cols + c1;
        while (cp < ce) {
            if ((((uintptr_t)cp) & 31) == 0 && cp + 4 <= ce) {
                const ulonglong2 g0 = __ldg(reinterpret_cast<const ulonglong2*>(cp));
                const ulonglong2 g1 = __ldg(reinterpret_cast<const ulonglong2*>(cp) + 1);
                if (g1.y <= thr) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) {
                        cell64<L>(P[j], g0.x, n[j], ninv[j]);
                        cell64<L>(P[j], g0.y, n[j], ninv[j]);
                        cell64<L>(P[j], g1.x, n[j], ninv[j]);
                        cell64<L>(P[j], g1.y, n[j], ninv[j]);
                    }
                    cp += 4;
                    cells += 4;
                    continue;
                }
            }
            const uint64_t q = __ldg(cp);
            if (q > thr) {
                const uint64_t e_new = T / q;
                const uint64_t d = e_cur - e_new;
                if (d) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], d, n[j], ninv[j]);
                    def += (u128)d * (64 * cells + 32 * L);
                }
                e_cur = e_new;
                thr = T / e_new;
            }
#pragma unroll
            for (int j = 0; j < RPT; ++j) cell64<L>(P[j], q, n[j], ninv[j]);
            ++cp;
            ++cells;
        }
#pragma unroll
        for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], e_cur, n[j], ninv[j]);
        def += (u128)e_cur * (64 * cells + 32 * L);
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        if (!live[j]) continue;
        const uint32_t r = rl + j * it.tps;
        uint4 o;
        o.x = A[j].w[0];
        o.y = A[j].w[1];
        o.z = L > 2 ? A[j].w[2 < L ? 2 : 0] : 0;
        o.w = L > 3 ? A[j].w[3 < L ? 3 : 0] : 0;
        part[bk.part_base + (uint64_t)s * bk.nrows + r] = o;
    }
    if (it.row0 == 0 && threadIdx.x % it.tps == 0) {
        Deficit dd;
        dd.lo = (uint64_t)def;
        dd.hi = (uint64_t)(def >> 64);
        defs[bk.def_base + s] = dd;
    }
}

// Sweep straight from a window's sieve bitmap: word w holds the odd numbers
// lo + 64w + 1 + 2b (bit b).  Bucket fields for the window: ncols = words used,
// split s = words [ncols*s/nsplit, ncols*(s+1)/nsplit); primes above `key`
// (the bucket's target or q_cap - 1) are skipped.  Otherwise as k_sweep64.
// With los (serving, where buckets sit at different places of the number
// line), each bucket has its own bitmap region: words from Bucket::cbase on,
// word w of the region holding los[bucket] + 64w + 1 + 2b.
template <int L, int RPT>
__global__ void __launch_bounds__(256)
k_sweep_bits(const Bucket* __restrict__ buckets, const SweepItem* __restrict__ items, const RowMod* __restrict__ mods,
             const uint32_t* __restrict__ bitmap, uint64_t lo, const uint64_t* __restrict__ keys,
             uint4* __restrict__ part, Deficit* __restrict__ defs, const uint64_t* __restrict__ los) {
    const SweepItem it = items[blockIdx.x];
    if (threadIdx.x >= (256 / it.tps) * it.tps) return;   // lanes past the CTA's last whole group
    const Bucket bk = buckets[it.bucket];
    const uint32_t s = it.split0 + threadIdx.x / it.tps;
    if (s >= bk.nsplit) return;
    const uint32_t rl = it.row0 + threadIdx.x % it.tps;
    uint32_t n[RPT][L];
    uint32_t ninv[RPT];
    bool live[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        const uint32_t r = rl + j * it.tps;
        live[j] = r < bk.nrows;
        const RowMod m = mods[bk.row_begin + (live[j] ? r : 0)];
#pragma unroll
        for (int k = 0; k < L; ++k) n[j][k] = m.n[k];
        ninv[j] = m.ninv;
    }
    const uint64_t T = bk.T, key = keys[it.bucket];
    const uint64_t w0 = (uint64_t)bk.ncols * s / bk.nsplit;
    const uint64_t w1 = (uint64_t)bk.ncols * (s + 1) / bk.nsplit;
    if (los) {
        lo = los[it.bucket];
        bitmap += bk.cbase;
    }
    Res<L> P[RPT], A[RPT];
#pragma unroll
    for (int j = 0; j < RPT; ++j) { set_small<L>(P[j], 1); set_small<L>(A[j], 1); }
    u128 def = 0;
    uint64_t e_cur = 0, thr = 0, cells = 0;
    bool started = false;
    for (uint64_t w = w0; w < w1; ++w) {
        uint32_t word = __ldg(bitmap + w);
        const uint64_t qb = lo + 64 * w + 1;
        while (word) {
            const int b = __ffs(word) - 1;
            word &= word - 1;
            const uint64_t q = qb + 2ull * b;
            if (q > key) { w = w1; break; }
            if (!started) {
                started = true;
                e_cur = T / q;
                thr = T / e_cur;
            } else if (q > thr) {
                const uint64_t e_new = T / q;
                const uint64_t d = e_cur - e_new;
                if (d) {
#pragma unroll
                    for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], d, n[j], ninv[j]);
                    def += (u128)d * (64 * cells + 32 * L);
                }
                e_cur = e_new;
                thr = T / e_new;
            }
#pragma unroll
            for (int j = 0; j < RPT; ++j) cell64<L>(P[j], q, n[j], ninv[j]);
            ++cells;
        }
    }
    if (started) {
#pragma unroll
        for (int j = 0; j < RPT; ++j) fold_pow<L>(A[j], P[j], e_cur, n[j], ninv[j]);
        def += (u128)e_cur * (64 * cells + 32 * L);
    }
#pragma unroll
    for (int j = 0; j < RPT; ++j) {
        if (!live[j]) continue;
        const uint32_t r = rl + j * it.tps;
        uint4 o;
        o.x = A[j].w[0];
        o.y = A[j].w[1];
        o.z = L > 2 ? A[j].w[2 < L ? 2 : 0] : 0;
        o.w = L > 3 ? A[j].w[3 < L ? 3 : 0] : 0;
        part[bk.part_base + (uint64_t)s * bk.nrows + r] = o;
    }
    if (it.row0 == 0 && threadIdx.x % it.tps == 0) {
        Deficit dd;
        dd.lo = (uint64_t)def;
        dd.hi = (uint64_t)(def >> 64);
        defs[bk.def_base + s] = dd;
    }
}

// number of set bits of a window bitmap standing for numbers <= key
__global__ void k_count_bits(const uint32_t* __restrict__ bitmap, uint64_t lo, uint64_t nwords, uint64_t key,
                             unsigned long long* __restrict__ out) {
    uint32_t c = 0;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t first = lo + 64 * w + 1;
        if (first > key) continue;
        uint32_t word = bitmap[w];
        if (first + 62 > key) {
            const uint32_t keep_bits = (uint32_t)((key - first) / 2 + 1);   // bits 0 .. keep_bits-1
            word &= keep_bits >= 32 ? ~0u : ((1u << keep_bits) - 1);
        }
        c += __popc(word);
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

// Clear the bits of integers below q_lo in a window bitmap (bit b of word w is
// the odd integer lo + 64w + 1 + 2b): a search that resumes at q_lo takes
// only the columns from there on.
__global__ void k_clear_below(uint32_t* __restrict__ bitmap, uint64_t lo, uint64_t q_lo, uint64_t nwords) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nwords) return;
    const uint64_t first = lo + 64 * w + 1;
    if (first >= q_lo) return;
    const uint64_t below = (q_lo - first + 1) / 2;           // bits 0 .. below-1 are < q_lo
    bitmap[w] &= below >= 32 ? 0u : ~((1u << below) - 1u);
}

// acc[row] *= prod over the window's splits; the bucket's first row also
// adds the splits' deficits (and 2^(32L) per product) into bdef[bucket]
template <int L>
__global__ void __launch_bounds__(128)
k_merge(const Bucket* __restrict__ buckets, const RowInfo* __restrict__ info, const RowMod* __restrict__ mods,
        const uint4* __restrict__ part, const Deficit* __restrict__ defs, uint32_t row_begin, uint32_t nrows,
        uint4* __restrict__ acc, Deficit* __restrict__ bdef) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const uint32_t row = row_begin + i;
    const uint32_t b = info[row].bucket;
    const Bucket bk = buckets[b];
    // buckets without splits in this launch, other limb widths, and rows that
    // are not (or no longer) in the bucket's row range are left alone
    if (bk.nsplit == 0 || bk.L != (uint32_t)L || row - bk.row_begin >= bk.nrows) return;
    const RowMod m = mods[row];
    uint32_t n[L];
#pragma unroll
    for (int k = 0; k < L; ++k) n[k] = m.n[k];
    const uint32_t rl = row - bk.row_begin;
    const uint4 a = acc[row];
    Res<L> X;
    X.w[0] = a.x; X.w[1] = a.y;
    if (L > 2) X.w[2 < L ? 2 : 0] = a.z;
    if (L > 3) X.w[3 < L ? 3 : 0] = a.w;
    for (uint32_t s = 0; s < bk.nsplit; ++s) {
        const uint4 v = part[bk.part_base + (uint64_t)s * bk.nrows + rl];
        Res<L> y;
        y.w[0] = v.x; y.w[1] = v.y;
        if (L > 2) y.w[2 < L ? 2 : 0] = v.z;
        if (L > 3) y.w[3 < L ? 3 : 0] = v.w;
        X = mont_mul<L>(X, y, n, m.ninv);
    }
    uint4 o;
    o.x = X.w[0];
    o.y = X.w[1];
    o.z = L > 2 ? X.w[2 < L ? 2 : 0] : 0;
    o.w = L > 3 ? X.w[3 < L ? 3 : 0] : 0;
    acc[row] = o;
    if (rl == 0) {
        u128 d = ((u128)bdef[b].hi << 64) | bdef[b].lo;
        for (uint32_t s = 0; s < bk.nsplit; ++s) {
            const Deficit x = defs[bk.def_base + s];
            d += (((u128)x.hi << 64) | x.lo) + 32 * L;
        }
        bdef[b].lo = (uint64_t)d;
        bdef[b].hi = (uint64_t)(d >> 64);
    }
}

__global__ void k_acc_init(uint32_t nrows, uint32_t nbuckets, uint4* __restrict__ acc, Deficit* __restrict__ bdef) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nrows) acc[i] = make_uint4(1, 0, 0, 0);
    if (i < nbuckets) { bdef[i].lo = 0; bdef[i].hi = 0; }
}

// acc[row] *= prod of the row's split partials, one CTA per row: strided
// products per thread, then a product tree in shared memory.  Deficit of the
// product: the splits' deficits + 2^(32L) for each of the nsplit + 256
// Montgomery products (nsplit strided, 255 tree, 1 into acc); row 0's CTA adds
// it to bdef[bucket].
template <int L>
__global__ void __launch_bounds__(256)
k_merge_cta(const Bucket* __restrict__ buckets, const RowInfo* __restrict__ info, const RowMod* __restrict__ mods,
            const uint4* __restrict__ part, const Deficit* __restrict__ defs, uint32_t row_begin,
            uint4* __restrict__ acc, Deficit* __restrict__ bdef) {
    __shared__ uint4 sx[256];
    __shared__ u128 sd[256];
    const uint32_t row = row_begin + blockIdx.x;
    const uint32_t b = info[row].bucket;
    const Bucket bk = buckets[b];
    if (bk.nsplit == 0 || bk.L != (uint32_t)L || row - bk.row_begin >= bk.nrows) return;   // uniform across the CTA
    const RowMod m = mods[row];
    uint32_t n[L];
#pragma unroll
    for (int k = 0; k < L; ++k) n[k] = m.n[k];
    const uint32_t rl = row - bk.row_begin;
    Res<L> X;
    set_small<L>(X, 1);
    u128 d = 0;
    for (uint32_t s = threadIdx.x; s < bk.nsplit; s += blockDim.x) {
        const uint4 v = part[bk.part_base + (uint64_t)s * bk.nrows + rl];
        Res<L> y;
        y.w[0] = v.x; y.w[1] = v.y;
        if (L > 2) y.w[2 < L ? 2 : 0] = v.z;
        if (L > 3) y.w[3 < L ? 3 : 0] = v.w;
        X = mont_mul<L>(X, y, n, m.ninv);
        if (rl == 0) {
            const Deficit x = defs[bk.def_base + s];
            d += ((u128)x.hi << 64) | x.lo;
        }
    }
    sx[threadIdx.x] = make_uint4(X.w[0], X.w[1], L > 2 ? X.w[2 < L ? 2 : 0] : 0, L > 3 ? X.w[3 < L ? 3 : 0] : 0);
    sd[threadIdx.x] = d;
    __syncthreads();
    for (uint32_t h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h) {
            const uint4 a = sx[threadIdx.x], c = sx[threadIdx.x + h];
            Res<L> A, C;
            A.w[0] = a.x; A.w[1] = a.y; C.w[0] = c.x; C.w[1] = c.y;
            if (L > 2) { A.w[2 < L ? 2 : 0] = a.z; C.w[2 < L ? 2 : 0] = c.z; }
            if (L > 3) { A.w[3 < L ? 3 : 0] = a.w; C.w[3 < L ? 3 : 0] = c.w; }
            A = mont_mul<L>(A, C, n, m.ninv);
            sx[threadIdx.x] = make_uint4(A.w[0], A.w[1], L > 2 ? A.w[2 < L ? 2 : 0] : 0, L > 3 ? A.w[3 < L ? 3 : 0] : 0);
            sd[threadIdx.x] += sd[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const uint4 a = acc[row], t = sx[0];
        Res<L> A, C;
        A.w[0] = a.x; A.w[1] = a.y; C.w[0] = t.x; C.w[1] = t.y;
        if (L > 2) { A.w[2 < L ? 2 : 0] = a.z; C.w[2 < L ? 2 : 0] = t.z; }
        if (L > 3) { A.w[3 < L ? 3 : 0] = a.w; C.w[3 < L ? 3 : 0] = t.w; }
        A = mont_mul<L>(A, C, n, m.ninv);
        acc[row] = make_uint4(A.w[0], A.w[1], L > 2 ? A.w[2 < L ? 2 : 0] : 0, L > 3 ? A.w[3 < L ? 3 : 0] : 0);
        if (rl == 0) {
            u128 tot = ((u128)bdef[b].hi << 64) | bdef[b].lo;
            tot += sd[0] + (u128)32 * L * ((u128)bk.nsplit + blockDim.x);
            bdef[b].lo = (uint64_t)tot;
            bdef[b].hi = (uint64_t)(tot >> 64);
        }
    }
}

// Serving sessions: fold each row's consecutive-integer tail (k_iterate items
// ipart[it_begin .. it_begin + it_count)) into its resident accumulator when
// the row is admitted.  The tail's power of two differs per row, so it is
// restored here; the one Montgomery product into acc removes 2^(32L) from
// every row alike, which the bucket's first row adds to bdef[bucket].
template <int L>
__global__ void __launch_bounds__(128)
k_tail_merge(const Bucket* __restrict__ buckets, const RowInfo* __restrict__ info, const RowMod* __restrict__ mods,
             const uint4* __restrict__ ipart, uint64_t K, uint32_t row_begin, uint32_t nrows,
             uint4* __restrict__ acc, Deficit* __restrict__ bdef) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nrows) return;
    const uint32_t row = row_begin + i;
    const RowInfo ri = info[row];
    const Bucket bk = buckets[ri.bucket];
    if (bk.L != (uint32_t)L || row - bk.row_begin >= bk.nrows) return;
    const RowMod m = mods[row];
    uint32_t n[L];
#pragma unroll
    for (int k = 0; k < L; ++k) n[k] = m.n[k];
    Res<L> X;
    set_small<L>(X, 1);
    u128 def = 0;
    for (uint32_t k = 0; k < ri.it_count; ++k) {
        const uint4 v = ipart[ri.it_begin + k];
        Res<L> y;
        y.w[0] = v.x; y.w[1] = v.y;
        if (L > 2) y.w[2 < L ? 2 : 0] = v.z;
        if (L > 3) y.w[3 < L ? 3 : 0] = v.w;
        X = mont_mul<L>(X, y, n, m.ninv);
        const uint64_t start = bk.T + 1 + (uint64_t)k * K;
        const uint64_t rest = ri.Tp - bk.T - (uint64_t)k * K;
        const uint64_t len = rest < K ? rest : K;
        def += (u128)len * (start + len - 1 < 0x80000000ull ? 32 : 64) + 32 * L;
    }
    // X * 2^def: Mont(2^def) = (2R)^def in the Montgomery domain
    Res<L> one;
    set_small<L>(one, 1);
    for (int k = 0; k < 32 * L; ++k) dbl_mod<L>(one, n);
    Res<L> two = one;
    dbl_mod<L>(two, n);
    X = mont_mul<L>(X, mont_pow<L>(two, def, one, n, m.ninv), n, m.ninv);
    const uint4 a = acc[row];
    Res<L> A;
    A.w[0] = a.x; A.w[1] = a.y;
    if (L > 2) A.w[2 < L ? 2 : 0] = a.z;
    if (L > 3) A.w[3 < L ? 3 : 0] = a.w;
    A = mont_mul<L>(A, X, n, m.ninv);
    acc[row] = make_uint4(A.w[0], A.w[1], L > 2 ? A.w[2 < L ? 2 : 0] : 0, L > 3 ? A.w[3 < L ? 3 : 0] : 0);
    if (row == bk.row_begin) {
        u128 d = ((u128)bdef[ri.bucket].hi << 64) | bdef[ri.bucket].lo;
        d += 32 * L;
        bdef[ri.bucket].lo = (uint64_t)d;
        bdef[ri.bucket].hi = (uint64_t)(d >> 64);
    }
}

// ===========================================================================
// launch wrappers
// ===========================================================================

void launch_sieve_segments(uint32_t seg0, uint32_t nseg, uint64_t limit, const uint32_t* base, uint32_t nbase,
                           uint32_t* bitmap, uint32_t* seg_count, cudaStream_t st) {
    if (!nseg) return;
    k_sieve_segments<<<nseg, SIEVE_THREADS, 0, st>>>(seg0, limit, base, nbase, bitmap, seg_count);
}
void launch_scan_counts(const uint32_t* counts, uint32_t n, uint64_t first, uint64_t* offsets, cudaStream_t st) {
    k_scan_counts<<<1, 1024, 0, st>>>(counts, n, first, offsets);
}
void launch_compact(uint32_t nseg, uint64_t lo0, const uint32_t* bitmap, const uint64_t* offsets,
                    uint32_t* out32, uint64_t* out64, cudaStream_t st) {
    if (!nseg) return;
    k_compact<<<nseg, COMPACT_THREADS, 0, st>>>(lo0, SEG_SPAN, bitmap, offsets, out32, out64, nullptr);
}
void launch_compact_multi(uint32_t nseg, const uint64_t* seg_lo, const uint32_t* bitmap, const uint64_t* offsets,
                          uint64_t* out64, cudaStream_t st) {
    if (!nseg) return;
    k_compact<<<nseg, COMPACT_THREADS, 0, st>>>(0, SEG_SPAN, bitmap, offsets, nullptr, out64, seg_lo);
}
void launch_window_primes_multi(const WinDesc* d, uint32_t nr, uint32_t nblocks, uint32_t* bitmap,
                                uint32_t* seg_count, cudaStream_t st) {
    if (!nr || !nblocks) return;
    k_window_primes_multi<<<nblocks, 256, 0, st>>>(d, nr, bitmap, seg_count);
}
void launch_count_leq(const uint32_t* cols, uint64_t ncols, const uint64_t* keys, uint32_t nkeys, uint64_t* out,
                      cudaStream_t st) {
    if (!nkeys) return;
    k_count_leq<<<(nkeys + 127) / 128, 128, 0, st>>>(cols, ncols, keys, nkeys, out);
}
void launch_setup_rows(const RowInfo* info, uint32_t nrows, RowMod* mods, cudaStream_t st) {
    if (!nrows) return;
    k_setup_rows<<<(nrows + 255) / 256, 256, 0, st>>>(info, nrows, mods);
}
void launch_group_products(const uint32_t* cols, uint64_t ngroups, uint32_t* gprod, uint8_t* gk, cudaStream_t st) {
    if (!ngroups) return;
    k_group_products<<<(unsigned)((ngroups + 127) / 128), 128, 0, st>>>(cols, ngroups, gprod, gk);
}
template <int V>
static void launch_sweep_v(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                           const RowMod* mods, const uint32_t* cols, uint4* part, Deficit* defs, cudaStream_t st,
                           ColGroups g) {
#define WL_SWEEP(LL, RR) k_sweep<LL, RR, V><<<nitems, 256, 0, st>>>(buckets, items, mods, cols, part, defs, g)
    if (L == 2) { if (rpt == 4) WL_SWEEP(2, 4); else if (rpt == 2) WL_SWEEP(2, 2); else WL_SWEEP(2, 1); }
    else if (L == 3) { if (rpt == 4) WL_SWEEP(3, 4); else if (rpt == 2) WL_SWEEP(3, 2); else WL_SWEEP(3, 1); }
    else { if (rpt == 4) WL_SWEEP(4, 4); else if (rpt == 2) WL_SWEEP(4, 2); else WL_SWEEP(4, 1); }
#undef WL_SWEEP
}
void launch_sweep(int variant, int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                  const RowMod* mods, const uint32_t* cols, uint4* part, Deficit* defs, cudaStream_t st,
                  ColGroups g) {
    if (!nitems) return;
    if (variant == 0) launch_sweep_v<0>(L, rpt, nitems, buckets, items, mods, cols, part, defs, st, g);
    else if (variant == 2) launch_sweep_v<2>(L, rpt, nitems, buckets, items, mods, cols, part, defs, st, g);
    else if (variant == 3) launch_sweep_v<3>(L, rpt, nitems, buckets, items, mods, cols, part, defs, st, g);
    else launch_sweep_v<1>(L, rpt, nitems, buckets, items, mods, cols, part, defs, st, g);
}
void launch_sweep_dense(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                        const RowMod* mods, const uint32_t* cols, const uint32_t* dsplit, uint4* part, Deficit* defs,
                        cudaStream_t st, int kernel, uint32_t hstep, unsigned long long* work) {
    if (!nitems) return;
    if (hstep == 0) hstep = 8;
#define WL_D(LL, MB, DWB, RR, SS) \
    k_sweep_dense<LL, MB, DWB, RR, SS><<<nitems, 256, 0, st>>>(buckets, items, mods, cols, dsplit, part, defs, hstep, \
                                                                work)
#define WL_DS(LL, MB, DWB) do {                                                                   \
        constexpr int nbk_ = (1 << DWB) - 1;                                                           \
        const int smem_ = nbk_ * 256 * (int)sizeof(uint4);                                             \
        static bool attr_ = false;                                                                      \
        if (!attr_) {                                                                                   \
            cudaFuncSetAttribute(k_sweep_dense<LL, MB, DWB, 1, 1, 1>,                                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, smem_);                   \
            attr_ = true;                                                                               \
        }                                                                                               \
        k_sweep_dense<LL, MB, DWB, 1, 1, 1><<<nitems, 256, smem_, st>>>(buckets, items, mods, cols, dsplit, \
                                                                      part, defs, hstep, work);         \
    } while (0)
    if (rpt == 2) {
        if (L == 2) WL_D(2, 2, 3, 2, 0); else if (L == 3) WL_D(3, 2, 3, 2, 0); else WL_D(4, 2, 3, 2, 0);
    } else if (kernel == DENSE_SMEM_W3) {
        if (L == 2) WL_DS(2, 4, 3); else if (L == 3) WL_DS(3, 4, 3); else WL_DS(4, 4, 3);
    } else if (kernel == DENSE_SMEM_W4) {
        if (L == 2) WL_DS(2, 2, 4); else if (L == 3) WL_DS(3, 2, 4); else WL_DS(4, 2, 4);
    } else if (kernel == DENSE_SORTED_W4) {
        if (L == 2) WL_D(2, 2, 4, 1, 1); else if (L == 3) WL_D(3, 2, 4, 1, 1); else WL_D(4, 2, 4, 1, 1);
    } else if (kernel == DENSE_SWITCH_W3) {
        if (L == 2) WL_D(2, 3, 3, 1, 0); else if (L == 3) WL_D(3, 3, 3, 1, 0); else WL_D(4, 3, 3, 1, 0);
    } else if (kernel == DENSE_SWITCH_W4) {
        if (L == 2) WL_D(2, 2, 4, 1, 0); else if (L == 3) WL_D(3, 2, 4, 1, 0); else WL_D(4, 2, 4, 1, 0);
    } else if (kernel == DENSE_SORTED_W3_2CTA) {
        if (L == 2) WL_D(2, 2, 3, 1, 1); else if (L == 3) WL_D(3, 2, 3, 1, 1); else WL_D(4, 2, 3, 1, 1);
    } else {   // DENSE_SORTED_W3
        if (L == 2) WL_D(2, 3, 3, 1, 1); else if (L == 3) WL_D(3, 3, 3, 1, 1); else WL_D(4, 3, 3, 1, 1);
    }
#undef WL_D
#undef WL_DS
}
void launch_iterate(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, uint32_t row_begin,
                    uint32_t nrows, uint32_t item_begin, uint32_t nitems, uint64_t K, uint4* out, cudaStream_t st) {
    if (!nitems) return;
    const unsigned g = (nitems + 255) / 256;
    if (L == 2) k_iterate<2><<<g, 256, 0, st>>>(buckets, info, mods, row_begin, nrows, item_begin, nitems, K, out);
    else if (L == 3) k_iterate<3><<<g, 256, 0, st>>>(buckets, info, mods, row_begin, nrows, item_begin, nitems, K, out);
    else k_iterate<4><<<g, 256, 0, st>>>(buckets, info, mods, row_begin, nrows, item_begin, nitems, K, out);
}
void launch_sieve_big(uint64_t lo, uint64_t hi, uint32_t nseg, uint32_t spc, const uint32_t* base, uint32_t nbase,
                      uint32_t* offsets, uint32_t* bitmap, uint32_t* seg_count, cudaStream_t st) {
    if (!nseg) return;
    const size_t smem = (BIG_WORDS + PRE_TABLE) * sizeof(uint32_t);
    cudaFuncSetAttribute(k_sieve_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const uint32_t ncta = (nseg + spc - 1) / spc;
    // sieving primes below 1024 (base starts at 67) are marked cooperatively
    uint32_t ncoop = 0;
    {
        static const uint32_t below1024 = 154;   // odd primes 67 .. 1021
        ncoop = nbase < below1024 ? nbase : below1024;
    }
    k_sieve_big<<<ncta, BIG_THREADS, smem, st>>>(lo, hi, nseg, spc, base, nbase, ncoop, offsets, bitmap, seg_count);
}
void launch_compact_big(uint32_t nseg, uint64_t lo0, const uint32_t* bitmap, const uint64_t* offsets, uint64_t* out,
                        cudaStream_t st) {
    if (!nseg) return;
    k_compact_big<<<nseg, 1024, 0, st>>>(lo0, bitmap, offsets, out);
}
void launch_count_leq64(const uint64_t* cols, uint64_t ncols, const uint64_t* keys, uint32_t nkeys, uint64_t* out,
                        cudaStream_t st) {
    if (!nkeys) return;
    k_count_leq64<<<(nkeys + 127) / 128, 128, 0, st>>>(cols, ncols, keys, nkeys, out);
}
void launch_sweep64(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items, const RowMod* mods,
                    const uint64_t* cols, uint4* part, Deficit* defs, cudaStream_t st) {
    if (!nitems) return;
#define WL_S64(LL, RR) k_sweep64<LL, RR><<<nitems, 256, 0, st>>>(buckets, items, mods, cols, part, defs)
    if (L == 2) { if (rpt == 2) WL_S64(2, 2); else WL_S64(2, 1); }
    else if (L == 3) { if (rpt == 2) WL_S64(3, 2); else WL_S64(3, 1); }
    else { if (rpt == 2) WL_S64(4, 2); else WL_S64(4, 1); }
#undef WL_S64
}
void launch_acc_init(uint32_t nrows, uint32_t nbuckets, uint4* acc, Deficit* bdef, cudaStream_t st) {
    const uint32_t n = nrows > nbuckets ? nrows : nbuckets;
    if (!n) return;
    k_acc_init<<<(n + 255) / 256, 256, 0, st>>>(nrows, nbuckets, acc, bdef);
}
void launch_merge_cta(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* part,
                      const Deficit* defs, uint32_t row_begin, uint32_t nrows, uint4* acc, Deficit* bdef,
                      cudaStream_t st) {
    if (!nrows) return;
    if (L == 2) k_merge_cta<2><<<nrows, 256, 0, st>>>(buckets, info, mods, part, defs, row_begin, acc, bdef);
    else if (L == 3) k_merge_cta<3><<<nrows, 256, 0, st>>>(buckets, info, mods, part, defs, row_begin, acc, bdef);
    else k_merge_cta<4><<<nrows, 256, 0, st>>>(buckets, info, mods, part, defs, row_begin, acc, bdef);
}

void launch_clear_below(uint32_t* bitmap, uint64_t lo, uint64_t q_lo, uint64_t nwords, cudaStream_t st) {
    if (q_lo <= lo || !nwords) return;
    const uint64_t lim = (q_lo - lo) / 64 + 1;
    const uint64_t need = nwords < lim ? nwords : lim;
    k_clear_below<<<(unsigned)((need + 255) / 256), 256, 0, st>>>(bitmap, lo, q_lo, need);
}

// The tail of rows [row_begin, row_begin + nrows) is in their running
// products (k_tail_merge): k_finish must not multiply it in again.
__global__ void k_clear_tail(RowInfo* __restrict__ info, uint32_t row_begin, uint32_t nrows) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nrows) {
        info[row_begin + i].it_begin = 0;
        info[row_begin + i].it_count = 0;
    }
}

void launch_clear_tail(RowInfo* info, uint32_t row_begin, uint32_t nrows, cudaStream_t st) {
    if (!nrows) return;
    k_clear_tail<<<(nrows + 255) / 256, 256, 0, st>>>(info, row_begin, nrows);
}

void launch_tail_merge(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* ipart,
                       uint64_t K, uint32_t row_begin, uint32_t nrows, uint4* acc, Deficit* bdef, cudaStream_t st) {
    if (!nrows) return;
    const unsigned g = (nrows + 127) / 128;
    if (L == 2) k_tail_merge<2><<<g, 128, 0, st>>>(buckets, info, mods, ipart, K, row_begin, nrows, acc, bdef);
    else if (L == 3) k_tail_merge<3><<<g, 128, 0, st>>>(buckets, info, mods, ipart, K, row_begin, nrows, acc, bdef);
    else k_tail_merge<4><<<g, 128, 0, st>>>(buckets, info, mods, ipart, K, row_begin, nrows, acc, bdef);
}
void launch_sweep_bits(int L, int rpt, uint32_t nitems, const Bucket* buckets, const SweepItem* items,
                       const RowMod* mods, const uint32_t* bitmap, uint64_t lo, const uint64_t* keys, uint4* part,
                       Deficit* defs, cudaStream_t st, const uint64_t* los) {
    if (!nitems) return;
#define WL_SB(LL, RR) k_sweep_bits<LL, RR><<<nitems, 256, 0, st>>>(buckets, items, mods, bitmap, lo, keys, part, defs, \
                                                                 los)
    if (L == 2) { if (rpt == 2) WL_SB(2, 2); else WL_SB(2, 1); }
    else if (L == 3) { if (rpt == 2) WL_SB(3, 2); else WL_SB(3, 1); }
    else { if (rpt == 2) WL_SB(4, 2); else WL_SB(4, 1); }
#undef WL_SB
}
void launch_count_bits(const uint32_t* bitmap, uint64_t lo, uint64_t nwords, uint64_t key, unsigned long long* out,
                       cudaStream_t st) {
    if (!nwords) return;
    k_count_bits<<<1184, 256, 0, st>>>(bitmap, lo, nwords, key, out);
}
void launch_merge(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* part,
                  const Deficit* defs, uint32_t row_begin, uint32_t nrows, uint4* acc, Deficit* bdef, cudaStream_t st) {
    if (!nrows) return;
    const unsigned g = (nrows + 127) / 128;
    if (L == 2) k_merge<2><<<g, 128, 0, st>>>(buckets, info, mods, part, defs, row_begin, nrows, acc, bdef);
    else if (L == 3) k_merge<3><<<g, 128, 0, st>>>(buckets, info, mods, part, defs, row_begin, nrows, acc, bdef);
    else k_merge<4><<<g, 128, 0, st>>>(buckets, info, mods, part, defs, row_begin, nrows, acc, bdef);
}
void launch_finish(int L, const Bucket* buckets, const RowInfo* info, const RowMod* mods, const uint4* part,
                   const Deficit* defs, uint64_t K, const uint4* ipart, uint32_t row_begin,
                   uint32_t nrows, int full, RowOut* out, cudaStream_t st, const uint4* acc1, const Deficit* def1,
                   const uint4* acc2, const Deficit* def2) {
    if (!nrows) return;
    const unsigned g = (nrows + 127) / 128;
    if (L == 2) k_finish<2><<<g, 128, 0, st>>>(buckets, info, mods, part, defs, K, ipart, row_begin, nrows, full, out, acc1, def1, acc2, def2, acc1 != nullptr);
    else if (L == 3) k_finish<3><<<g, 128, 0, st>>>(buckets, info, mods, part, defs, K, ipart, row_begin, nrows, full, out, acc1, def1, acc2, def2, acc1 != nullptr);
    else k_finish<4><<<g, 128, 0, st>>>(buckets, info, mods, part, defs, K, ipart, row_begin, nrows, full, out, acc1, def1, acc2, def2, acc1 != nullptr);
}
void launch_rows_product(const uint64_t* ps, uint64_t n_rows, const uint64_t* parts, uint32_t nparts, uint64_t* out,
                         cudaStream_t st) {
    if (!n_rows || !nparts) return;
    k_rows_product<<<(unsigned)((n_rows + 127) / 128), 128, 0, st>>>(ps, n_rows, parts, nparts, out);
}

}  // namespace wl
