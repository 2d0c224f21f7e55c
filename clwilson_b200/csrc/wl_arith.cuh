// wl_arith.cuh -- modular arithmetic modulo n = p^2 for the Wilson-prime engine.
//
// Residues modulo n = p^2 (p < 2^62, so n < 2^124) are held in L little-endian
// 32-bit limbs, L = 2 (p < 2^31), 3 (p < 2^47) or 4 (p < 2^62).  Montgomery
// reduction uses R = 2^(32L) for full products and 2^32 for the hot "cell"
// step, which multiplies a residue by one 32-bit sieving prime q:
//
//     cell(x, q) = (x*q + m*n) / 2^32,   m = (x*q mod 2^32) * (-n^-1) mod 2^32
//
// Values are kept lazily reduced: every routine accepts and returns x < 2n.
// That holds for cell() when q < 2^31 (x*q/2^32 < n), and for the full product
// when 4n < R, which is why the widths stop at p < 2^31 / 2^47 / 2^62.  For
// 2^31 <= q < 2^32 cell_wide() adds one conditional subtraction of n.
//
// The engine never converts a sieving prime into Montgomery form: each cell
// removes a factor 2^32 that is tracked as an exponent ("deficit") shared by
// every row of a sweep and restored once per row at the end (see
// wl_kernels.cu).  This replaces the reference's per-column conversion
// m2p_mul_r2 + m2p_mul (kernels/mulsmall.cl:36-58) with a single
// 1-limb x L-limb step.
#pragma once
#include <stdint.h>
#include "wl_internal.h"

namespace wl {

typedef unsigned __int128 u128;

template <int L> struct Res { uint32_t w[L]; };


// ---------------------------------------------------------------------------
// Hot step: x <- (x*q + m*n) / 2^32 as one PTX carry chain (integer pipe).
// Operation count: 4L+1 multiplies (mul/mad lo/hi) and 2 carry additions.
// ---------------------------------------------------------------------------

__device__ __forceinline__ void cell(Res<2>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    asm("{\n\t"
        ".reg .u32 t0, t1, t2, m, z;\n\t"
        "mul.lo.u32      t0, %2, %4;\n\t"
        "mul.hi.u32      t1, %2, %4;\n\t"
        "mul.hi.u32      t2, %3, %4;\n\t"
        "mad.lo.cc.u32   t1, %3, %4, t1;\n\t"
        "addc.u32        t2, t2, 0;\n\t"
        "mul.lo.u32      m, t0, %7;\n\t"
        "mad.lo.cc.u32   z, m, %5, t0;\n\t"
        "madc.lo.cc.u32  t1, m, %6, t1;\n\t"
        "addc.u32        t2, t2, 0;\n\t"
        "mad.hi.cc.u32   t1, m, %5, t1;\n\t"
        "madc.hi.u32     t2, m, %6, t2;\n\t"
        "mov.u32         %0, t1;\n\t"
        "mov.u32         %1, t2;\n\t"
        "}"
        : "=r"(x.w[0]), "=r"(x.w[1])
        : "r"(x.w[0]), "r"(x.w[1]), "r"(q), "r"(n[0]), "r"(n[1]), "r"(ninv));
}

__device__ __forceinline__ void cell(Res<3>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    asm("{\n\t"
        ".reg .u32 t0, t1, t2, t3, m, z;\n\t"
        "mul.lo.u32      t0, %3, %6;\n\t"
        "mul.hi.u32      t1, %3, %6;\n\t"
        "mul.hi.u32      t2, %4, %6;\n\t"
        "mul.hi.u32      t3, %5, %6;\n\t"
        "mad.lo.cc.u32   t1, %4, %6, t1;\n\t"
        "madc.lo.cc.u32  t2, %5, %6, t2;\n\t"
        "addc.u32        t3, t3, 0;\n\t"
        "mul.lo.u32      m, t0, %10;\n\t"
        "mad.lo.cc.u32   z, m, %7, t0;\n\t"
        "madc.lo.cc.u32  t1, m, %8, t1;\n\t"
        "madc.lo.cc.u32  t2, m, %9, t2;\n\t"
        "addc.u32        t3, t3, 0;\n\t"
        "mad.hi.cc.u32   t1, m, %7, t1;\n\t"
        "madc.hi.cc.u32  t2, m, %8, t2;\n\t"
        "madc.hi.u32     t3, m, %9, t3;\n\t"
        "mov.u32         %0, t1;\n\t"
        "mov.u32         %1, t2;\n\t"
        "mov.u32         %2, t3;\n\t"
        "}"
        : "=r"(x.w[0]), "=r"(x.w[1]), "=r"(x.w[2])
        : "r"(x.w[0]), "r"(x.w[1]), "r"(x.w[2]), "r"(q), "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(ninv));
}

__device__ __forceinline__ void cell(Res<4>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    asm("{\n\t"
        ".reg .u32 t0, t1, t2, t3, t4, m, z;\n\t"
        "mul.lo.u32      t0, %4, %8;\n\t"
        "mul.hi.u32      t1, %4, %8;\n\t"
        "mul.hi.u32      t2, %5, %8;\n\t"
        "mul.hi.u32      t3, %6, %8;\n\t"
        "mul.hi.u32      t4, %7, %8;\n\t"
        "mad.lo.cc.u32   t1, %5, %8, t1;\n\t"
        "madc.lo.cc.u32  t2, %6, %8, t2;\n\t"
        "madc.lo.cc.u32  t3, %7, %8, t3;\n\t"
        "addc.u32        t4, t4, 0;\n\t"
        "mul.lo.u32      m, t0, %13;\n\t"
        "mad.lo.cc.u32   z, m, %9, t0;\n\t"
        "madc.lo.cc.u32  t1, m, %10, t1;\n\t"
        "madc.lo.cc.u32  t2, m, %11, t2;\n\t"
        "madc.lo.cc.u32  t3, m, %12, t3;\n\t"
        "addc.u32        t4, t4, 0;\n\t"
        "mad.hi.cc.u32   t1, m, %9, t1;\n\t"
        "madc.hi.cc.u32  t2, m, %10, t2;\n\t"
        "madc.hi.cc.u32  t3, m, %11, t3;\n\t"
        "madc.hi.u32     t4, m, %12, t4;\n\t"
        "mov.u32         %0, t1;\n\t"
        "mov.u32         %1, t2;\n\t"
        "mov.u32         %2, t3;\n\t"
        "mov.u32         %3, t4;\n\t"
        "}"
        : "=r"(x.w[0]), "=r"(x.w[1]), "=r"(x.w[2]), "=r"(x.w[3])
        : "r"(x.w[0]), "r"(x.w[1]), "r"(x.w[2]), "r"(x.w[3]), "r"(q),
          "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]), "r"(ninv));
}

// The same step with 32x32->64 products (mad.wide.u32): the two product rows
// x*q and m*n are formed as chains of 64-bit partial sums, so carries become
// 64-bit additions on the integer ALU instead of carry-flag multiplies.
// 2L wide multiplies + 1 low multiply.
template <int L>
__host__ __device__ __forceinline__ void cell_w(Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    uint64_t P = (uint64_t)x.w[0] * q;
    const uint32_t t0 = (uint32_t)P;
    uint32_t X[L];                                   // (x*q) >> 32, L limbs
#pragma unroll
    for (int k = 1; k < L; ++k) {
        P = (uint64_t)x.w[k] * q + (P >> 32);
        X[k - 1] = (uint32_t)P;
    }
    X[L - 1] = (uint32_t)(P >> 32);
    const uint32_t m = t0 * ninv;
    uint64_t A = (uint64_t)m * n[0] + t0;            // low word is zero
#pragma unroll
    for (int k = 1; k < L; ++k) {
        A = (uint64_t)m * n[k] + X[k - 1] + (A >> 32);
        x.w[k - 1] = (uint32_t)A;
    }
    x.w[L - 1] = X[L - 1] + (uint32_t)(A >> 32);
}

// Step j of the Montgomery product of x by a multi-limb multiplier
// W = sum_j w_j 2^(32j) (an exact product of several columns, shared by every
// row): with x fixed and the accumulator t zero before the first step,
//     t <- (t + x*w_j + m*n) / 2^32,   m = -(t + x*w_j) * n^-1 mod 2^32.
// After the k limbs of W, t = x*W / 2^(32k) mod n.  With x < 2n and
// t < x + n before a step, t + x*w_j + m*n < 2^32 (x + n), so t < x + n < 3n
// after it: L limbs hold t while 3n < 2^(32L) (n = p^2 with p below 2^31,
// 2^47, 2^62 for L = 2, 3, 4), and one conditional subtraction after the last
// limb brings it below 2n.  The same 2L + 1 multiplies as a cell, for 32 bits
// of multiplier instead of one column of 27 to 32 bits.
template <int L>
__host__ __device__ __forceinline__ void limb_step(uint32_t (&t)[L], const Res<L>& x, uint32_t w,
                                                   const uint32_t* n, uint32_t ninv) {
    uint64_t S = (uint64_t)x.w[0] * w + t[0];
    const uint32_t u0 = (uint32_t)S;
    uint32_t U[L];                                   // (t + x*w) >> 32, L limbs
#pragma unroll
    for (int k = 1; k < L; ++k) {
        S = (uint64_t)x.w[k] * w + t[k] + (S >> 32);
        U[k - 1] = (uint32_t)S;
    }
    U[L - 1] = (uint32_t)(S >> 32);
    const uint32_t m = u0 * ninv;
    uint64_t A = (uint64_t)m * n[0] + u0;            // low word is zero
#pragma unroll
    for (int k = 1; k < L; ++k) {
        A = (uint64_t)m * n[k] + U[k - 1] + (A >> 32);
        t[k - 1] = (uint32_t)A;
    }
    t[L - 1] = U[L - 1] + (uint32_t)(A >> 32);
}

// As cell_w, with the first reduction product replaced by its high half:
// lo(m*n0) = -t0 mod 2^32, so (m*n0 + t0) >> 32 = hi(m*n0) + (t0 != 0).
__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b) {
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

template <int L>
__host__ __device__ __forceinline__ void cell_h(Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    uint64_t P = (uint64_t)x.w[0] * q;
    const uint32_t t0 = (uint32_t)P;
    uint32_t X[L];
#pragma unroll
    for (int k = 1; k < L; ++k) {
        P = (uint64_t)x.w[k] * q + (P >> 32);
        X[k - 1] = (uint32_t)P;
    }
    X[L - 1] = (uint32_t)(P >> 32);
    const uint32_t m = t0 * ninv;
    uint64_t A = (uint64_t)(mulhi32(m, n[0]) + (t0 != 0u)) << 32;
#pragma unroll
    for (int k = 1; k < L; ++k) {
        A = (uint64_t)m * n[k] + X[k - 1] + (A >> 32);
        x.w[k - 1] = (uint32_t)A;
    }
    x.w[L - 1] = X[L - 1] + (uint32_t)(A >> 32);
}

// x <- x - n if x >= n, as one asm block so that no compiler-generated carry
// instruction can land inside the borrow chain; maps [0, 3n) to [0, 2n).
__device__ __forceinline__ void cond_sub_chain(Res<3>& x, const uint32_t* n) {
    asm("{\n\t"
        ".reg .u32 s0, s1, s2, b;\n\t"
        ".reg .pred k;\n\t"
        "sub.cc.u32   s0, %0, %3;\n\t"
        "subc.cc.u32  s1, %1, %4;\n\t"
        "subc.cc.u32  s2, %2, %5;\n\t"
        "mov.u32      b, 0;\n\t"
        "subc.u32     b, b, b;\n\t"
        "setp.eq.u32  k, b, 0;\n\t"
        "@k mov.u32   %0, s0;\n\t"
        "@k mov.u32   %1, s1;\n\t"
        "@k mov.u32   %2, s2;\n\t"
        "}"
        : "+r"(x.w[0]), "+r"(x.w[1]), "+r"(x.w[2])
        : "r"(n[0]), "r"(n[1]), "r"(n[2]));
}
__device__ __forceinline__ void cond_sub_chain(Res<4>& x, const uint32_t* n) {
    asm("{\n\t"
        ".reg .u32 s0, s1, s2, s3, b;\n\t"
        ".reg .pred k;\n\t"
        "sub.cc.u32   s0, %0, %4;\n\t"
        "subc.cc.u32  s1, %1, %5;\n\t"
        "subc.cc.u32  s2, %2, %6;\n\t"
        "subc.cc.u32  s3, %3, %7;\n\t"
        "mov.u32      b, 0;\n\t"
        "subc.u32     b, b, b;\n\t"
        "setp.eq.u32  k, b, 0;\n\t"
        "@k mov.u32   %0, s0;\n\t"
        "@k mov.u32   %1, s1;\n\t"
        "@k mov.u32   %2, s2;\n\t"
        "@k mov.u32   %3, s3;\n\t"
        "}"
        : "+r"(x.w[0]), "+r"(x.w[1]), "+r"(x.w[2]), "+r"(x.w[3])
        : "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]));
}
__device__ __forceinline__ void cond_sub_chain(Res<2>& x, const uint32_t* n) {
    asm("{\n\t"
        ".reg .u32 s0, s1, b;\n\t"
        ".reg .pred k;\n\t"
        "sub.cc.u32   s0, %0, %2;\n\t"
        "subc.cc.u32  s1, %1, %3;\n\t"
        "mov.u32      b, 0;\n\t"
        "subc.u32     b, b, b;\n\t"
        "setp.eq.u32  k, b, 0;\n\t"
        "@k mov.u32   %0, s0;\n\t"
        "@k mov.u32   %1, s1;\n\t"
        "}"
        : "+r"(x.w[0]), "+r"(x.w[1])
        : "r"(n[0]), "r"(n[1]));
}

// Cell with any 32-bit q: result < 3n before the subtraction, < 2n after.
template <int L>
__device__ __forceinline__ void cell_wide(Res<L>& x, uint32_t q, const uint32_t* n, uint32_t ninv) {
    cell(x, q, n, ninv);
    cond_sub_chain(x, n);
}

// ---------------------------------------------------------------------------
// Portable multi-limb helpers (compiler-scheduled; used off the hot loop).
// ---------------------------------------------------------------------------

template <int L>
__device__ __forceinline__ void set_small(Res<L>& x, uint64_t v) {
    x.w[0] = (uint32_t)v;
    if (L > 1) x.w[1] = (uint32_t)(v >> 32);
#pragma unroll
    for (int i = 2; i < L; ++i) x.w[i] = 0;
}

template <int L>
__device__ __forceinline__ bool geq(const Res<L>& a, const uint32_t* b) {
#pragma unroll
    for (int i = L - 1; i >= 0; --i) {
        if (a.w[i] != b[i]) return a.w[i] > b[i];
    }
    return true;
}

template <int L>
__device__ __forceinline__ bool is_zero(const Res<L>& a) {
    uint32_t o = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) o |= a.w[i];
    return o == 0;
}

// a - b over L limbs, returns the borrow
template <int L>
__device__ __forceinline__ uint32_t sub_limbs(Res<L>& a, const uint32_t* b) {
    uint64_t br = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t d = (uint64_t)a.w[i] - b[i] - br;
        a.w[i] = (uint32_t)d;
        br = (d >> 63) & 1;
    }
    return (uint32_t)br;
}
template <int L>
__device__ __forceinline__ uint32_t add_limbs(Res<L>& a, const uint32_t* b) {
    uint64_t c = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t s = (uint64_t)a.w[i] + b[i] + c;
        a.w[i] = (uint32_t)s;
        c = s >> 32;
    }
    return (uint32_t)c;
}

// Full reduction of x < 2n to [0, n).
template <int L>
__device__ __forceinline__ void reduce_full(Res<L>& x, const uint32_t* n) {
    if (geq<L>(x, n)) sub_limbs<L>(x, n);
}

// Montgomery product: a*b / R mod n, R = 2^(32L); a, b < 2n -> result < 2n.
// Coarsely integrated operand scanning with 64-bit accumulators.
template <int L>
__device__ __forceinline__ Res<L> mont_mul(const Res<L>& a, const Res<L>& b, const uint32_t* n, uint32_t ninv) {
    uint32_t t[L + 2];
#pragma unroll
    for (int i = 0; i < L + 2; ++i) t[i] = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < L; ++j) {
            uint64_t s = (uint64_t)a.w[j] * b.w[i] + t[j] + c;
            t[j] = (uint32_t)s;
            c = s >> 32;
        }
        uint64_t s = (uint64_t)t[L] + c;
        t[L] = (uint32_t)s;
        t[L + 1] = (uint32_t)(s >> 32);
        uint32_t m = t[0] * ninv;
        c = ((uint64_t)m * n[0] + t[0]) >> 32;
#pragma unroll
        for (int j = 1; j < L; ++j) {
            uint64_t s2 = (uint64_t)m * n[j] + t[j] + c;
            t[j - 1] = (uint32_t)s2;
            c = s2 >> 32;
        }
        s = (uint64_t)t[L] + c;
        t[L - 1] = (uint32_t)s;
        t[L] = t[L + 1] + (uint32_t)(s >> 32);
    }
    Res<L> r;
#pragma unroll
    for (int i = 0; i < L; ++i) r.w[i] = t[i];
    return r;
}

// Montgomery step with a 64-bit multiplier v < 2^63: x*v / 2^64 mod n.
// Two rounds of the cell recurrence; x < 2n -> result < 2n.
template <int L>
__device__ __forceinline__ void cell64(Res<L>& x, uint64_t v, const uint32_t* n, uint32_t ninv) {
    uint32_t t[L + 2];
#pragma unroll
    for (int i = 0; i < L + 2; ++i) t[i] = 0;
    const uint32_t vw[2] = { (uint32_t)v, (uint32_t)(v >> 32) };
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < L; ++j) {
            uint64_t s = (uint64_t)x.w[j] * vw[i] + t[j] + c;
            t[j] = (uint32_t)s;
            c = s >> 32;
        }
        uint64_t s = (uint64_t)t[L] + c;
        t[L] = (uint32_t)s;
        t[L + 1] = (uint32_t)(s >> 32);
        uint32_t m = t[0] * ninv;
        c = ((uint64_t)m * n[0] + t[0]) >> 32;
#pragma unroll
        for (int j = 1; j < L; ++j) {
            uint64_t s2 = (uint64_t)m * n[j] + t[j] + c;
            t[j - 1] = (uint32_t)s2;
            c = s2 >> 32;
        }
        s = (uint64_t)t[L] + c;
        t[L - 1] = (uint32_t)s;
        t[L] = t[L + 1] + (uint32_t)(s >> 32);
    }
#pragma unroll
    for (int i = 0; i < L; ++i) x.w[i] = t[i];
}

// Lazily reduced modular add / sub in [0, 2n) (needs 4n < 2^(32L)).
template <int L>
__device__ __forceinline__ Res<L> add_mod2n(Res<L> a, const Res<L>& b, const uint32_t* n) {
    add_limbs<L>(a, b.w);
    uint32_t n2[L];
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) { n2[i] = (n[i] << 1) | c; c = n[i] >> 31; }
    if (geq<L>(a, n2)) sub_limbs<L>(a, n2);
    return a;
}
template <int L>
__device__ __forceinline__ Res<L> sub_mod2n(Res<L> a, const Res<L>& b, const uint32_t* n) {
    uint32_t br = sub_limbs<L>(a, b.w);
    if (br) {
        uint32_t n2[L];
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < L; ++i) { n2[i] = (n[i] << 1) | c; c = n[i] >> 31; }
        add_limbs<L>(a, n2);
    }
    return a;
}

// x <- 2x mod n for x < n (full reduction kept)
template <int L>
__device__ __forceinline__ void dbl_mod(Res<L>& x, const uint32_t* n) {
    uint32_t c = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) { uint32_t nc = x.w[i] >> 31; x.w[i] = (x.w[i] << 1) | c; c = nc; }
    // x < 2n < 2^(32L): no carry out of the top limb since 4n < R
    if (geq<L>(x, n)) sub_limbs<L>(x, n);
}

// base^e (Montgomery domain; one = R mod n), left-to-right binary, e < 2^128
template <int L>
__device__ __forceinline__ Res<L> mont_pow(const Res<L>& base, u128 e, const Res<L>& one,
                                           const uint32_t* n, uint32_t ninv) {
    if (e == 0) return one;
    int top = 127;
    while (!((e >> top) & 1)) --top;
    Res<L> r = base;
    for (int b = top - 1; b >= 0; --b) {
        r = mont_mul<L>(r, r, n, ninv);
        if ((e >> b) & 1) r = mont_mul<L>(r, base, n, ninv);
    }
    return r;
}

// ---------------------------------------------------------------------------
// Single-word arithmetic modulo an odd m < 2^62 (R = 2^64), for primality
// tests and Cornacchia's algorithm.
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint64_t inv64(uint64_t m) {   // m^-1 mod 2^64 (Newton)
    uint64_t x = m;                  // correct to 3 bits for odd m
#pragma unroll
    for (int i = 0; i < 5; ++i) x *= 2 - m * x;
    return x;
}
// a*b*2^-64 mod m for a, b < 2m (lazy), result < 2m; minv = -m^-1 mod 2^64
__device__ __forceinline__ uint64_t mul64(uint64_t a, uint64_t b, uint64_t m, uint64_t minv) {
    uint64_t lo = a * b, hi = __umul64hi(a, b);
    uint64_t k = lo * minv;
    uint64_t klo = k * m, khi = __umul64hi(k, m);
    uint64_t s = lo + klo;
    uint64_t c = (s < lo) ? 1 : 0;
    return hi + khi + c;
}
__device__ __forceinline__ uint64_t red64(uint64_t a, uint64_t m) { return a >= m ? a - m : a; }

struct Mod64 {
    uint64_t m, minv, one, r2;   // one = 2^64 mod m, r2 = 2^128 mod m
    __device__ void init(uint64_t mod) {
        m = mod;
        minv = 0 - inv64(mod);
        one = (0 - mod) % mod;
        // r2 = one * 2^64 mod m by 64 doublings
        uint64_t x = one;
        for (int i = 0; i < 64; ++i) { x <<= 1; if (x >= m) x -= m; }
        r2 = x;
    }
    __device__ __forceinline__ uint64_t to(uint64_t x) const { return mul64(x % m, r2, m, minv); }
    __device__ __forceinline__ uint64_t from(uint64_t x) const { return red64(mul64(x, 1, m, minv), m); }
    __device__ __forceinline__ uint64_t mul(uint64_t a, uint64_t b) const { return mul64(a, b, m, minv); }
    __device__ uint64_t pow(uint64_t b, uint64_t e) const {   // Montgomery domain
        uint64_t r = one;
        while (e) { if (e & 1) r = mul(r, b); b = mul(b, b); e >>= 1; }
        return r;
    }
};

// integer square root of a 64-bit value (Newton from an overestimate)
__device__ __forceinline__ uint64_t isqrt64(uint64_t n) {
    if (n < 2) return n;
    int bits = 64 - __clzll(n);
    uint64_t x = 1ULL << ((bits + 1) / 2);     // x >= sqrt(n)
    while (true) {
        uint64_t y = (x + n / x) >> 1;
        if (y >= x) break;
        x = y;
    }
    while (x * x > n) --x;
    while ((x + 1) * (x + 1) <= n) ++x;
    return x;
}

// Exponent of the prime q in T!: sum over k of floor(T / q^k) (Legendre's
// formula; the reference's getPower, cl_wilson.cpp:1293-1313).  The terms come
// as running quotients, floor(T / q^k) = floor(floor(T / q^(k-1)) / q), so a
// term costs one division, and once a quotient and q fit 32 bits that division
// is a 32-bit one (a 64-bit division costs several times as many multiplies).
__host__ __device__ __forceinline__ uint64_t legendre(uint64_t T, uint64_t q) {
    uint64_t t = T / q, e = 0;
    while (t) {
        e += t;
        if (t < q) break;                           // the next term is zero
        t = ((t | q) >> 32) == 0 ? (uint64_t)((uint32_t)t / (uint32_t)q) : t / q;
    }
    return e;
}

}  // namespace wl
