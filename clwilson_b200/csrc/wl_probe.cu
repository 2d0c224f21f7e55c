// wl_probe.cu -- integer-pipe microbenchmarks that set the roofline of the
// column sweep (include/wilson_probe.h).
//
//   WL_PROBE_MAD     mad.lo.u32, 8 independent chains per thread
//   WL_PROBE_MADHI   mad.hi.u32, 8 independent chains per thread
//   WL_PROBE_CELL2/3/4  the sweep's cell step (wl_arith.cuh) at L = 2, 3, 4,
//                    4 independent rows per thread, operands in registers
//   WL_PROBE_DFMA    fma.rn.f64, 8 independent chains per thread
//   WL_PROBE_MAD_DFMA / WL_PROBE_MADWIDE_DFMA  mad.lo.u32 (or mad.wide.u32) and
//                    fma.rn.f64 chains interleaved, both counted: whether the
//                    FP64 pipe adds multiply throughput next to the integer one
//   WL_PROBE_CELL2_FP64  an exact Montgomery cell mod p^2 (p < 2^31) in FP64
//                    (cell_fp below), 2 rows per thread
//   WL_PROBE_CELL2_MIX   per CTA, warps 0-5 run the integer cell and warps 6-7
//                    the FP64 cell, 2 rows per thread (all cells counted)
//
// Each result is operations (or cells) per second over the whole GPU, timed
// with CUDA events around one launch sized to run for tens of milliseconds.
#include "wilson.h"
#include "wilson_probe.h"
#include "wl_internal.h"
#include "wl_arith.cuh"

#ifndef WL_CELL_VARIANT
#define WL_CELL_VARIANT 0
#endif

namespace wl {

__global__ void __launch_bounds__(256) k_probe_mad(uint32_t iters, uint32_t seed, uint32_t* out) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8 + k;
    const uint32_t m = 0x9E3779B1u ^ seed, c = 0x7F4A7C15u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) x ^= a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

__global__ void __launch_bounds__(256) k_probe_madhi(uint32_t iters, uint32_t seed, uint32_t* out) {
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8 + k;
    const uint32_t m = 0x9E3779B1u ^ seed, c = 0x7F4A7C15u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) asm volatile("mad.hi.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) x ^= a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

__global__ void __launch_bounds__(256) k_probe_madwide(uint32_t iters, uint32_t seed, uint32_t* out) {
    uint64_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = seed + threadIdx.x * 8 + k;
    const uint32_t m = 0x9E3779B1u ^ seed, c = 0x7F4A7C15u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                uint32_t lo = (uint32_t)a[k];
                asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(a[k]) : "r"(lo), "r"(m));
            }
        }
    }
    uint32_t x = c;
#pragma unroll
    for (int k = 0; k < 8; ++k) x ^= (uint32_t)a[k] ^ (uint32_t)(a[k] >> 32);
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

// MODE 0: fma.rn.f64 only; 1: mad.lo.u32 + fma.rn.f64; 2: mad.wide.u32 + fma.rn.f64
template <int MODE>
__global__ void __launch_bounds__(256) k_probe_dfma(uint32_t iters, uint32_t seed, uint32_t* out) {
    double d[8];
    uint32_t a[8];
    uint64_t w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        d[k] = 1.0 + (double)(threadIdx.x + k) * 1e-3;
        a[k] = seed + threadIdx.x * 8 + k;
        w[k] = a[k];
    }
    const double dm = 0.9999999, dc = 1e-3;
    const uint32_t m = 0x9E3779B1u ^ seed, c = 0x7F4A7C15u;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                asm volatile("fma.rn.f64 %0, %0, %1, %2;" : "+d"(d[k]) : "d"(dm), "d"(dc));
                if (MODE == 1) asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(c));
                if (MODE == 2) {
                    uint32_t lo = (uint32_t)w[k];
                    asm volatile("mad.wide.u32 %0, %1, %2, %0;" : "+l"(w[k]) : "r"(lo), "r"(m));
                }
            }
        }
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) x ^= (uint32_t)__double2uint_rz(d[k]) ^ a[k] ^ (uint32_t)w[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

// An exact Montgomery cell in FP64 for n = p^2 < 2^62: x <- x * q * 2^-42 (mod n)
// with x held as three 21-bit limbs in doubles (value below 2^52 + n, so
// below 2^63), two radix-2^21 reduction steps.  Every product and partial sum
// is an integer below 2^53, so each operation is exact; floor(t * 2^-21) is a
// round-down fma against 2^52.  Checked bit for bit against 128-bit
// arithmetic on 4,096 moduli x 1,000 cells.
struct ResF { double x0, x1, x2; };
struct ModF { double n0, n1, n2, ninv; };        // 21-bit limbs of n, -n^-1 mod 2^21

__device__ __forceinline__ double floor_sc(double t) { return __fma_rd(t, 0x1p-21, 0x1p52) - 0x1p52; }

__device__ __forceinline__ void cell_fp(ResF& x, double q, const ModF& m) {
    const double t0 = x.x0 * q, t1 = x.x1 * q, t2 = x.x2 * q;
    const double a0 = floor_sc(t0);
    const double b0 = fma(a0, -0x1p21, t0);
    const double p1 = b0 * m.ninv;
    const double m1 = fma(floor_sc(p1), -0x1p21, p1);
    const double c0 = fma(m1, m.n0, b0) * 0x1p-21;
    const double u0 = (fma(m1, m.n1, t1) + a0) + c0;
    const double u1 = fma(m1, m.n2, t2);
    const double a1 = floor_sc(u0);
    const double b1 = fma(a1, -0x1p21, u0);
    const double p2 = b1 * m.ninv;
    const double m2 = fma(floor_sc(p2), -0x1p21, p2);
    const double c1 = fma(m2, m.n0, b1) * 0x1p-21;
    const double v0 = (fma(m2, m.n1, u1) + a1) + c1;
    const double v1 = m2 * m.n2;
    const double k0 = floor_sc(v0);
    x.x0 = fma(k0, -0x1p21, v0);
    const double w = k0 + v1;
    x.x2 = floor_sc(w);
    x.x1 = fma(x.x2, -0x1p21, w);
}

// MODE 1: FP64 cells only; 2: warps 0-5 integer cells, warps 6-7 FP64 cells
template <int MODE>
__global__ void __launch_bounds__(256, 4) k_probe_cellfp(uint32_t iters, uint32_t seed, uint32_t* out) {
    const uint64_t n = 1000000007ull * 1000000007ull;   // (10^9 + 7)^2
    uint32_t x = (uint32_t)n;
    for (int k = 0; k < 5; ++k) x *= 2u - (uint32_t)n * x;
    const uint32_t ninv = 0u - x;
    const bool fp = MODE == 1 || (threadIdx.x >> 5) >= 6;
    uint32_t q = 0x10001u + 2 * threadIdx.x + seed;
    uint32_t o = 0;
    if (fp) {
        ModF m;
        m.n0 = (double)(n & 0x1FFFFF); m.n1 = (double)((n >> 21) & 0x1FFFFF); m.n2 = (double)(n >> 42);
        m.ninv = (double)(ninv & 0x1FFFFF);
        ResF f[2];
        for (int j = 0; j < 2; ++j) { f[j].x0 = threadIdx.x + j; f[j].x1 = 1; f[j].x2 = 0; }
        for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                cell_fp(f[0], (double)q, m);
                cell_fp(f[1], (double)q, m);
                q += 2;
            }
        }
        o = (uint32_t)(f[0].x0 + f[1].x1);
    } else {
        uint32_t nn[2] = { (uint32_t)n, (uint32_t)(n >> 32) };
        Res<2> r[2];
        for (int j = 0; j < 2; ++j) { r[j].w[0] = threadIdx.x + j; r[j].w[1] = 1; }
        for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                cell_w<2>(r[0], q, nn, ninv);
                cell_w<2>(r[1], q, nn, ninv);
                q += 2;
            }
        }
        o = r[0].w[0] ^ r[1].w[1];
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = o;
}

template <int L, int V>
__global__ void __launch_bounds__(256) k_probe_cell(uint32_t iters, uint32_t seed, uint32_t* out) {
    // a fixed odd modulus n < 2^(32L-2) and its -n^-1 mod 2^32
    uint32_t n[L];
#pragma unroll
    for (int k = 0; k < L; ++k) n[k] = 0x9E3779B9u ^ (seed * (k + 1));
    n[0] |= 1u;
    n[L - 1] &= 0x3FFFFFFFu;
    uint32_t x = n[0];
    for (int k = 0; k < 5; ++k) x *= 2u - n[0] * x;
    const uint32_t ninv = 0u - x;
    Res<L> r[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) set_small<L>(r[j], threadIdx.x + 1 + j);
    uint32_t q = 0x10001u + 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                if (V == 0) cell(r[j], q, n, ninv);
                else if (V == 1) cell_w<L>(r[j], q, n, ninv);
                else cell_h<L>(r[j], q, n, ninv);
            }
            q += 2;
        }
    }
    uint32_t o = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int k = 0; k < L; ++k) o ^= r[j].w[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = o;
}

}  // namespace wl

using namespace wl;

extern "C" int wl_probe(int device, int which, double* rate) {
    if (!rate) return WL_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return WL_ERR_CUDA;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const unsigned blocks = (unsigned)sms * 8, threads = 256;
    uint32_t* out = nullptr;
    if (cudaMalloc(&out, (size_t)blocks * threads * 4) != cudaSuccess) return WL_ERR_NOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double per_iter = 0;     // operations per thread per iteration
    uint32_t iters = 0;
    auto launch = [&](uint32_t it) {
        switch (which) {
            case WL_PROBE_MAD: k_probe_mad<<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_MADHI: k_probe_madhi<<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_CELL2: k_probe_cell<2, WL_CELL_VARIANT><<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_CELL3: k_probe_cell<3, WL_CELL_VARIANT><<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_CELL4: k_probe_cell<4, WL_CELL_VARIANT><<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_MADWIDE: k_probe_madwide<<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_DFMA: k_probe_dfma<0><<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_MAD_DFMA: k_probe_dfma<1><<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_MADWIDE_DFMA: k_probe_dfma<2><<<blocks, threads>>>(it, 12345u, out); break;
            case WL_PROBE_CELL2_FP64: k_probe_cellfp<1><<<blocks, threads>>>(it, 0u, out); break;
            case WL_PROBE_CELL2_MIX: k_probe_cellfp<2><<<blocks, threads>>>(it, 0u, out); break;
            case 100: k_probe_cell<2, 0><<<blocks, threads>>>(it, 12345u, out); break;
            case 101: k_probe_cell<2, 1><<<blocks, threads>>>(it, 12345u, out); break;
            case 102: k_probe_cell<2, 2><<<blocks, threads>>>(it, 12345u, out); break;
            case 110: k_probe_cell<3, 0><<<blocks, threads>>>(it, 12345u, out); break;
            case 111: k_probe_cell<3, 1><<<blocks, threads>>>(it, 12345u, out); break;
            case 112: k_probe_cell<3, 2><<<blocks, threads>>>(it, 12345u, out); break;
            case 120: k_probe_cell<4, 0><<<blocks, threads>>>(it, 12345u, out); break;
            case 121: k_probe_cell<4, 1><<<blocks, threads>>>(it, 12345u, out); break;
            default: k_probe_cell<4, 2><<<blocks, threads>>>(it, 12345u, out); break;
        }
    };
    if (which == WL_PROBE_MAD || which == WL_PROBE_MADHI || which == WL_PROBE_MADWIDE || which == WL_PROBE_DFMA) {
        per_iter = 32;
        iters = 200000;
    } else if (which == WL_PROBE_MAD_DFMA || which == WL_PROBE_MADWIDE_DFMA) {
        per_iter = 64;   // both kinds of operation
        iters = 100000;
    }
    else if (which == WL_PROBE_CELL2_FP64 || which == WL_PROBE_CELL2_MIX) {
        per_iter = 16;   // 2 rows x 8 cells
        iters = 4000;
    }
    else if ((which >= WL_PROBE_CELL2 && which <= WL_PROBE_CELL4) || (which >= 100 && which <= 122)) {
        per_iter = 16; iters = 20000;
    }
    else { cudaFree(out); return WL_ERR_ARG; }
    launch(iters / 10);   // warm-up
    cudaEventRecord(e0);
    launch(iters);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess || ms <= 0) return WL_ERR_CUDA;
    *rate = (double)blocks * threads * per_iter * iters / (ms * 1e-3);
    return 0;
}
