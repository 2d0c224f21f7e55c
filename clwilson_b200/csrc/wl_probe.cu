// wl_probe.cu -- integer-pipe microbenchmarks that set the roofline of the
// column sweep (include/wilson_probe.h).
//
//   WL_PROBE_MAD     mad.lo.u32, 8 independent chains per thread
//   WL_PROBE_MADHI   mad.hi.u32, 8 independent chains per thread
//   WL_PROBE_CELL2/3/4  the sweep's cell step (wl_arith.cuh) at L = 2, 3, 4,
//                    4 independent rows per thread, operands in registers
//   WL_PROBE_MADWIDE mad.wide.u32, 8 independent chains per thread
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
    if (which == WL_PROBE_MAD || which == WL_PROBE_MADHI || which == WL_PROBE_MADWIDE) {
        per_iter = 32;
        iters = 200000;
    } else if ((which >= WL_PROBE_CELL2 && which <= WL_PROBE_CELL4) || (which >= 100 && which <= 122)) {
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
