// wl_noalloc.cu -- the column product of one class without any device allocation.
//
// wl_column_product_noalloc() runs the same kernels as the engine's capped
// sweep (k_setup_rows, k_sweep, k_finish) for caller-owned input and output
// buffers, with every intermediate (row constants, split partial products,
// split deficits, launch descriptors) in one fixed, file-scope device array.
// It is for callers that cannot allocate device memory while they run: hosts
// that reserve all device memory in their own pool at start-up and forbid
// cudaMalloc afterwards (cudaMalloc/cudaFree synchronise the device and fail
// once the pool holds the memory), and real-time paths that must not take the
// driver's allocation lock.
//
// The scratch array is allocated by the CUDA runtime when the library is
// loaded, on every GPU that loads it, and held until the process exits.
#include "wilson.h"
#include "wl_internal.h"

namespace {

constexpr uint32_t NA_MAX_ROWS = WL_NOALLOC_MAX_ROWS;
constexpr uint32_t NA_MAX_PARTIALS = WL_NOALLOC_MAX_PARTIALS;   // splits x rows
constexpr uint32_t NA_MAX_SPLITS = 1024;
constexpr uint32_t NA_MAX_ITEMS = (NA_MAX_ROWS / 256) * NA_MAX_SPLITS + NA_MAX_SPLITS;

// byte offsets of the scratch regions (each 256-byte aligned)
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t OFF_BUCKET = 0;
constexpr size_t OFF_ITEMS = align256(OFF_BUCKET + sizeof(wl::Bucket));
constexpr size_t OFF_INFO = align256(OFF_ITEMS + sizeof(wl::SweepItem) * NA_MAX_ITEMS);
constexpr size_t OFF_MODS = align256(OFF_INFO + sizeof(wl::RowInfo) * NA_MAX_ROWS);
constexpr size_t OFF_OUT = align256(OFF_MODS + sizeof(wl::RowMod) * NA_MAX_ROWS);
constexpr size_t OFF_DEFS = align256(OFF_OUT + sizeof(wl::RowOut) * NA_MAX_ROWS);
constexpr size_t OFF_PART = align256(OFF_DEFS + sizeof(wl::Deficit) * NA_MAX_SPLITS);
constexpr size_t SCRATCH_BYTES = align256(OFF_PART + 16ull * NA_MAX_PARTIALS);
static_assert(SCRATCH_BYTES <= WL_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

}  // namespace

// The scratch itself: shared by every call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[WL_NOALLOC_SCRATCH_BYTES];

namespace {

// Fill the bucket, the sweep descriptors and the row records from the
// caller's primes (so that no host-to-device copy is needed either).
__global__ void k_noalloc_prep(const uint64_t* __restrict__ primes, uint32_t nrows, uint64_t T, uint32_t ncols,
                               uint32_t nsplit, uint32_t L, uint32_t tps, uint32_t nitems) {
    unsigned char* base = g_noalloc_scratch;
    wl::Bucket* bk = reinterpret_cast<wl::Bucket*>(base + OFF_BUCKET);
    wl::SweepItem* items = reinterpret_cast<wl::SweepItem*>(base + OFF_ITEMS);
    wl::RowInfo* info = reinterpret_cast<wl::RowInfo*>(base + OFF_INFO);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        wl::Bucket b;
        b.T = T;
        b.part_base = 0;
        b.ncols = ncols;
        b.row_begin = 0;
        b.nrows = nrows;
        b.nsplit = nsplit;
        b.def_base = 0;
        b.L = L;
        b.type = 0;
        b.range = 0;
        b.cdense = 0;
        b.ndense = 0;
        b.dstart = 0;
        b.cbase = 0;
        *bk = b;
    }
    if (i < nitems) {
        wl::SweepItem it;
        it.bucket = 0;
        it.tps = tps;
        if (tps == 256) {
            it.row0 = (i / nsplit) * 256;
            it.split0 = i % nsplit;
        } else {
            it.row0 = 0;
            it.split0 = i * (256 / tps);
        }
        items[i] = it;
    }
    if (i < nrows) {
        wl::RowInfo r;
        r.p = primes[i];
        r.Tp = T;
        r.bucket = 0;
        r.it_begin = 0;
        r.it_count = 0;
        r.type = 0;
        info[i] = r;
    }
}

__global__ void k_noalloc_out(uint32_t nrows, uint64_t* __restrict__ s0s1) {
    const wl::RowOut* out = reinterpret_cast<const wl::RowOut*>(g_noalloc_scratch + OFF_OUT);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nrows) {
        s0s1[2 * i] = out[i].s0;
        s0s1[2 * i + 1] = out[i].s1;
    }
}

// device address of the scratch array, resolved once per device
constexpr int NA_MAX_DEVICES = 64;
unsigned char* g_scratch_addr[NA_MAX_DEVICES] = {};
int g_sms[NA_MAX_DEVICES] = {};

}  // namespace

extern "C" int wl_column_product_noalloc(const uint64_t* primes, uint32_t nrows, uint64_t p_bound, uint64_t T,
                                         const uint32_t* cols, uint32_t ncols, uint64_t* s0s1, void* stream) {
    if (!primes || !s0s1 || nrows == 0 || T == 0 || p_bound > WL_MAXP + 1 || p_bound < 6) return WL_ERR_ARG;
    if (ncols > 0 && !cols) return WL_ERR_ARG;
    if (nrows > NA_MAX_ROWS) return WL_ERR_TOO_LARGE;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return WL_ERR_CUDA;
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            return WL_ERR_CUDA;
        }
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
        g_sms[dev] = sms;
        g_scratch_addr[dev] = static_cast<unsigned char*>(ptr);
    }
    unsigned char* base = g_scratch_addr[dev];
    const int L = p_bound - 1 < (1ull << 31) ? 2 : (p_bound - 1 < (1ull << 47) ? 3 : 4);

    // split the columns so that about 2 x (SMs x 2048) threads work, each
    // split at least 2048 columns long, within the scratch limits
    uint32_t nsplit = 1;
    if (ncols > 0) {
        const uint64_t want = ((uint64_t)g_sms[dev] * 4096 + nrows - 1) / nrows;
        uint64_t s = want;
        s = s < ncols / 2048 ? s : ncols / 2048;
        s = s < NA_MAX_SPLITS ? s : NA_MAX_SPLITS;
        s = s < NA_MAX_PARTIALS / nrows ? s : NA_MAX_PARTIALS / nrows;
        nsplit = s > 0 ? (uint32_t)s : 1;
    }
    if ((uint64_t)nsplit * nrows > NA_MAX_PARTIALS) return WL_ERR_TOO_LARGE;
    uint32_t tps, nitems;
    if (nrows >= 256) {
        tps = 256;
        nitems = ((nrows + 255) / 256) * nsplit;
    } else {
        tps = 1;
        while (tps < nrows) tps <<= 1;
        const uint32_t per = 256 / tps;
        nitems = (nsplit + per - 1) / per;
    }
    if (nitems > NA_MAX_ITEMS) return WL_ERR_TOO_LARGE;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t prep_threads = nitems > nrows ? nitems : nrows;
    k_noalloc_prep<<<(prep_threads + 255) / 256, 256, 0, st>>>(primes, nrows, T, ncols, nsplit, (uint32_t)L, tps,
                                                                nitems);
    wl::Bucket* bk = reinterpret_cast<wl::Bucket*>(base + OFF_BUCKET);
    wl::SweepItem* items = reinterpret_cast<wl::SweepItem*>(base + OFF_ITEMS);
    wl::RowInfo* info = reinterpret_cast<wl::RowInfo*>(base + OFF_INFO);
    wl::RowMod* mods = reinterpret_cast<wl::RowMod*>(base + OFF_MODS);
    wl::RowOut* out = reinterpret_cast<wl::RowOut*>(base + OFF_OUT);
    wl::Deficit* defs = reinterpret_cast<wl::Deficit*>(base + OFF_DEFS);
    uint4* part = reinterpret_cast<uint4*>(base + OFF_PART);
    wl::launch_setup_rows(info, nrows, mods, st);
    wl::launch_sweep(1, L, 1, nitems, bk, items, mods, cols, part, defs, st);
    wl::launch_finish(L, bk, info, mods, part, defs, 1, nullptr, 0, nrows, 0, out, st);
    k_noalloc_out<<<(nrows + 255) / 256, 256, 0, st>>>(nrows, s0s1);
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    return 0;
}
