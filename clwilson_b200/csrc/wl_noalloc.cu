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
//
// The input contract is checked on the device, since the inputs live there:
// a row whose prime is even, below 5 or not below p_bound, and every row when
// the columns are not ascending primes in [2, T], get s0 = s1 = UINT64_MAX.
#include <atomic>
#include <mutex>

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
constexpr size_t OFF_FLAG = align256(OFF_DEFS + sizeof(wl::Deficit) * NA_MAX_SPLITS);
constexpr size_t OFF_PART = align256(OFF_FLAG + sizeof(uint32_t));
constexpr size_t SCRATCH_BYTES = align256(OFF_PART + 16ull * NA_MAX_PARTIALS);
constexpr uint32_t BAD_ROW = 0xFFFFFFFFu;   // RowInfo.type of a row whose prime breaks the contract
static_assert(SCRATCH_BYTES <= WL_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds the stated size");

}  // namespace

// The scratch itself: shared by every call on a device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[WL_NOALLOC_SCRATCH_BYTES];

namespace {

// The column-contract flag starts at zero in every call (the array keeps the
// previous call's contents).
__global__ void k_noalloc_clear() {
    *reinterpret_cast<uint32_t*>(g_noalloc_scratch + OFF_FLAG) = 0;
}

// Fill the bucket, the sweep descriptors and the row records from the
// caller's primes (so that no host-to-device copy is needed either), and
// check the inputs: each prime odd in [5, p_bound), the columns ascending in
// [2, T].
__global__ void k_noalloc_prep(const uint64_t* __restrict__ primes, uint32_t nrows, uint64_t p_bound, uint64_t T,
                               const uint32_t* __restrict__ cols, uint32_t ncols, uint32_t nsplit, uint32_t L,
                               uint32_t tps, uint32_t nitems) {
    unsigned char* base = g_noalloc_scratch;
    wl::Bucket* bk = reinterpret_cast<wl::Bucket*>(base + OFF_BUCKET);
    wl::SweepItem* items = reinterpret_cast<wl::SweepItem*>(base + OFF_ITEMS);
    wl::RowInfo* info = reinterpret_cast<wl::RowInfo*>(base + OFF_INFO);
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t nthreads = gridDim.x * blockDim.x;
    bool cols_ok = true;
    for (uint32_t j = i; j < ncols; j += nthreads) {
        const uint32_t q = cols[j];
        cols_ok &= q >= 2u && (uint64_t)q <= T && (j == 0 || cols[j - 1] < q);
    }
    if (!cols_ok) *reinterpret_cast<uint32_t*>(base + OFF_FLAG) = 1u;
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
        const bool ok = (r.p & 1) && r.p >= 5 && r.p < p_bound;
        r.type = ok ? 0u : BAD_ROW;
        info[i] = r;
    }
}

__global__ void k_noalloc_out(uint32_t nrows, uint64_t* __restrict__ s0s1) {
    const wl::RowOut* out = reinterpret_cast<const wl::RowOut*>(g_noalloc_scratch + OFF_OUT);
    const wl::RowInfo* info = reinterpret_cast<const wl::RowInfo*>(g_noalloc_scratch + OFF_INFO);
    const bool cols_bad = *reinterpret_cast<const uint32_t*>(g_noalloc_scratch + OFF_FLAG) != 0;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nrows) {
        const bool bad = cols_bad || info[i].type == BAD_ROW;
        s0s1[2 * i] = bad ? ~0ull : out[i].s0;
        s0s1[2 * i + 1] = bad ? ~0ull : out[i].s1;
    }
}

// device address of the scratch array, resolved once per device; the first
// call on a device takes the mutex, later ones only read the atomic
constexpr int NA_MAX_DEVICES = 64;
std::atomic<unsigned char*> g_scratch_addr[NA_MAX_DEVICES];
int g_sms[NA_MAX_DEVICES] = {};
std::mutex g_resolve_mutex;

int resolve_scratch(int dev, unsigned char** base, int* sms) {
    unsigned char* b = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!b) {
        std::lock_guard<std::mutex> lock(g_resolve_mutex);
        b = g_scratch_addr[dev].load(std::memory_order_relaxed);
        if (!b) {
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr) {
                cudaGetLastError();
                return WL_ERR_CUDA;
            }
            int n = 0;
            if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
                cudaGetLastError();
                n = 148;
            }
            g_sms[dev] = n;
            b = static_cast<unsigned char*>(ptr);
            g_scratch_addr[dev].store(b, std::memory_order_release);
        }
    }
    *base = b;
    *sms = g_sms[dev];
    return 0;
}

}  // namespace

extern "C" int wl_column_product_noalloc(const uint64_t* primes, uint32_t nrows, uint64_t p_bound, uint64_t T,
                                         const uint32_t* cols, uint32_t ncols, uint64_t* s0s1, void* stream) {
    if (!primes || !s0s1 || nrows == 0 || T == 0 || p_bound > WL_MAXP + 1 || p_bound < 6) return WL_ERR_ARG;
    if (ncols > 0 && !cols) return WL_ERR_ARG;
    if (nrows > NA_MAX_ROWS) return WL_ERR_TOO_LARGE;
    // an error left by the caller's earlier CUDA work stays the caller's: report it, launch nothing
    if (cudaPeekAtLastError() != cudaSuccess) return WL_ERR_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return WL_ERR_CUDA;
    unsigned char* base = nullptr;
    int sms = 0;
    if (resolve_scratch(dev, &base, &sms)) return WL_ERR_CUDA;
    const int L = p_bound - 1 < (1ull << 31) ? 2 : (p_bound - 1 < (1ull << 47) ? 3 : 4);

    // split the columns so that about 2 x (SMs x 2048) threads work, each
    // split at least 2048 columns long, within the scratch limits
    uint32_t nsplit = 1;
    if (ncols > 0) {
        const uint64_t want = ((uint64_t)sms * 4096 + nrows - 1) / nrows;
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
    // each launch's own error is checked right after it
    k_noalloc_clear<<<1, 1, 0, st>>>();
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    k_noalloc_prep<<<(prep_threads + 255) / 256, 256, 0, st>>>(primes, nrows, p_bound, T, cols, ncols, nsplit,
                                                                (uint32_t)L, tps, nitems);
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    wl::Bucket* bk = reinterpret_cast<wl::Bucket*>(base + OFF_BUCKET);
    wl::SweepItem* items = reinterpret_cast<wl::SweepItem*>(base + OFF_ITEMS);
    wl::RowInfo* info = reinterpret_cast<wl::RowInfo*>(base + OFF_INFO);
    wl::RowMod* mods = reinterpret_cast<wl::RowMod*>(base + OFF_MODS);
    wl::RowOut* out = reinterpret_cast<wl::RowOut*>(base + OFF_OUT);
    wl::Deficit* defs = reinterpret_cast<wl::Deficit*>(base + OFF_DEFS);
    uint4* part = reinterpret_cast<uint4*>(base + OFF_PART);
    wl::launch_setup_rows(info, nrows, mods, st);
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    wl::launch_sweep(1, L, 1, nitems, bk, items, mods, cols, part, defs, st);
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    wl::launch_finish(L, bk, info, mods, part, defs, 1, nullptr, 0, nrows, 0, out, st);
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    k_noalloc_out<<<(nrows + 255) / 256, 256, 0, st>>>(nrows, s0s1);
    if (cudaGetLastError() != cudaSuccess) return WL_ERR_CUDA;
    return 0;
}
