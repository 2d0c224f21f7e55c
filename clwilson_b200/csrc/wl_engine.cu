// wl_engine.cu -- host engine and C ABI of the Wilson-prime search.
//
// One search (or a batch of ranges) runs as:
//   1. test primes: deterministic Miller-Rabin over each window [pmin, pmax)
//      into an ordered list on the device (k_window_primes_multi, k_compact), all
//      ranges in one launch each;
//   2. classification into (range, class) buckets with the reference's shared
//      class target = the target of the first prime of the class
//      (cl_wilson.cpp:1549-1586);
//   3. the column cache: every prime below the largest needed column, sieved
//      once per context on the device and kept resident (k_sieve_segments);
//   4. the column sweep over splits of each bucket's columns (k_sweep where
//      exponents change rarely, k_sweep_dense where they change at almost
//      every prime; columns above 2^32 from a windowed sieve, run_big_columns),
//      split products merged per row (k_merge*), the consecutive-integer tail
//      (k_iterate), and the class lift + quotient (k_finish);
//   5. results.txt lines (ascending p) and the checksum on the host
//      (cl_wilson.cpp:872-900).
// A batch (wl_batch) issues the device work of step 4 -- every sweep launch
// of both streams, the merges, the tail and the lift -- as one CUDA graph,
// captured from the two streams and launched once (ChainGraph).
// Also here: searches in pieces (q_lo / init of run_ranges) and the
// row-wise product of pieces (wl_rows_product), kernel tuning, and the C ABI;
// serving sessions are in wl_serve.cu.
#include <algorithm>
#include <cerrno>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "wilson.h"
#include "wl_internal.h"
#include "wl_host.h"
#include "wl_plan.h"

using namespace wl;

namespace {

uint64_t pi_upper_bound(uint64_t x) {   // Rosser-Schoenfeld: pi(x) < 1.25506 x / ln x for x > 1
    if (x < 64) return 64;
    return (uint64_t)(1.2551 * (double)x / std::log((double)x)) + 64;
}

}  // namespace

// Sweep kernel choices measured best on B200 (the digit-sorted dense kernel
// with 3-bit windows and its buckets in shared memory, 4 CTAs per SM, H every
// 8 columns; the wide-product cell, two rows per
// thread for large buckets; CTA-per-row merges from 64 splits).  The
// environment overrides them for experiments: WL_CELL_VARIANT, WL_DENSE_SORT,
// WL_DENSE_CFG (42: 4-bit windows), WL_DENSE_HSTEP, WL_DENSE_KERNEL (a
// WL_DENSE_* value); wl_autotune measures them.
static void default_tuning(wl_ctx* c) {
    const char* e;
    int kernel = DENSE_SMEM_W3, hstep = 8;
    const int sort = (e = getenv("WL_DENSE_SORT")) ? atoi(e) : 1;
    const int cfg = (e = getenv("WL_DENSE_CFG")) ? atoi(e) : 0;
    if ((e = getenv("WL_DENSE_HSTEP")) && atoi(e) > 0) hstep = atoi(e);
    if (sort) kernel = cfg == 42 ? DENSE_SORTED_W4 : DENSE_SMEM_W3;
    const int forced = (e = getenv("WL_DENSE_KERNEL")) ? atoi(e) : -1;   // a WL_DENSE_* value
    for (int L = 2; L <= 4; ++L) {
        int k = kernel;
        if (!sort) k = (cfg == 42 || (cfg == 0 && L != 4)) ? DENSE_SWITCH_W4 : DENSE_SWITCH_W3;
        if (forced >= 0 && forced <= DENSE_SORTED_W3_2CTA) k = forced;
        c->tune.sparse_variant[L - 2] = c->cell_variant;
        c->tune.sparse_rpt[L - 2] = 2;
        c->tune.dense_kernel[L - 2] = k;
        c->tune.dense_hstep[L - 2] = hstep;
        c->tune.ms[L - 2] = 0;
    }
    c->tune.merge_cta_min = 64;
}

// ---------------------------------------------------------------------------
// column cache
// ---------------------------------------------------------------------------

int ensure_columns(wl_ctx* c, uint64_t limit) {
    if (limit <= c->col_limit) return 0;
    const uint64_t top = 1ull << 32;
    if (limit > top) return WL_ERR_UNSUPPORTED;
    uint64_t nl = std::max<uint64_t>(limit, std::min<uint64_t>(top, 2 * c->col_limit));
    nl = (nl + SEG_SPAN - 1) / SEG_SPAN * SEG_SPAN;
    if (nl > top) nl = top;
    const uint32_t nseg = (uint32_t)(nl / SEG_SPAN);
    RC(ensure(c->bitmap, (size_t)nseg * SEG_WORDS * 4));
    RC(ensure(c->segcount, (size_t)nseg * 4));
    RC(ensure(c->offsets, (size_t)(nseg + 1) * 8));
    RC(ensure(c->cols, (size_t)pi_upper_bound(nl) * 4 + 64));
    cudaEventRecord(c->ev[6], c->st);
    launch_sieve_segments(0, nseg, nl, as<uint32_t>(c->base), c->nbase, as<uint32_t>(c->bitmap),
                          as<uint32_t>(c->segcount), c->st);
    launch_scan_counts(as<uint32_t>(c->segcount), nseg, 1, as<uint64_t>(c->offsets), c->st);
    launch_compact(nseg, 0, as<uint32_t>(c->bitmap), as<uint64_t>(c->offsets), as<uint32_t>(c->cols), nullptr,
                   c->st);
    c->launches += 3;
    static const uint32_t two = 2;
    CK(cudaMemcpyAsync(as<uint32_t>(c->cols), &two, 4, cudaMemcpyHostToDevice, c->st));
    uint64_t total = 0;
    CK(cudaMemcpyAsync(&total, as<uint64_t>(c->offsets) + nseg, 8, cudaMemcpyDeviceToHost, c->st));
    cudaEventRecord(c->ev[7], c->st);
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    float ms = 0;
    cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
    c->ms_sieve += ms;
    c->sieve_ints += nl;
    // bitmap written, then read by the write-out; segment counts written and
    // read; offsets written and read; the column table written
    c->sieve_bytes += 2ull * nseg * SEG_WORDS * 4 + 2ull * nseg * 4 + 2ull * (nseg + 1) * 8 + total * 4;
    c->ncols = total;
    c->col_limit = nl;
    // the exact products of the table's aligned column groups
    c->ngroups = 0;
    const uint64_t ng = total / COL_GROUP;
    RC(ensure(c->gprod, (size_t)ng * COL_GROUP * 4 + 16));
    RC(ensure(c->gk, (size_t)ng + 16));
    launch_group_products(as<uint32_t>(c->cols), ng, as<uint32_t>(c->gprod), as<uint8_t>(c->gk), c->st);
    c->launches++;
    c->ngroups = ng;
    return 0;
}

// ---------------------------------------------------------------------------
// the search pipeline over a set of ranges
// ---------------------------------------------------------------------------


struct HostBucket {
    uint32_t range, type, L;
    uint64_t T;
    std::vector<uint64_t> primes;   // ascending
    std::vector<uint32_t> src;      // index into the range's prime list
};

struct RunOut {
    std::vector<wl_row> rows;             // all rows, ranges in order, ascending p within a range
    std::vector<uint64_t> range_row_off;  // rows of range r: [off[r], off[r+1])
    std::vector<uint64_t> range_targets;  // 3 per range
    uint64_t pi_maxtarget = 0, cells = 0, tail = 0;
};

// The device chain of a batch as one CUDA graph: stream capture of the main
// stream (the dense sweep's stream joins it through the fork event and is
// joined back), then one instantiation and one launch.  Early returns while
// capturing end the capture (the partial graph is dropped); the graph and
// its executable are destroyed with this object, which outlives the call's
// final stream synchronisation.
struct ChainGraph {
    cudaStream_t capturing = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t nodes = 0;
    double ms_build = 0;   // host time of end of capture + instantiation
    int begin(cudaStream_t st) {
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        capturing = st;
        return 0;
    }
    // event records inside the capture become event-record nodes, so the
    // phase timings still come from the graph's own run
    cudaError_t record(cudaEvent_t e, cudaStream_t st) const {
        return capturing ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal) : cudaEventRecord(e, st);
    }
    int launch() {
        const auto t0 = std::chrono::steady_clock::now();
        cudaStream_t st = capturing;
        capturing = nullptr;
        CK(cudaStreamEndCapture(st, &graph));
        CK(cudaGraphGetNodes(graph, nullptr, &nodes));
        CK(cudaGraphInstantiate(&exec, graph, 0));
        ms_build = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        CK(cudaGraphLaunch(exec, st));
        return 0;
    }
    ~ChainGraph() {
        if (capturing) {
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(capturing, &g);
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();   // the call already returns its own error
        }
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
    }
};

// ---------------------------------------------------------------------------
// columns above 2^32: windows of the number line are sieved on the device,
// swept (k_sweep64) and merged into a per-row accumulator (k_merge) that
// k_finish folds in.  Runs on its own stream; the main stream waits for it.
// ---------------------------------------------------------------------------

static uint64_t isqrt_u64(uint64_t n) {
    uint64_t r = (uint64_t)std::sqrt((long double)n);
    while (r * r > n) --r;
    while ((r + 1) * (r + 1) <= n) ++r;
    return r;
}

static int run_big_columns(wl_ctx* c, const std::vector<Bucket>& db, const std::vector<RowInfo>& ri, uint32_t nrows,
                           const std::vector<uint64_t>& keys_host_order, uint64_t big_need, uint64_t maxt0, bool full,
                           uint64_t qcap, uint64_t q_lo, uint64_t* pi_big) {
    (void)keys_host_order;
    cudaStream_t s3 = c->st3;
    CK(cudaStreamWaitEvent(s3, c->rows_ready, 0));   // row tables and moduli
    CK(cudaEventRecord(c->big0, s3));
    const uint64_t LO = 1ull << 32;
    const uint64_t WIN = 1ull << 33;
    const uint32_t SPC = 8;
    // per-bucket upper key (device order)
    std::vector<uint64_t> bkey(db.size());
    for (size_t b = 0; b < db.size(); ++b) {
        uint64_t key = db[b].T;
        if (!full && qcap - 1 < key) key = qcap - 1;
        bkey[b] = key;
    }
    // sieving primes: odd primes 67 .. isqrt(big_need - 1) from the column cache
    // (cols[0] = 2, cols[1..17] = 3..61, cols[18] = 67)
    const uint64_t root = isqrt_u64(big_need - 1);
    uint64_t nroot = 0;
    {
        RC(ensure(c->wkeys, 16));
        RC(ensure(c->wcounts, 16));
        CK(cudaMemcpyAsync(c->wkeys.p, &root, 8, cudaMemcpyHostToDevice, s3));
        launch_count_leq(as<uint32_t>(c->cols), c->ncols, as<uint64_t>(c->wkeys), 1, as<uint64_t>(c->wcounts), s3);
        c->launches++;
        CK(cudaMemcpyAsync(&nroot, c->wcounts.p, 8, cudaMemcpyDeviceToHost, s3));
        CK(cudaStreamSynchronize(s3));
    }
    const uint32_t nbase = nroot > 18 ? (uint32_t)(nroot - 18) : 0;
    const uint32_t* base = as<uint32_t>(c->cols) + 18;

    // running per-row accumulators (raw 1) and per-bucket deficits (0)
    RC(ensure(c->bacc, (size_t)nrows * 16 + 16));
    RC(ensure(c->bdef, db.size() * sizeof(Deficit) + 16));
    launch_acc_init(nrows, (uint32_t)db.size(), as<uint4>(c->bacc), as<Deficit>(c->bdef), s3);
    c->launches++;
    // row groups by limb width (rows are ordered by width)
    std::vector<std::pair<int, std::pair<uint32_t, uint32_t>>> lgroups;
    for (uint32_t rb = 0; rb < nrows;) {
        const int L = (int)db[ri[rb].bucket].L;
        uint32_t re = rb;
        while (re < nrows && (int)db[ri[re].bucket].L == L) ++re;
        lgroups.push_back({ L, { rb, re } });
        rb = re;
    }
    const double target_threads = (double)c->sms * 2048.0 * 4.0;
    *pi_big = 0;
    // device: per-bucket keys for the bitmap sweep, the pi(maxtarget) counter
    RC(ensure(c->wkeys, db.size() * 8 + 16));
    RC(ensure(c->wcounts, 16));
    CK(cudaMemcpyAsync(c->wkeys.p, bkey.data(), db.size() * 8, cudaMemcpyHostToDevice, s3));
    CK(cudaMemsetAsync(c->wcounts.p, 0, 8, s3));
    std::vector<Bucket> wb(db);
    std::vector<SweepItem> all;
    for (uint64_t w0 = LO; w0 < big_need; w0 += WIN) {
        const uint64_t w1 = std::min(w0 + WIN, big_need);
        if (w1 <= q_lo) continue;   // a resumed search starts at q_lo
        const uint32_t nseg = (uint32_t)((w1 - w0 + BIG_SPAN - 1) / BIG_SPAN);
        const uint32_t ncta = (nseg + SPC - 1) / SPC;
        RC(ensure(c->bbitmap, (size_t)nseg * BIG_WORDS * 4));
        RC(ensure(c->bsegcount, (size_t)nseg * 4));
        RC(ensure(c->boffs, (size_t)ncta * std::max<uint32_t>(nbase, 1) * 4));
        launch_sieve_big(w0, w1, nseg, SPC, base, nbase, as<uint32_t>(c->boffs), as<uint32_t>(c->bbitmap),
                         as<uint32_t>(c->bsegcount), s3);
        c->launches++;
        if (q_lo > w0) {
            launch_clear_below(as<uint32_t>(c->bbitmap), w0, q_lo, (uint64_t)nseg * BIG_WORDS, s3);
            c->launches++;
        }
        if (maxt0 >= w0) {
            launch_count_bits(as<uint32_t>(c->bbitmap), w0, (uint64_t)nseg * BIG_WORDS, maxt0,
                              as<unsigned long long>(c->wcounts), s3);
            c->launches++;
        }
        // window buckets: the words covering w0 .. min(key, w1 - 1), split by work
        double W = 0;
        std::vector<uint64_t> nw(db.size(), 0);
        for (size_t b = 0; b < db.size(); ++b) {
            if (bkey[b] < w0) continue;
            const uint64_t top = std::min(bkey[b], w1 - 1);
            nw[b] = (top - w0) / 64 + 1;
            W += (double)db[b].nrows * (double)nw[b];
        }
        if (W == 0) continue;
        struct Grp { int L, rpt; std::vector<SweepItem> items; };
        std::vector<Grp> groups;
        uint64_t part_total = 0;
        uint32_t def_total = 0;
        uint32_t maxs = 0;
        for (size_t b = 0; b < db.size(); ++b) {
            Bucket& x = wb[b];
            x = db[b];
            x.ncols = (uint32_t)nw[b];
            x.cdense = 0;
            x.ndense = 0;
            x.cbase = 0;
            x.part_base = part_total;
            x.def_base = def_total;
            if (!nw[b]) { x.nsplit = 0; continue; }
            const int rpt = x.nrows >= 512 ? 2 : 1;
            uint64_t S = (uint64_t)std::ceil((double)rpt * (double)nw[b] * target_threads / W);
            S = std::max<uint64_t>(1, std::min<uint64_t>(S, std::max<uint64_t>(1, nw[b] / 256)));
            x.nsplit = (uint32_t)S;
            maxs = std::max<uint32_t>(maxs, x.nsplit);
            part_total += S * x.nrows;
            def_total += (uint32_t)S;
            std::vector<RowTile> tiles;
            row_tiles(x.nrows, rpt, 1, tiles);
            for (const RowTile& t : tiles) {
                Grp* g = nullptr;
                for (auto& gg : groups) if (gg.L == (int)x.L && gg.rpt == t.rpt) g = &gg;
                if (!g) { groups.push_back({ (int)x.L, t.rpt, {} }); g = &groups.back(); }
                tile_items(t, 0, (uint32_t)S, [&](uint32_t r0, uint32_t s2, uint32_t tp) {
                    g->items.push_back({ (uint32_t)b, r0, s2, tp });
                });
            }
        }
        // the previous window's copies must be done before these host vectors change
        CK(cudaStreamSynchronize(s3));
        CK(cudaGetLastError());
        all.clear();
        for (auto& g : groups) all.insert(all.end(), g.items.begin(), g.items.end());
        RC(ensure(c->wbuckets, wb.size() * sizeof(Bucket)));
        RC(ensure(c->witems, all.size() * sizeof(SweepItem) + 16));
        RC(ensure(c->wpart, part_total * 16 + 16));
        RC(ensure(c->wdefs, (size_t)def_total * sizeof(Deficit) + 16));
        CK(cudaMemcpyAsync(c->wbuckets.p, wb.data(), wb.size() * sizeof(Bucket), cudaMemcpyHostToDevice, s3));
        CK(cudaMemcpyAsync(c->witems.p, all.data(), all.size() * sizeof(SweepItem), cudaMemcpyHostToDevice, s3));
        size_t ioff = 0;
        for (auto& g : groups) {
            launch_sweep_bits(g.L, g.rpt, (uint32_t)g.items.size(), as<Bucket>(c->wbuckets),
                              as<SweepItem>(c->witems) + ioff, as<RowMod>(c->rowmod), as<uint32_t>(c->bbitmap), w0,
                              as<uint64_t>(c->wkeys), as<uint4>(c->wpart), as<Deficit>(c->wdefs), s3);
            c->launches++;
            ioff += g.items.size();
        }
        for (auto& g : lgroups) {
            if (maxs >= (uint32_t)c->tune.merge_cta_min)
                launch_merge_cta(g.first, as<Bucket>(c->wbuckets), as<RowInfo>(c->rowinfo), as<RowMod>(c->rowmod),
                                 as<uint4>(c->wpart), as<Deficit>(c->wdefs), g.second.first,
                                 g.second.second - g.second.first, as<uint4>(c->bacc), as<Deficit>(c->bdef), s3);
            else
                launch_merge(g.first, as<Bucket>(c->wbuckets), as<RowInfo>(c->rowinfo), as<RowMod>(c->rowmod),
                             as<uint4>(c->wpart), as<Deficit>(c->wdefs), g.second.first, g.second.second - g.second.first,
                             as<uint4>(c->bacc), as<Deficit>(c->bdef), s3);
            c->launches++;
        }
    }
    {
        unsigned long long pi = 0;
        CK(cudaMemcpyAsync(&pi, c->wcounts.p, 8, cudaMemcpyDeviceToHost, s3));
        CK(cudaStreamSynchronize(s3));
        CK(cudaGetLastError());
        *pi_big = pi;
    }
    CK(cudaEventRecord(c->big1, s3));
    CK(cudaEventRecord(c->join, s3));
    CK(cudaStreamWaitEvent(c->st, c->join, 0));
    CK(cudaEventSynchronize(c->big1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->big0, c->big1);
    c->ms_big = ms;
    return 0;
}

// Test primes of each range, ascending, by deterministic Miller-Rabin over
// the range's window (k_window_primes_multi, k_compact: one launch each for
// all ranges); rs[i] gets the range's window layout and its offset and count
// in tps.
int gen_test_primes(wl_ctx* c, const wl_range* ranges, size_t nr, std::vector<RangeState>& rs,
                    std::vector<uint64_t>& tps, bool allow_empty) {
    rs.assign(nr, RangeState());
    std::vector<uint64_t> pmins(nr), pmaxs(nr);
    for (size_t i = 0; i < nr; ++i) {
        pmins[i] = ranges[i].pmin;
        pmaxs[i] = ranges[i].pmax;
    }
    std::vector<WindowPlan> wp;
    uint64_t words = 0, segs = 0, blocks = 0;
    plan_windows(pmins.data(), pmaxs.data(), nr, SEG_SPAN, wp, &words, &segs, &blocks);
    for (size_t i = 0; i < nr; ++i) {
        RangeState& r = rs[i];
        r.pmin = pmins[i];
        r.pmax = pmaxs[i];
        r.lo0 = wp[i].lo0;
        r.nseg = wp[i].nseg;
        r.word_off = wp[i].word_off;
        r.seg_off = wp[i].seg_off;
    }
    RC(ensure(c->bitmap, std::max<uint64_t>(words * 4, c->bitmap.cap)));
    RC(ensure(c->segcount, std::max<uint64_t>(segs * 4, c->segcount.cap)));
    RC(ensure(c->offsets, std::max<uint64_t>((segs + 1) * 8, c->offsets.cap)));
    // every range in one launch, each over its own integers only (512 per block)
    if (blocks >= (1ull << 31)) return WL_ERR_UNSUPPORTED;
    std::vector<WinDesc> wd(nr);
    for (size_t i = 0; i < nr; ++i)
        wd[i] = WinDesc{ wp[i].lo0, pmins[i], pmaxs[i], wp[i].word_off, wp[i].seg_off, (uint32_t)wp[i].block0, 0 };
    RC(ensure(c->windesc, nr * sizeof(WinDesc)));
    CK(cudaMemcpyAsync(c->windesc.p, wd.data(), nr * sizeof(WinDesc), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemsetAsync(c->bitmap.p, 0, words * 4, c->st));
    CK(cudaMemsetAsync(c->segcount.p, 0, segs * 4, c->st));
    launch_window_primes_multi(as<WinDesc>(c->windesc), (uint32_t)nr, (uint32_t)blocks, as<uint32_t>(c->bitmap),
                               as<uint32_t>(c->segcount), c->st);
    c->launches++;
    c->h2d += nr * sizeof(WinDesc);
    std::vector<uint32_t> segcnt(segs);
    CK(cudaMemcpyAsync(segcnt.data(), c->segcount.p, segs * 4, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    c->d2h += segs * 4;
    std::vector<uint64_t> offs(segs + 1);
    uint64_t total = 0;
    for (size_t i = 0; i < nr; ++i) {
        RangeState& r = rs[i];
        r.tp_off = total;
        for (uint32_t s = 0; s < r.nseg; ++s) {
            offs[r.seg_off + s] = total;
            total += segcnt[r.seg_off + s];
        }
        r.ntp = total - r.tp_off;
        if (r.ntp == 0 && !allow_empty) return WL_ERR_NOPRIMES;
    }
    offs[segs] = total;
    if (total >= (1ull << 31)) return WL_ERR_UNSUPPORTED;
    RC(ensure(c->tp, total * 8));
    std::vector<uint64_t> seg_lo(segs);
    for (size_t i = 0; i < nr; ++i)
        for (uint32_t s = 0; s < rs[i].nseg; ++s) seg_lo[rs[i].seg_off + s] = rs[i].lo0 + (uint64_t)s * SEG_SPAN;
    RC(ensure(c->seglo, segs * 8));
    CK(cudaMemcpyAsync(c->offsets.p, offs.data(), (segs + 1) * 8, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->seglo.p, seg_lo.data(), segs * 8, cudaMemcpyHostToDevice, c->st));
    c->h2d += (segs + 1) * 8 + segs * 8;
    // every range's segments in one ordered write-out
    launch_compact_multi((uint32_t)segs, as<uint64_t>(c->seglo), as<uint32_t>(c->bitmap), as<uint64_t>(c->offsets),
                         as<uint64_t>(c->tp), c->st);
    c->launches++;
    tps.assign(total, 0);
    CK(cudaMemcpyAsync(tps.data(), c->tp.p, total * 8, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    c->d2h += total * 8;
    return 0;
}

// Columns q in [q_lo, q_cap) (q_cap = 0: through the class target, then the
// tail and the lift); init: the rows' running products before q_lo, two
// digits (s0, s1) per row in output order, or NULL for 1.
static int run_ranges(wl_ctx* c, const wl_range* ranges, size_t nr, uint64_t qcap, RunOut& out, wl_stats* st,
                      uint64_t q_lo = 2, const uint64_t* init = nullptr, bool graph = false) {
    const bool full = (qcap == 0);
    c->launches = 0;
    c->h2d = c->d2h = 0;
    c->ms_sieve = 0;
    c->sieve_ints = c->sieve_bytes = 0;
    c->ms_big = 0;
    for (size_t i = 0; i < nr; ++i) RC(wl_check_range(ranges[i].pmin, ranges[i].pmax));

    cudaEventRecord(c->ev[0], c->st);

    // ---- 1. test primes ----------------------------------------------------
    std::vector<RangeState> rs;
    std::vector<uint64_t> tps;
    RC(gen_test_primes(c, ranges, nr, rs, tps));
    cudaEventRecord(c->ev[1], c->st);
    const uint64_t total = tps.size();
    const uint32_t nrows = (uint32_t)total;

    // ---- 2. classification and buckets ---------------------------------------
    std::vector<HostBucket> hb;
    hb.reserve(nr * 3);
    for (size_t i = 0; i < nr; ++i) {
        RangeState& r = rs[i];
        int bidx[3] = { -1, -1, -1 };
        const int L = limb_width(r.pmax - 1);
        for (uint64_t k = 0; k < r.ntp; ++k) {
            const uint64_t p = tps[r.tp_off + k];
            uint32_t t;
            uint64_t Tp;
            if (p % 3 == 1) { t = 0; Tp = (p - 1) / 6; }
            else if (p % 12 == 5) { t = 1; Tp = (p - 1) / 4; }
            else if (p % 12 == 11) { t = 2; Tp = (p - 1) / 2; }
            else return WL_ERR_ARG;   // p = 2, 3 never occur since pmin >= 5
            if (bidx[t] < 0) {
                bidx[t] = (int)hb.size();
                HostBucket b;
                b.range = (uint32_t)i;
                b.type = t;
                b.L = (uint32_t)L;
                b.T = Tp;
                hb.push_back(b);
                r.T[t] = Tp;
            }
            hb[bidx[t]].primes.push_back(p);
            hb[bidx[t]].src.push_back((uint32_t)k);
            r.per_class[t]++;
        }
    }
    // device order of buckets: by limb width, then range, then class
    std::vector<uint32_t> border(hb.size());
    for (size_t i = 0; i < hb.size(); ++i) border[i] = (uint32_t)i;
    std::stable_sort(border.begin(), border.end(), [&](uint32_t a, uint32_t b) { return hb[a].L < hb[b].L; });

    // ---- 3. columns ------------------------------------------------------------
    uint64_t need = 0;
    std::vector<uint64_t> keys(hb.size());
    for (size_t i = 0; i < hb.size(); ++i) {
        uint64_t key = hb[i].T;
        if (!full && qcap - 1 < key) key = qcap - 1;
        keys[i] = key;
        need = std::max(need, key + 1);
    }
    // the largest class target of the first range (for pi(maxtarget))
    uint64_t maxt0 = std::max(rs[0].T[0], std::max(rs[0].T[1], rs[0].T[2]));
    // columns above 2^32 come from the windowed sieve (run_big_columns); the
    // cache holds every prime below min(need, 2^32), which includes the
    // sieving primes of the windows (< 2^31)
    const uint64_t big_need = need > (1ull << 32) ? need : 0;
    RC(ensure_columns(c, std::min<uint64_t>(need, 1ull << 32)));
    keys.push_back(full ? maxt0 : std::min(maxt0, qcap - 1));
    // dense columns: q below the point where floor(T/q) drops at about every
    // prime (T*ln(q)/q^2 >~ 1); there the prefix fold would pay a modular
    // exponentiation per column, above it the fold is rarer than a cell
    const size_t nb = hb.size();
    for (size_t i = 0; i < nb; ++i) {
        const double T = (double)hb[i].T;
        double q = std::sqrt(T) + 2;
        for (int k = 0; k < 4; ++k) q = std::sqrt(T * std::log(std::max(q, 3.0))) + 2;
        uint64_t qd = q >= 1.8e19 ? ~0ull : (uint64_t)q;
        keys.push_back(std::min<uint64_t>(qd, keys[i]));
    }
    if (q_lo > 2) keys.push_back(q_lo - 1);   // columns already multiplied in (init)
    RC(ensure(c->keys, keys.size() * 8));
    RC(ensure(c->counts, keys.size() * 8));
    CK(cudaMemcpyAsync(c->keys.p, keys.data(), keys.size() * 8, cudaMemcpyHostToDevice, c->st));
    launch_count_leq(as<uint32_t>(c->cols), c->ncols, as<uint64_t>(c->keys), (uint32_t)keys.size(),
                     as<uint64_t>(c->counts), c->st);
    c->launches++;
    std::vector<uint64_t> ncol(keys.size());
    CK(cudaMemcpyAsync(ncol.data(), c->counts.p, keys.size() * 8, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());
    c->h2d += keys.size() * 8;
    c->d2h += keys.size() * 8;
    out.pi_maxtarget = ncol[nb];
    uint64_t* ndn = ncol.data() + nb + 1;   // dense column counts per bucket
    // a search resumed at q_lo: each bucket's columns start at cb_lo[i] (the
    // primes below q_lo); from here on ncol and ndn count columns from there
    std::vector<uint64_t> cb_lo(nb, 0);
    if (q_lo > 2) {
        const uint64_t c_lo = ncol[2 * nb + 1];
        for (size_t i = 0; i < nb; ++i) {
            cb_lo[i] = std::min(c_lo, ncol[i]);
            ndn[i] = ndn[i] > cb_lo[i] ? ndn[i] - cb_lo[i] : 0;
            ncol[i] -= cb_lo[i];
        }
    }

    // ---- 4. device layout: rows, buckets, splits, items ------------------------
    std::vector<Bucket> db(hb.size());
    std::vector<RowInfo> ri(nrows);
    std::vector<uint64_t> row_src(nrows);    // global output index (range-major, ascending p)
    // work weights: cells per row, dense columns by the cost model
    std::vector<double> dcost(nb, 0.0);
    std::vector<std::vector<double>> dgrid(nb), dcum(nb);
    for (size_t i = 0; i < nb; ++i) {
        if (!ndn[i]) continue;
        double cols_est = 1;
        const double qd = (double)std::min<uint64_t>(keys[nb + 1 + i], keys[i]);
        dense_cost_grid((double)hb[i].T, qd, dgrid[i], dcum[i], &cols_est);
        dcost[i] = dcum[i].back() * (double)ndn[i] / std::max(cols_est, 1.0);
    }
    double W = 0;
    for (size_t i = 0; i < nb; ++i)
        W += (double)hb[i].primes.size() * ((double)(ncol[i] - ndn[i]) + dcost[i]);
    const double target_threads = (double)c->sms * 2048.0 * 4.0;
    std::vector<uint64_t> dkeys;                 // interior dense boundaries (values), all buckets
    std::vector<uint32_t> dkeys_bucket_start, dkeys_n;
    std::vector<char> dequal;                    // per bucket (device order): equal dense splits
    uint32_t row = 0;
    uint64_t part_total = 0;
    uint32_t def_total = 0;
    out.cells = 0;
    // sweep items per launch, with each item's modelled cost (rows x cells per
    // row of its splits): a launch runs its items longest first, so that the
    // last CTAs to start are short ones
    struct ItemGroup { int L, rpt; bool dense; std::vector<SweepItem> items; std::vector<double> cost; };
    std::vector<ItemGroup> groups;
    auto group_for = [&](int L, int rpt, bool dense) -> ItemGroup& {
        for (auto& g : groups) if (g.L == L && g.rpt == rpt && g.dense == dense) return g;
        groups.push_back({ L, rpt, dense, {}, {} });
        return groups.back();
    };
    // rows one item of a tile covers, times the splits it holds
    auto item_rows = [](const RowTile& t, uint32_t nrows) -> double {
        const uint32_t left = nrows - t.row0;
        const uint32_t span = t.tps * (uint32_t)t.rpt;
        return (double)(left < span ? left : span) * (double)tile_groups(t);
    };
    // splits per bucket (wl_plan.h), lengthened when the split partials would
    // not fit a third of the free device memory (24 GiB at most)
    std::vector<SplitBucket> sbs(nb);
    for (size_t i = 0; i < nb; ++i) {
        sbs[i].nrows = (uint32_t)hb[i].primes.size();
        sbs[i].rpt = sparse_rpt_for(c->tune.sparse_rpt[hb[i].L - 2], sbs[i].nrows);
        sbs[i].ndense = ndn[i];
        sbs[i].nsparse = ncol[i] - ndn[i];
        sbs[i].dcost = dcost[i];
    }
    double scale = 1.0;
    {
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) { cudaGetLastError(); free_b = 8ull << 30; }
        const double budget = std::min<double>((double)(free_b + c->part.cap) / 3.0, 24.0 * (1ull << 30)) / 16.0;
        scale = split_scale(sbs, W, target_threads, budget);
    }
    auto plan_splits = [&](size_t i, double sc, uint64_t* Sd_out, uint64_t* Ss_out) {
        plan_bucket_splits(sbs[i], W, target_threads, sc, Sd_out, Ss_out);
    };
    for (uint32_t oi = 0; oi < border.size(); ++oi) {
        const uint32_t i = border[oi];
        const HostBucket& h = hb[i];
        Bucket& b = db[oi];
        b.T = h.T;
        b.ncols = (uint32_t)ncol[i];
        b.row_begin = row;
        b.nrows = (uint32_t)h.primes.size();
        b.L = h.L;
        b.type = h.type;
        b.range = h.range;
        const int rpt = sparse_rpt_for(c->tune.sparse_rpt[b.L - 2], b.nrows);
        const uint64_t nd = ndn[i];
        uint64_t Sd = 0, Ss = 0;
        plan_splits(i, scale, &Sd, &Ss);
        b.cdense = (uint32_t)nd;
        b.ndense = (uint32_t)Sd;
        b.dstart = (uint32_t)dkeys_bucket_start.size();
        b.cbase = (uint32_t)cb_lo[i];
        dkeys_bucket_start.push_back((uint32_t)dkeys.size());
        dkeys_n.push_back((uint32_t)Sd);
        dequal.push_back(cb_lo[i] > 0);
        // interior boundaries at equal cumulative cost (values q: split k ends at
        // q_k), interpolated inside a grid step: there are more splits than grid
        // points when the dense region is long, and a boundary snapped to the
        // grid would leave empty splits next to ones many times too long
        for (uint64_t k = 1; k < Sd && !cb_lo[i]; ++k)
            dkeys.push_back((uint64_t)dense_boundary(dgrid[i], dcum[i], k, Sd));
        b.nsplit = (uint32_t)(Sd + Ss);
        const uint64_t S = b.nsplit;
        b.part_base = part_total;
        b.def_base = def_total;
        part_total += S * b.nrows;
        def_total += (uint32_t)S;
        out.cells += (uint64_t)b.nrows * b.ncols;
        std::vector<RowTile> tiles;
        if (Ss) {
            const double per_split = (double)(b.ncols - b.cdense) / (double)Ss;   // sparse: equal splits
            row_tiles(b.nrows, rpt, 1, tiles);
            for (const RowTile& t : tiles) {
                ItemGroup& g = group_for((int)b.L, t.rpt, false);
                const double c = per_split * item_rows(t, b.nrows);
                tile_items(t, (uint32_t)Sd, (uint32_t)S, [&](uint32_t r0, uint32_t s2, uint32_t tp) {
                    g.items.push_back({ oi, r0, s2, tp });
                    g.cost.push_back(c);
                });
            }
        }
        if (Sd) {
            int drpt;
            uint32_t dtps;
            dense_shape(b.nrows, &drpt, &dtps);
            const double per_split = dcost[i] / (double)Sd;   // dense: splits of equal modelled cost
            row_tiles(b.nrows, drpt, 8, tiles, true);
            for (const RowTile& t : tiles) {
                ItemGroup& g = group_for((int)b.L, t.rpt, true);
                const double c = per_split * item_rows(t, b.nrows);
                tile_items(t, 0, (uint32_t)Sd, [&](uint32_t r0, uint32_t s2, uint32_t tp) {
                    g.items.push_back({ oi, r0, s2, tp });
                    g.cost.push_back(c);
                });
            }
        }
        for (uint32_t k = 0; k < b.nrows; ++k) {
            RowInfo& x = ri[row + k];
            x.p = h.primes[k];
            x.type = h.type;
            x.Tp = h.type == 0 ? (x.p - 1) / 6 : (h.type == 1 ? (x.p - 1) / 4 : (x.p - 1) / 2);
            x.bucket = oi;
            x.it_begin = 0;
            x.it_count = 0;
            row_src[row + k] = rs[h.range].tp_off + h.src[k];
        }
        row += b.nrows;
    }
    // dense split starts: [0, count(cols <= q_1), ..., cdense] per bucket (device order)
    std::vector<uint32_t> dsplit;
    {
        std::vector<uint64_t> dcounts(dkeys.size());
        if (!dkeys.empty()) {
            RC(ensure(c->keys, dkeys.size() * 8));
            RC(ensure(c->counts, dkeys.size() * 8));
            CK(cudaMemcpyAsync(c->keys.p, dkeys.data(), dkeys.size() * 8, cudaMemcpyHostToDevice, c->st));
            launch_count_leq(as<uint32_t>(c->cols), c->ncols, as<uint64_t>(c->keys), (uint32_t)dkeys.size(),
                             as<uint64_t>(c->counts), c->st);
            c->launches++;
            CK(cudaMemcpyAsync(dcounts.data(), c->counts.p, dkeys.size() * 8, cudaMemcpyDeviceToHost, c->st));
            CK(cudaStreamSynchronize(c->st));
            CK(cudaGetLastError());
            c->h2d += dkeys.size() * 8;
            c->d2h += dkeys.size() * 8;
        }
        for (uint32_t oi = 0; oi < db.size(); ++oi) {
            Bucket& b = db[oi];
            const uint32_t k0 = dkeys_bucket_start[oi], n = dkeys_n[oi];
            b.dstart = (uint32_t)dsplit.size();
            if (!n) continue;
            dsplit.push_back(0);
            if (dequal[oi]) {
                // resumed bucket: equal splits of the remaining dense columns
                for (uint32_t k = 1; k < n; ++k) dsplit.push_back((uint32_t)((uint64_t)b.cdense * k / n));
                dsplit.push_back(b.cdense);
                continue;
            }
            uint32_t prev = 0;
            for (uint32_t k = 1; k < n; ++k) {
                uint32_t v = (uint32_t)std::min<uint64_t>(dcounts[k0 + k - 1], b.cdense);
                v = std::max(v, prev);
                dsplit.push_back(v);
                prev = v;
            }
            dsplit.push_back(b.cdense);
        }
    }

    // consecutive-integer tail (full search only): row r has it_count chunks of
    // K integers starting at T+1; the items themselves are derived on the device
    uint64_t n_items = 0, K = 1;
    out.tail = 0;
    if (full) {
        uint64_t Wt = 0;
        for (uint32_t r = 0; r < nrows; ++r) Wt += ri[r].Tp - db[ri[r].bucket].T;
        out.tail = Wt;
        const double tgt_items = (double)c->sms * 2048.0 * 2.0;
        K = std::max<uint64_t>(1024, (uint64_t)std::ceil((double)Wt / tgt_items));
        K = std::min<uint64_t>(K, 1u << 30);
        for (uint32_t r = 0; r < nrows; ++r) {
            const uint64_t len = ri[r].Tp - db[ri[r].bucket].T;
            ri[r].it_begin = (uint32_t)n_items;
            ri[r].it_count = (uint32_t)((len + K - 1) / K);
            n_items += ri[r].it_count;
        }
        if (n_items >= (1ull << 32)) return WL_ERR_UNSUPPORTED;
    } else {
        for (uint32_t r = 0; r < nrows; ++r) { ri[r].it_begin = 0; ri[r].it_count = 0; }
    }

    // ---- 5. upload and launch ----------------------------------------------------
    size_t nitems_total = 0;
    for (auto& g : groups) nitems_total += g.items.size();
    RC(ensure(c->buckets, db.size() * sizeof(Bucket)));
    RC(ensure(c->rowinfo, (size_t)nrows * sizeof(RowInfo)));
    RC(ensure(c->rowmod, (size_t)nrows * sizeof(RowMod)));
    RC(ensure(c->items, nitems_total * sizeof(SweepItem) + 16));
    RC(ensure(c->part, part_total * 16 + 16));
    RC(ensure(c->ipart, n_items * 16 + 16));
    RC(ensure(c->defs, (size_t)def_total * sizeof(Deficit) + 16));
    RC(ensure(c->rowout, (size_t)nrows * sizeof(RowOut)));
    RC(ensure(c->dsplit, dsplit.size() * 4 + 16));
    if (!dsplit.empty())
        CK(cudaMemcpyAsync(c->dsplit.p, dsplit.data(), dsplit.size() * 4, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->buckets.p, db.data(), db.size() * sizeof(Bucket), cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(c->rowinfo.p, ri.data(), (size_t)nrows * sizeof(RowInfo), cudaMemcpyHostToDevice, c->st));
    std::vector<SweepItem> all_items;
    all_items.reserve(nitems_total);
    for (auto& g : groups) {
        std::vector<uint32_t> ord(g.items.size());
        for (uint32_t k = 0; k < ord.size(); ++k) ord[k] = k;
        std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b2) { return g.cost[a] > g.cost[b2]; });
        for (uint32_t k : ord) all_items.push_back(g.items[k]);
    }
    if (!all_items.empty())
        CK(cudaMemcpyAsync(c->items.p, all_items.data(), all_items.size() * sizeof(SweepItem),
                           cudaMemcpyHostToDevice, c->st));
    c->h2d += db.size() * sizeof(Bucket) + (size_t)nrows * sizeof(RowInfo) + all_items.size() * sizeof(SweepItem);

    // per-row accumulators of the column products (1, or the resumed products)
    RC(ensure(c->uacc, (size_t)nrows * 16 + 16));
    RC(ensure(c->udef, db.size() * sizeof(Deficit) + 16));
    RC(ensure(c->work, 24));
    // from here to the lift the device work is fixed by the plan above: a
    // batch issues it as one graph (no initial products to upload and no
    // columns above 2^32, whose windows are planned from device counts)
    ChainGraph cg;
    if (graph && !init && !big_need) RC(cg.begin(c->st));
    launch_acc_init(nrows, (uint32_t)db.size(), as<uint4>(c->uacc), as<Deficit>(c->udef), c->st);
    c->launches++;
    if (init) {
        // the running products before q_lo, as values s0 + p*s1 < p^2 (deficit 0)
        std::vector<uint4> iv(nrows);
        for (uint32_t r = 0; r < nrows; ++r) {
            const uint64_t s0 = init[2 * row_src[r]], s1 = init[2 * row_src[r] + 1], p = ri[r].p;
            if (s0 >= p || s1 >= p) return WL_ERR_ARG;
            const unsigned __int128 v = (unsigned __int128)s1 * p + s0;
            iv[r] = make_uint4((uint32_t)v, (uint32_t)(v >> 32), (uint32_t)(v >> 64), (uint32_t)(v >> 96));
        }
        CK(cudaMemcpyAsync(c->uacc.p, iv.data(), (size_t)nrows * 16, cudaMemcpyHostToDevice, c->st));
        c->h2d += (size_t)nrows * 16;
    }
    launch_setup_rows(as<RowInfo>(c->rowinfo), nrows, as<RowMod>(c->rowmod), c->st);
    c->launches++;
    CK(cudaMemsetAsync(c->work.p, 0, 24, c->st));
    CK(cudaEventRecord(c->rows_ready, c->st));
    cg.record(c->ev[2], c->st);
    size_t ioff = 0;
    bool forked = false;
    for (auto& g : groups) {
        if (g.dense && !g.items.empty() && !forked) {
            CK(cudaEventRecord(c->fork, c->st));
            CK(cudaStreamWaitEvent(c->st2, c->fork, 0));
            forked = true;
        }
        if (g.dense)
            launch_sweep_dense(g.L, g.rpt, (uint32_t)g.items.size(), as<Bucket>(c->buckets), as<SweepItem>(c->items) + ioff,
                               as<RowMod>(c->rowmod), as<uint32_t>(c->cols), as<uint32_t>(c->dsplit),
                               as<uint4>(c->part), as<Deficit>(c->defs), c->st2, c->tune.dense_kernel[g.L - 2],
                               (uint32_t)c->tune.dense_hstep[g.L - 2], as<unsigned long long>(c->work));
        else
            launch_sweep(c->tune.sparse_variant[g.L - 2], g.L, g.rpt, (uint32_t)g.items.size(), as<Bucket>(c->buckets),
                         as<SweepItem>(c->items) + ioff, as<RowMod>(c->rowmod), as<uint32_t>(c->cols),
                         as<uint4>(c->part), as<Deficit>(c->defs), c->st, col_groups(c));
        if (!g.items.empty()) c->launches++;
        ioff += g.items.size();
    }
    if (forked) {
        CK(cudaEventRecord(c->join, c->st2));
        CK(cudaStreamWaitEvent(c->st, c->join, 0));
    }
    // merge every row's split partials into its accumulator
    {
        uint32_t maxs = 0;
        for (auto& x : db) maxs = std::max(maxs, x.nsplit);
        for (uint32_t rb = 0; rb < nrows;) {
            const int L = (int)db[ri[rb].bucket].L;
            uint32_t re = rb;
            while (re < nrows && (int)db[ri[re].bucket].L == L) ++re;
            if (maxs >= (uint32_t)c->tune.merge_cta_min)
                launch_merge_cta(L, as<Bucket>(c->buckets), as<RowInfo>(c->rowinfo), as<RowMod>(c->rowmod),
                                 as<uint4>(c->part), as<Deficit>(c->defs), rb, re - rb, as<uint4>(c->uacc),
                                 as<Deficit>(c->udef), c->st);
            else
                launch_merge(L, as<Bucket>(c->buckets), as<RowInfo>(c->rowinfo), as<RowMod>(c->rowmod),
                             as<uint4>(c->part), as<Deficit>(c->defs), rb, re - rb, as<uint4>(c->uacc),
                             as<Deficit>(c->udef), c->st);
            c->launches++;
            rb = re;
        }
    }
    bool big = false;
    if (big_need) {
        uint64_t pi_big = 0;
        RC(run_big_columns(c, db, ri, nrows, keys, big_need, maxt0, full, qcap, q_lo, &pi_big));
        out.pi_maxtarget += pi_big;
        big = true;
    }
    cg.record(c->ev[3], c->st);
    // rows are ordered by limb width: one tail and one finish launch per width
    uint32_t rb = 0;
    std::vector<std::pair<int, std::pair<uint32_t, uint32_t>>> lgroups;   // L, [row begin, row end)
    while (rb < nrows) {
        const int L = (int)db[ri[rb].bucket].L;
        uint32_t re = rb;
        while (re < nrows && (int)db[ri[re].bucket].L == L) ++re;
        lgroups.push_back({ L, { rb, re } });
        rb = re;
    }
    for (auto& g : lgroups) {
        const uint32_t ib = ri[g.second.first].it_begin;
        const uint32_t last = g.second.second - 1;
        const uint32_t ie = ri[last].it_begin + ri[last].it_count;
        if (ie > ib) {
            launch_iterate(g.first, as<Bucket>(c->buckets), as<RowInfo>(c->rowinfo), as<RowMod>(c->rowmod),
                           g.second.first, g.second.second - g.second.first, ib, ie - ib, K, as<uint4>(c->ipart),
                           c->st);
            c->launches++;
        }
    }
    cg.record(c->ev[4], c->st);
    for (auto& g : lgroups) {
        launch_finish(g.first, as<Bucket>(c->buckets), as<RowInfo>(c->rowinfo), as<RowMod>(c->rowmod),
                      as<uint4>(c->part), as<Deficit>(c->defs), K, as<uint4>(c->ipart),
                      g.second.first, g.second.second - g.second.first, full ? 1 : 0, as<RowOut>(c->rowout), c->st,
                      as<uint4>(c->uacc), as<Deficit>(c->udef), big ? as<uint4>(c->bacc) : nullptr,
                      big ? as<Deficit>(c->bdef) : nullptr);
        c->launches++;
    }
    if (cg.capturing) RC(cg.launch());
    std::vector<RowOut> ro(nrows);
    CK(cudaMemcpyAsync(ro.data(), c->rowout.p, (size_t)nrows * sizeof(RowOut), cudaMemcpyDeviceToHost, c->st));
    c->d2h += (size_t)nrows * sizeof(RowOut);
    unsigned long long dwork[3] = { 0, 0, 0 };
    CK(cudaMemcpyAsync(dwork, c->work.p, 24, cudaMemcpyDeviceToHost, c->st));
    c->d2h += 24;
    cudaEventRecord(c->ev[5], c->st);
    CK(cudaStreamSynchronize(c->st));
    CK(cudaGetLastError());

    // ---- 6. gather rows in range order, ascending p ------------------------------
    out.rows.assign(nrows, wl_row{});
    for (uint32_t r = 0; r < nrows; ++r) {
        wl_row& w = out.rows[row_src[r]];
        w.p = ri[r].p;
        w.s0 = ro[r].s0;
        w.s1 = ro[r].s1;
        w.rem = ro[r].rem;
        w.quot = ro[r].quot;
        w.type = ri[r].type;
        w.status = ro[r].status;
    }
    out.range_row_off.assign(nr + 1, 0);
    out.range_targets.assign(nr * 3, 0);
    for (size_t i = 0; i < nr; ++i) {
        out.range_row_off[i] = rs[i].tp_off;
        for (int t = 0; t < 3; ++t) out.range_targets[i * 3 + t] = rs[i].T[t];
    }
    out.range_row_off[nr] = total;

    if (st) {
        memset(st, 0, sizeof(*st));
        st->tested = total;
        for (size_t i = 0; i < nr; ++i)
            for (int t = 0; t < 3; ++t) st->per_class[t] += rs[i].per_class[t];
        for (int t = 0; t < 3; ++t) st->targets[t] = rs[0].T[t];
        st->pi_maxtarget = out.pi_maxtarget;
        st->cells = out.cells;
        st->tail_steps = out.tail;
        // -1 where a span cannot be timed (its error is not left pending)
        auto span = [](cudaEvent_t e0, cudaEvent_t e1) -> double {
            float a = 0;
            if (cudaEventElapsedTime(&a, e0, e1) == cudaSuccess) return a;
            (void)cudaGetLastError();
            return -1.0;
        };
        st->ms_device = span(c->ev[0], c->ev[5]);
        st->ms_primes = span(c->ev[0], c->ev[1]);
        st->ms_sieve = c->ms_sieve;
        st->ms_sweep = span(c->ev[2], c->ev[3]);
        st->ms_iterate = span(c->ev[3], c->ev[4]);
        st->ms_finish = span(c->ev[4], c->ev[5]);
        st->kernel_launches = c->launches;
        st->h2d_bytes = c->h2d;
        st->d2h_bytes = c->d2h;
        st->ms_big = c->ms_big;
        st->sieve_integers = c->sieve_ints;
        st->sieve_bytes = c->sieve_bytes;
        st->dense_column_cells = dwork[0];
        st->dense_window_cells = dwork[1];
        st->dense_products = dwork[2];
        st->graph_nodes = cg.nodes;
        st->ms_graph_build = cg.ms_build;
    }
    return 0;
}

// results.txt value of one row (cl_wilson.cpp:872-898): 1 if it is a result line
int result_of(const wl_row& r, int32_t* value) {
    const uint64_t negq = r.p - r.quot;
    const uint64_t smallest = r.quot <= negq ? r.quot : negq;
    if (r.quot == 0) { *value = 0; return 1; }
    if (smallest < 1000) { *value = (smallest == r.quot) ? (int32_t)r.quot : -(int32_t)negq; return 1; }
    return 0;
}

static int summarize(const RunOut& ro, size_t nr, bool full, wl_range_result* rr, wl_result* res, size_t cap,
                     size_t* nres, wl_stats* st) {
    size_t k = 0;
    int err = 0;
    uint64_t total_ck = 0;
    uint32_t total_res = 0;
    for (size_t i = 0; i < nr; ++i) {
        uint64_t ck = 0;
        uint32_t cnt = 0, status = 0;
        for (uint64_t j = ro.range_row_off[i]; j < ro.range_row_off[i + 1]; ++j) {
            const wl_row& r = ro.rows[j];
            if (full) {
                ck += r.p + r.rem + r.quot;
                int32_t v;
                if (result_of(r, &v)) {
                    if (res && k < cap) { res[k].p = r.p; res[k].value = v; res[k].pad = 0; }
                    ++k;
                    ++cnt;
                }
                if (r.status && !status) status = r.status;
            } else {
                ck += r.p + r.s0 + r.s1;
            }
        }
        if (rr) {
            rr[i].tested = ro.range_row_off[i + 1] - ro.range_row_off[i];
            rr[i].checksum = ck;
            for (int t = 0; t < 3; ++t) rr[i].targets[t] = ro.range_targets[i * 3 + t];
            rr[i].results = cnt;
            rr[i].status = status;
        }
        total_ck += ck;
        total_res += cnt;
        if (status == 1 && !err) err = WL_ERR_WILSON_CHECK;
        if (status == 2 && !err) err = WL_ERR_NO_REPR;
    }
    if (nres) *nres = k;
    if (st) {
        st->checksum = total_ck;
        st->results = total_res;
    }
    if (err) return err;
    if (res && k > cap) return WL_ERR_CAPACITY;
    return 0;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" {

const char* wl_strerror(int code) {
    switch (code) {
        case WL_OK: return "ok";
        case WL_ERR_ARG: return "invalid argument or range";
        case WL_ERR_CUDA: return "CUDA error";
        case WL_ERR_NOPRIMES: return "there are no primes to test in this range!";
        case WL_ERR_UNSUPPORTED: return "configuration not supported by this library";
        case WL_ERR_WILSON_CHECK: return "Wilson quotient check failed";
        case WL_ERR_NO_REPR: return "representation a, c or u not found";
        case WL_ERR_CAPACITY: return "result buffer too small";
        case WL_ERR_NOMEM: return "device allocation failed";
        case WL_ERR_TOO_LARGE: return "request exceeds the fixed scratch of the no-allocation entry point";
        default: return "unknown error";
    }
}

int wl_check_range(uint64_t pmin, uint64_t pmax) {
    if (pmin < 5 || pmax > WL_MAXP || pmin >= pmax) return WL_ERR_ARG;
    if (pmax - pmin > WL_MAX_WIDTH) return WL_ERR_ARG;
    return 0;
}

int wl_open(int device, wl_ctx** out) {
    if (!out) return WL_ERR_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return WL_ERR_CUDA;
    }
    wl_ctx* c = new wl_ctx();
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess) { delete c; return WL_ERR_CUDA; }
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    if (const char* v = getenv("WL_CELL_VARIANT")) c->cell_variant = atoi(v);
    default_tuning(c);
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->st3, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return WL_ERR_CUDA;
    }
    for (auto& e : c->ev) cudaEventCreate(&e);
    cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming);
    cudaEventCreate(&c->big0);
    cudaEventCreateWithFlags(&c->rows_ready, cudaEventDisableTiming);
    cudaEventCreate(&c->big1);
    // odd primes below 2^16: the sieving primes of the column sieve (q < 2^32)
    std::vector<uint8_t> comp(65536, 0);
    std::vector<uint32_t> base;
    for (uint32_t i = 3; i < 65536; i += 2) {
        if (comp[i]) continue;
        base.push_back(i);
        for (uint32_t j = i * i; j < 65536; j += 2 * i) comp[j] = 1;
    }
    c->nbase = (uint32_t)base.size();
    if (ensure(c->base, base.size() * 4) ||
        cudaMemcpy(c->base.p, base.data(), base.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
        wl_close(c);
        return WL_ERR_CUDA;
    }
    *out = c;
    return 0;
}

void wl_close(wl_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    DevBuf* bufs[] = { &c->base, &c->cols, &c->bitmap, &c->segcount, &c->offsets, &c->tp, &c->keys, &c->counts,
                       &c->buckets, &c->rowinfo, &c->rowmod, &c->items, &c->part, &c->ipart, &c->dsplit,
                       &c->bbitmap, &c->bsegcount, &c->boffsets, &c->boffs, &c->wcols, &c->wbuckets, &c->witems,
                       &c->wpart, &c->wdefs, &c->bacc, &c->bdef, &c->wkeys, &c->wcounts, &c->uacc, &c->udef,
                       &c->defs, &c->rowout, &c->prod, &c->windesc, &c->seglo, &c->work };
    for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
    for (auto& e : c->ev) if (e) cudaEventDestroy(e);
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    if (c->big0) cudaEventDestroy(c->big0);
    if (c->rows_ready) cudaEventDestroy(c->rows_ready);
    if (c->big1) cudaEventDestroy(c->big1);
    if (c->st2) cudaStreamDestroy(c->st2);
    if (c->st3) cudaStreamDestroy(c->st3);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

void* wl_stream(wl_ctx* c) { return c ? (void*)c->st : nullptr; }

void wl_drop_columns(wl_ctx* c) {
    if (!c) return;
    c->ncols = 0;
    c->col_limit = 0;
    c->ngroups = 0;
}

int wl_search(wl_ctx* c, uint64_t pmin, uint64_t pmax, uint64_t q_cap, wl_result* results, size_t cap,
              wl_stats* stats) {
    if (!c) return WL_ERR_ARG;
    cudaSetDevice(c->device);
    wl_range r = { pmin, pmax };
    RunOut ro;
    RC(run_ranges(c, &r, 1, q_cap, ro, stats));
    return summarize(ro, 1, q_cap == 0, nullptr, results, cap, nullptr, stats);
}

int wl_rows(wl_ctx* c, uint64_t pmin, uint64_t pmax, uint64_t q_cap, wl_row* rows, size_t cap, size_t* nrows,
            wl_stats* stats) {
    if (!c) return WL_ERR_ARG;
    cudaSetDevice(c->device);
    wl_range r = { pmin, pmax };
    RunOut ro;
    RC(run_ranges(c, &r, 1, q_cap, ro, stats));
    if (nrows) *nrows = ro.rows.size();
    if (rows) {
        const size_t n = std::min(cap, ro.rows.size());
        memcpy(rows, ro.rows.data(), n * sizeof(wl_row));
    }
    int e = summarize(ro, 1, q_cap == 0, nullptr, nullptr, 0, nullptr, stats);
    if (e) return e;
    if (rows && cap < ro.rows.size()) return WL_ERR_CAPACITY;
    return 0;
}

int wl_rows_from(wl_ctx* c, uint64_t pmin, uint64_t pmax, uint64_t q_lo, uint64_t q_cap, const uint64_t* init,
                 wl_row* rows, size_t cap, size_t* nrows, wl_stats* stats) {
    if (!c || q_lo < 2) return WL_ERR_ARG;
    cudaSetDevice(c->device);
    wl_range r = { pmin, pmax };
    RunOut ro;
    RC(run_ranges(c, &r, 1, q_cap, ro, stats, q_lo, init));
    if (nrows) *nrows = ro.rows.size();
    if (rows) {
        const size_t n = std::min(cap, ro.rows.size());
        memcpy(rows, ro.rows.data(), n * sizeof(wl_row));
    }
    int e = summarize(ro, 1, q_cap == 0, nullptr, nullptr, 0, nullptr, stats);
    if (e) return e;
    if (rows && cap < ro.rows.size()) return WL_ERR_CAPACITY;
    return 0;
}

int wl_search_from(wl_ctx* c, uint64_t pmin, uint64_t pmax, uint64_t q_lo, const uint64_t* init, wl_result* results,
                   size_t cap, wl_stats* stats) {
    if (!c || q_lo < 2) return WL_ERR_ARG;
    cudaSetDevice(c->device);
    wl_range r = { pmin, pmax };
    RunOut ro;
    RC(run_ranges(c, &r, 1, 0, ro, stats, q_lo, init));
    return summarize(ro, 1, true, nullptr, results, cap, nullptr, stats);
}

int wl_rows_product(wl_ctx* c, size_t n, const uint64_t* p, size_t nparts, const uint64_t* parts, uint64_t* out) {
    if (!c || nparts == 0 || nparts > (1u << 16) || n > (1ull << 32)) return WL_ERR_ARG;
    if (n == 0) return 0;
    if (!p || !parts || !out) return WL_ERR_ARG;
    for (size_t i = 0; i < n; ++i)
        if (p[i] < 5 || p[i] > WL_MAXP || !(p[i] & 1)) return WL_ERR_ARG;
    for (size_t k = 0; k < nparts; ++k) {   // part by part, in memory order
        const uint64_t* d = parts + k * 2 * n;
        bool bad = false;
        for (size_t i = 0; i < n; ++i) bad |= (d[2 * i] >= p[i]) | (d[2 * i + 1] >= p[i]);
        if (bad) return WL_ERR_ARG;
    }
    cudaSetDevice(c->device);
    const size_t pb = n * 8, xb = nparts * n * 16, ob = n * 16;
    RC(ensure(c->prod, pb + xb + ob));
    uint64_t* dp = as<uint64_t>(c->prod);
    uint64_t* dx = dp + n;
    uint64_t* dout = dx + 2 * nparts * n;
    CK(cudaMemcpyAsync(dp, p, pb, cudaMemcpyHostToDevice, c->st));
    CK(cudaMemcpyAsync(dx, parts, xb, cudaMemcpyHostToDevice, c->st));
    launch_rows_product(dp, n, dx, (uint32_t)nparts, dout, c->st);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout, ob, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
}

int wl_batch(wl_ctx* c, const wl_range* ranges, size_t n, uint64_t q_cap, wl_range_result* out,
             wl_result* results, size_t cap, size_t* nresults, wl_stats* stats) {
    if (!c || !ranges || n == 0) return WL_ERR_ARG;
    cudaSetDevice(c->device);
    RunOut ro;
    static const bool direct = getenv("WL_BATCH_GRAPH") && atoi(getenv("WL_BATCH_GRAPH")) == 0;
    RC(run_ranges(c, ranges, n, q_cap, ro, stats, 2, nullptr, !direct));
    return summarize(ro, n, q_cap == 0, out, results, cap, nresults, stats);
}

int wl_get_tuning(wl_ctx* c, wl_tuning* out) {
    if (!c || !out) return WL_ERR_ARG;
    *out = c->tune;
    return 0;
}

int wl_set_tuning(wl_ctx* c, const wl_tuning* t) {
    if (!c || !t) return WL_ERR_ARG;
    for (int i = 0; i < 3; ++i) {
        if (t->sparse_variant[i] < 0 || t->sparse_variant[i] > 3 ||
            (t->sparse_rpt[i] != 1 && t->sparse_rpt[i] != 2 && t->sparse_rpt[i] != 4) ||
            t->dense_kernel[i] < 0 || t->dense_kernel[i] > DENSE_SORTED_W3_2CTA || t->dense_hstep[i] < 1 ||
            t->dense_hstep[i] > 4096)
            return WL_ERR_ARG;
    }
    if (t->merge_cta_min < 1) return WL_ERR_ARG;
    c->tune = *t;
    return 0;
}

// One tuning measurement: the sweep-phase device time of the sample (best of
// `reps` runs) and a digest of its rows, which every candidate must reproduce.
static int tune_time(wl_ctx* c, const wl_range* r, size_t nr, uint64_t qcap, int reps, double* ms,
                     uint64_t* digest) {
    double best = 1e300;
    for (int rep = 0; rep < reps; ++rep) {
        RunOut ro;
        wl_stats st;
        RC(run_ranges(c, r, nr, qcap, ro, &st));
        best = std::min(best, st.ms_sweep);
        uint64_t d = 0;
        for (const wl_row& w : ro.rows) d = d * 0x9E3779B97F4A7C15ull + (w.p ^ w.s0 ^ (w.s1 << 1) ^ (w.quot << 2));
        *digest = d;
    }
    *ms = best;
    return 0;
}

// Coordinate descent over the variants for the limb widths in `mask`, each
// candidate applied to all of them, timed on ranges r[0..nr): the prefix-fold
// sweep, then the dense sweep, then the merge fan-in.  A candidate replaces
// the current choice only when it is more than 2% faster (run-to-run noise is
// about 1%).
static int tune_on(wl_ctx* c, const wl_range* r, size_t nr, uint64_t qcap, uint32_t mask, double* best_ms) {
    uint64_t want = 0;
    double ms;
    uint64_t dg;
    // calibration run (also the reference digest); one run per candidate when a run is long
    RC(tune_time(c, r, nr, qcap, 1, &ms, &want));
    const int reps = ms > 1000.0 ? 1 : 2;
    RC(tune_time(c, r, nr, qcap, reps, &ms, &dg));
    if (dg != want) return WL_ERR_CUDA;
    double cur = ms;
    auto apply = [&](auto f) { for (int L = 2; L <= 4; ++L) if (mask & (1u << (L - 2))) f(L - 2); };
    auto trial = [&](const wl_tuning& t, bool* better) -> int {
        const wl_tuning keep = c->tune;
        c->tune = t;
        RC(tune_time(c, r, nr, qcap, reps, &ms, &dg));
        if (dg != want) {
            fprintf(stderr, "wilson: autotune: kernel variants disagree\n");
            c->tune = keep;
            return WL_ERR_CUDA;
        }
        *better = ms < cur * 0.98;
        if (*better) cur = ms;
        else c->tune = keep;
        return 0;
    };
    // (variant, rows per thread) besides (1, 2)
    const int sparse_c[5][2] = { { 1, 1 }, { 0, 2 }, { 2, 2 }, { 1, 4 }, { 3, 4 } };
    for (auto& sc : sparse_c) {
        wl_tuning t = c->tune;
        apply([&](int i) { t.sparse_variant[i] = sc[0]; t.sparse_rpt[i] = sc[1]; });
        bool b;
        RC(trial(t, &b));
    }
    const int dense_c[9][2] = { { DENSE_SMEM_W3, 4 }, { DENSE_SMEM_W3, 12 }, { DENSE_SMEM_W3, 16 },
                                { DENSE_SORTED_W3, 8 }, { DENSE_SORTED_W4, 8 }, { DENSE_SWITCH_W3, 8 },
                                { DENSE_SWITCH_W4, 8 }, { DENSE_SMEM_W4, 8 }, { DENSE_SORTED_W3_2CTA, 8 } };
    for (auto& dc : dense_c) {
        wl_tuning t = c->tune;
        apply([&](int i) { t.dense_kernel[i] = dc[0]; t.dense_hstep[i] = dc[1]; });
        bool b;
        RC(trial(t, &b));
    }
    for (int m : { 16, 256 }) {
        wl_tuning t = c->tune;
        t.merge_cta_min = m;
        bool b;
        RC(trial(t, &b));
    }
    *best_ms = cur;
    return 0;
}

int wl_autotune(wl_ctx* c, const wl_range* ranges, size_t n, uint64_t q_cap, uint32_t limbs_mask, wl_tuning* out) {
    if (!c || (n && !ranges)) return WL_ERR_ARG;
    cudaSetDevice(c->device);
    if (!limbs_mask) limbs_mask = 7;
    if (n) {
        // the caller's workload: one choice for all its limb widths
        uint32_t mask = 0;
        for (size_t k = 0; k < n; ++k) {
            RC(wl_check_range(ranges[k].pmin, ranges[k].pmax));
            mask |= 1u << (limb_width(ranges[k].pmax - 1) - 2);
        }
        double ms = 0;
        RC(tune_on(c, ranges, n, q_cap, mask & limbs_mask, &ms));
        for (int L = 2; L <= 4; ++L) if (mask & (1u << (L - 2))) c->tune.ms[L - 2] = ms;
    } else {
        // built-in samples, one per limb width, a mix of prefix-fold and dense columns
        struct Sample { wl_range r; uint64_t qcap; };
        const Sample smp[3] = { { { 1000000000ull, 1000300000ull }, 0 },
                                { { 100000000000ull, 100000100000ull }, 1ull << 30 },
                                { { (1ull << 62) - 100001ull, (1ull << 62) - 1ull }, 1ull << 27 } };
        for (int L = 2; L <= 4; ++L) {
            if (!(limbs_mask & (1u << (L - 2)))) continue;
            double ms = 0;
            RC(tune_on(c, &smp[L - 2].r, 1, smp[L - 2].qcap, 1u << (L - 2), &ms));
            c->tune.ms[L - 2] = ms;
        }
    }
    if (out) *out = c->tune;
    return 0;
}

// The reference CLI's number syntax (putil.c:34-116): an integer in C
// notation (decimal, 0x.. hex, 0.. octal) and at most one scale suffix --
// K M G T P (powers of 1000), k m g t p (powers of 1024), e<n> / E<n> (10^n),
// b<n> / B<n> (2^n).  Returns 0, -1 (not a number of that form) or -2 (outside
// [lo, hi], or overflow while scaling).
int wl_parse_uint64(uint64_t* result, const char* str, uint64_t lo, uint64_t hi) {
    if (!result || !str) return -1;
    struct Suffix { char c; uint64_t base; unsigned count; };   // count 0: the count follows the letter
    static const Suffix suffixes[] = {
        { 'K', 1000, 1 }, { 'M', 1000, 2 }, { 'G', 1000, 3 }, { 'T', 1000, 4 }, { 'P', 1000, 5 },
        { 'k', 1024, 1 }, { 'm', 1024, 2 }, { 'g', 1024, 3 }, { 't', 1024, 4 }, { 'p', 1024, 5 },
        { 'e', 10, 0 },   { 'E', 10, 0 },   { 'b', 2, 0 },    { 'B', 2, 0 },
    };
    errno = 0;
    char* rest = nullptr;
    uint64_t value = strtoull(str, &rest, 0);
    if (errno != 0 || value > hi) return -2;
    if (*rest != '\0') {
        const Suffix* sx = nullptr;
        for (const Suffix& x : suffixes)
            if (x.c == *rest) sx = &x;
        if (!sx) return -1;
        unsigned long times = sx->count;
        if (times == 0) {
            times = strtoul(rest + 1, &rest, 0);
            if (errno != 0) return -2;
        } else {
            ++rest;
        }
        if (*rest != '\0') return -1;
        for (; times > 0 && value != 0; --times) {
            if (value > hi / sx->base) return -2;
            value *= sx->base;
        }
    }
    if (value < lo) return -2;
    *result = value;
    return 0;
}

}  // extern "C"
