// wl_serve.cu -- serving sessions of the Wilson-prime engine (wl_server_*).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <thread>
#include <vector>

#include "wilson.h"
#include "wl_internal.h"
#include "wl_host.h"
#include "wl_pool.h"

using namespace wl;

// ===========================================================================
// Serving: a resident session with continuous batching (wl_server_*).
//
// The rows of every admitted request live in a device row pool (RowInfo,
// RowMod, a running product per row, RowOut); their (request, class) buckets
// hold a slot of the bucket table (persistent descriptor plus the bucket's
// accumulated power-of-two deficit).  One scheduler thread owns the GPU:
//   admit   queued requests in FIFO order while the pool has room: test
//           primes, classes and targets, column counts, moduli, and for a full
//           search the consecutive-integer tail folded into each row's running
//           product (k_iterate + k_tail_merge);
//   step    every admitted bucket advances by one chunk of its columns (its
//           share of the step's cell budget): the engine's sweep kernels
//           over [pos, pos + len) -- through Bucket::cbase -- in one launch per
//           (limb width, sweep kind) for all buckets, then k_merge* folds the
//           chunk's split products into the resident running products.  A
//           bucket whose columns go past 2^32 continues above the resident
//           table with chunks of the number line: each chunk is sieved on the
//           device (k_sieve_big, into the bucket's own bitmap region) and swept
//           straight from the bitmap (k_sweep_bits), as the reference's
//           getsegprps chunks above 2^32 (cl_wilson.cpp:1368-1397);
//   finish  requests whose buckets reached their last column: k_finish in
//           merged mode over the request's rows, queued right behind the step,
//           then the rows read back, result lines and checksum
//           (cl_wilson.cpp:872-900); the rows and slots are freed.
// Steps are pipelined: two sets of step buffers, so the scheduler plans and
// queues step k+1 while step k runs, and completes step k (its timing and the
// requests whose lift followed it) meanwhile.  Admissions and cancellations
// drain the pipeline first (admission synchronises the stream and may grow
// the column table; a cancelled request's rows must not be in use).
// ===========================================================================

namespace {

struct SBucket {
    bool used = false;
    uint64_t ncols = 0, cdense = 0, pos = 0;   // columns [0, ncols), dense [0, cdense), next column
    uint32_t nrows = 0, L = 2;
    // columns above 2^32 (key >= 2^32): integers [bpos, bend) still to sieve and
    // sweep, bend = key + 1; nroot sieving primes (67 .. sqrt(key)) for them
    uint64_t bpos = 0, bend = 0, key = 0;
    uint32_t nroot = 0;
    bool stop = false;                         // cancelled: no further chunks
    bool done() const { return pos >= ncols && bpos >= bend; }
    bool idle() const { return stop || done(); }
};

constexpr uint64_t BIG_LO = 1ull << 32;   // first integer above the resident column table
// cost of sieving one integer above 2^32, in cells of the sweep (measured on B200)
constexpr double BIG_SIEVE_CELLS = 1.6;

uint64_t isqrt_floor(uint64_t n) {
    uint64_t r = (uint64_t)std::sqrt((long double)n);
    while (r * r > n) --r;
    while ((r + 1) * (r + 1) <= n) ++r;
    return r;
}

struct SReq {
    uint64_t id = 0, pmin = 0, pmax = 0, qcap = 0;
    int state = WL_REQ_QUEUED, rc = 0;
    bool cancel = false;
    bool have_tps = false;
    std::vector<uint64_t> tps;        // test primes, ascending
    uint32_t r0 = 0, nrows = 0;
    int L = 2;
    std::vector<uint32_t> bids;
    std::vector<uint64_t> primes;     // pool order: row r0 + k holds primes[k]
    std::vector<uint32_t> types;
    uint64_t targets[3] = { 0, 0, 0 };
    uint64_t checksum = 0, cells = 0;
    uint64_t tested = 0;              // set under the server's mutex
    std::vector<wl_row> rows;         // ascending p, once done
    std::vector<wl_result> lines;
    bool finishing = false;           // its lift is queued behind a step (scheduler thread only)
    bool cancel_seen = false;         // the scheduler stopped its buckets (scheduler thread only)
    double t_submit = 0, t_admit = 0, t_done = 0;
};

}  // namespace

struct wl_server {
    wl_ctx* c = nullptr;
    uint32_t pool_cap = 0, bucket_cap = 0;
    uint64_t step_cells = 0;
    uint32_t shares = WL_SHARES_LEAST_WORK;
    DevBuf info, mods, acc, out, pbuckets, bdef, ipart;
    // Two sets of a step's buffers: the scheduler plans and queues step k+1
    // into one set while step k still runs on the other, and completes step k
    // (its timing, the requests whose lift followed it) meanwhile.
    struct Slot {
        DevBuf sbuckets, items, part, defs;          // descriptors, sweep items, split products
        DevBuf bbitmap, bsegcount, boffs, bkeys, blos;   // columns above 2^32: bitmaps and their keys
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        bool inflight = false;
        std::vector<SReq*> finishing;                // their lift runs right after this step
        uint32_t dirty_top = 1u << 30;               // device descriptors at or above: all nsplit = 0
    } slot[2];
    int cur = 0;
    std::vector<SBucket> sb;
    std::vector<Bucket> pdesc;                 // persistent descriptors (device copy: pbuckets)
    RowPool pool;                              // rows of the device row pool
    std::set<uint32_t> free_bids;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<SReq*> queue;
    std::map<uint64_t, SReq*> reqs;
    std::vector<SReq*> active;                 // scheduler thread only
    std::thread worker;
    bool stop = false;
    // something may let queued requests in: a submit, a cancel, rows freed
    // (under mu); admission is tried only then, since it drains the pipeline
    bool admit_pending = false;
    uint64_t next_id = 1;
    wl_server_stats stats = {};    // published copy (under mu)
    wl_server_stats ws = {};       // scheduler thread's own
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaMemPool_t mpool = nullptr;   // the step buffers' stream-ordered pool
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
};

// A step buffer of at least `bytes`.  Step buffers come from the session's own
// stream-ordered pool: one that must grow is freed and reallocated in the
// order of the main stream, behind the step in flight, so the host does not
// wait for that step (cudaFree would wait for the whole device: tens of
// milliseconds, at times more, with the GPU idle until the next step is
// queued), and the pool keeps freed memory for the next growth instead of
// handing it back to the driver.  A buffer grows to half as much again as its
// old size, or to `bytes` if more.
static int ensure_step(wl_server* s, DevBuf& b, size_t bytes) {
    if (bytes <= b.cap && b.p) return 0;
    cudaStream_t st = s->c->st;
    const size_t want = std::max<size_t>(bytes, 256);
    const size_t grown = std::max(want, b.cap + b.cap / 2);
    if (b.p) cudaFreeAsync(b.p, st);
    b.p = nullptr;
    b.cap = 0;
    if (cudaMallocFromPoolAsync(&b.p, grown, s->mpool, st) == cudaSuccess) {
        b.cap = grown;
        return 0;
    }
    cudaGetLastError();
    if (grown != want && cudaMallocFromPoolAsync(&b.p, want, s->mpool, st) == cudaSuccess) {
        b.cap = want;
        return 0;
    }
    cudaGetLastError();
    b.p = nullptr;
    return WL_ERR_NOMEM;
}

static void serve_release(wl_server* s, SReq* q) {
    s->admit_pending = true;
    for (uint32_t bid : q->bids) {
        s->sb[bid] = SBucket();
        memset(&s->pdesc[bid], 0, sizeof(Bucket));
        s->free_bids.insert(bid);
    }
    q->bids.clear();
    if (q->nrows) s->pool.release(q->r0, q->nrows);
    q->nrows = 0;
}

static uint64_t class_target(uint64_t p, uint32_t* type) {
    if (p % 3 == 1) { *type = 0; return (p - 1) / 6; }
    if (p % 12 == 5) { *type = 1; return (p - 1) / 4; }
    *type = 2;
    return (p - 1) / 2;
}

// Admission of queued requests in FIFO order, all in one pass: one test-prime
// pass over their ranges, one column-count query, the uploads while the stream
// is idle, then every request's setup and tail launches and one synchronisation.
// result[k]: 0 admitted, 1 no room yet (this and every later candidate stay
// queued), < 0 the request fails with that code.
static void serve_admit_batch(wl_server* s, const std::vector<SReq*>& cands, std::vector<int>& result) {
    wl_ctx* c = s->c;
    const size_t nc = cands.size();
    result.assign(nc, 1);
    cudaEventRecord(s->e0, c->st);
    // 1. test primes of the candidates that have none yet
    {
        std::vector<size_t> need;
        std::vector<wl_range> rr;
        for (size_t k = 0; k < nc; ++k)
            if (!cands[k]->have_tps) {
                need.push_back(k);
                rr.push_back({ cands[k]->pmin, cands[k]->pmax });
            }
        if (!need.empty()) {
            std::vector<RangeState> rs;
            std::vector<uint64_t> tps;
            const int e = gen_test_primes(c, rr.data(), rr.size(), rs, tps, true);
            s->ws.launches += 2;
            for (size_t j = 0; j < need.size(); ++j) {
                SReq* q = cands[need[j]];
                if (e) { result[need[j]] = e; continue; }
                q->tps.assign(tps.begin() + rs[j].tp_off, tps.begin() + rs[j].tp_off + rs[j].ntp);
                q->have_tps = true;
            }
        }
    }
    // 2. classes and targets; bucket slots and pool rows, first come first served
    struct Adm {
        SReq* q;
        std::vector<uint64_t> byc[3];
        uint64_t T[3];
        std::vector<int> kt;
        std::vector<uint64_t> keys;
    };
    std::vector<Adm> adm;
    uint64_t need = 0;
    for (size_t k = 0; k < nc; ++k) {
        if (result[k] < 0) continue;
        SReq* q = cands[k];
        const bool full = q->qcap == 0;
        const uint32_t n = (uint32_t)q->tps.size();
        if (n == 0) { result[k] = WL_ERR_NOPRIMES; continue; }
        if (n > s->pool_cap) { result[k] = WL_ERR_NOMEM; continue; }
        Adm a;
        a.q = q;
        a.T[0] = a.T[1] = a.T[2] = 0;
        for (uint64_t p : q->tps) {
            uint32_t t;
            const uint64_t Tp = class_target(p, &t);
            if (a.byc[t].empty()) a.T[t] = Tp;
            a.byc[t].push_back(p);
        }
        for (int t = 0; t < 3; ++t) {
            if (a.byc[t].empty()) continue;
            const uint64_t key = full ? a.T[t] : std::min(a.T[t], q->qcap - 1);
            a.kt.push_back(t);
            a.keys.push_back(key);
        }
        uint32_t r0 = 0;
        if (s->free_bids.size() < a.kt.size() || !s->pool.alloc(n, &r0)) break;
        q->r0 = r0;
        q->nrows = n;
        q->L = limb_width(q->pmax - 1);
        for (int t = 0; t < 3; ++t) q->targets[t] = a.T[t];
        for (size_t i = 0; i < a.kt.size(); ++i) {
            q->bids.push_back(*s->free_bids.begin());
            s->free_bids.erase(s->free_bids.begin());
            need = std::max(need, std::min(a.keys[i], BIG_LO - 1) + 1);
        }
        result[k] = 0;
        adm.push_back(std::move(a));
    }
    if (adm.empty()) return;
    auto fail_admitted = [&](int e) {
        for (size_t k = 0; k < nc; ++k)
            if (result[k] == 0) result[k] = e;
    };
    // 3. column counts of every admitted bucket (all columns below 2^32, dense
    // columns, and for buckets that go past 2^32 the sieving primes up to the
    // square root of their key)
    std::vector<uint64_t> keys;
    for (auto& a : adm)
        for (uint64_t key : a.keys) keys.push_back(std::min(key, BIG_LO - 1));
    const size_t nk = keys.size();
    size_t kj = 0;
    for (auto& a : adm)
        for (size_t i = 0; i < a.kt.size(); ++i, ++kj) {
            const double Td = (double)a.T[a.kt[i]];
            double qd = std::sqrt(Td) + 2;
            for (int k = 0; k < 4; ++k) qd = std::sqrt(Td * std::log(std::max(qd, 3.0))) + 2;
            keys.push_back(std::min<uint64_t>(qd >= 1.8e19 ? ~0ull : (uint64_t)qd, keys[kj]));
        }
    for (auto& a : adm)
        for (uint64_t key : a.keys) keys.push_back(key >= BIG_LO ? isqrt_floor(key) : 0);
    int e = ensure_columns(c, need);
    if (!e) e = ensure(c->keys, keys.size() * 8);
    if (!e) e = ensure(c->counts, keys.size() * 8);
    if (e) { fail_admitted(e); return; }
    std::vector<uint64_t> cnt(keys.size());
    if (cudaMemcpyAsync(c->keys.p, keys.data(), keys.size() * 8, cudaMemcpyHostToDevice, c->st) != cudaSuccess) {
        fail_admitted(WL_ERR_CUDA);
        return;
    }
    launch_count_leq(as<uint32_t>(c->cols), c->ncols, as<uint64_t>(c->keys), (uint32_t)keys.size(),
                     as<uint64_t>(c->counts), c->st);
    s->ws.launches++;
    if (cudaMemcpyAsync(cnt.data(), c->counts.p, keys.size() * 8, cudaMemcpyDeviceToHost, c->st) != cudaSuccess ||
        cudaStreamSynchronize(c->st) != cudaSuccess) {
        cudaGetLastError();
        fail_admitted(WL_ERR_CUDA);
        return;
    }
    // 4. buckets, rows and tail items on the host (tail items indexed globally
    // in the admission's tail buffer)
    std::vector<std::vector<RowInfo>> ris(adm.size());
    std::vector<uint64_t> Ks(adm.size(), 1), item_off(adm.size(), 0), nitems(adm.size(), 0);
    uint64_t items_total = 0;
    size_t ki = 0;
    for (size_t ai = 0; ai < adm.size(); ++ai) {
        Adm& a = adm[ai];
        SReq* q = a.q;
        const bool full = q->qcap == 0;
        std::vector<RowInfo>& ri = ris[ai];
        ri.resize(q->nrows);
        uint32_t row = q->r0;
        uint64_t Wt = 0;
        for (size_t i = 0; i < a.kt.size(); ++i, ++ki) {
            const int t = a.kt[i];
            const uint32_t bid = q->bids[i];
            SBucket& b = s->sb[bid];
            b.used = true;
            b.ncols = cnt[ki];
            b.cdense = std::min(cnt[nk + ki], cnt[ki]);
            b.pos = 0;
            b.nrows = (uint32_t)a.byc[t].size();
            b.L = (uint32_t)q->L;
            b.key = a.keys[i];
            b.bpos = BIG_LO;
            b.bend = b.key >= BIG_LO ? b.key + 1 : BIG_LO;
            // column cache: cols[0 .. 17] = 2 .. 61, the presieve of k_sieve_big
            b.nroot = b.key >= BIG_LO && cnt[2 * nk + ki] > 18 ? (uint32_t)(cnt[2 * nk + ki] - 18) : 0;
            Bucket& d = s->pdesc[bid];
            memset(&d, 0, sizeof(d));
            d.T = a.T[t];
            d.row_begin = row;
            d.nrows = b.nrows;
            d.L = b.L;
            d.type = (uint32_t)t;
            q->cells += (uint64_t)b.nrows * b.ncols;
            for (uint64_t p : a.byc[t]) {
                RowInfo& x = ri[row - q->r0];
                uint32_t tt;
                x.p = p;
                x.Tp = class_target(p, &tt);
                x.type = (uint32_t)t;
                x.bucket = bid;
                x.it_begin = 0;
                x.it_count = 0;
                if (full) Wt += x.Tp - d.T;
                q->primes.push_back(p);
                q->types.push_back((uint32_t)t);
                ++row;
            }
        }
        q->cells += Wt;
        if (full && Wt) {
            uint64_t K = std::max<uint64_t>(1024, (uint64_t)std::ceil((double)Wt / ((double)c->sms * 2048.0 * 2.0)));
            K = std::min<uint64_t>(K, 1u << 30);
            uint64_t ni = 0;
            for (uint32_t k = 0; k < q->nrows; ++k) {
                const uint64_t len = ri[k].Tp - s->pdesc[ri[k].bucket].T;
                ri[k].it_begin = (uint32_t)(items_total + ni);
                ri[k].it_count = (uint32_t)((len + K - 1) / K);
                ni += ri[k].it_count;
            }
            Ks[ai] = K;
            item_off[ai] = items_total;
            nitems[ai] = ni;
            items_total += ni;
        }
    }
    if (items_total >= (1ull << 32)) { fail_admitted(WL_ERR_UNSUPPORTED); return; }
    if (items_total && (e = ensure(s->ipart, items_total * 16 + 16))) { fail_admitted(e); return; }
    // 5. uploads (the stream is idle), then the launches, one synchronisation
    bool ok = true;
    for (size_t ai = 0; ai < adm.size() && ok; ++ai) {
        SReq* q = adm[ai].q;
        ok &= cudaMemcpyAsync(as<RowInfo>(s->info) + q->r0, ris[ai].data(), (size_t)q->nrows * sizeof(RowInfo),
                              cudaMemcpyHostToDevice, c->st) == cudaSuccess;
        for (uint32_t bid : q->bids) {
            ok &= cudaMemcpyAsync(as<Bucket>(s->pbuckets) + bid, &s->pdesc[bid], sizeof(Bucket),
                                  cudaMemcpyHostToDevice, c->st) == cudaSuccess;
            ok &= cudaMemsetAsync(as<Deficit>(s->bdef) + bid, 0, sizeof(Deficit), c->st) == cudaSuccess;
        }
    }
    for (size_t ai = 0; ai < adm.size() && ok; ++ai) {
        SReq* q = adm[ai].q;
        launch_setup_rows(as<RowInfo>(s->info) + q->r0, q->nrows, as<RowMod>(s->mods) + q->r0, c->st);
        launch_acc_init(q->nrows, 0, as<uint4>(s->acc) + q->r0, nullptr, c->st);
        s->ws.launches += 2;
        if (nitems[ai]) {
            launch_iterate(q->L, as<Bucket>(s->pbuckets), as<RowInfo>(s->info), as<RowMod>(s->mods), q->r0, q->nrows,
                           (uint32_t)item_off[ai], (uint32_t)nitems[ai], Ks[ai], as<uint4>(s->ipart), c->st);
            launch_tail_merge(q->L, as<Bucket>(s->pbuckets), as<RowInfo>(s->info), as<RowMod>(s->mods),
                              as<uint4>(s->ipart), Ks[ai], q->r0, q->nrows, as<uint4>(s->acc), as<Deficit>(s->bdef),
                              c->st);
            launch_clear_tail(as<RowInfo>(s->info), q->r0, q->nrows, c->st);
            s->ws.launches += 3;
        }
    }
    cudaEventRecord(s->e1, c->st);
    if (!ok || cudaStreamSynchronize(c->st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        cudaGetLastError();
        fail_admitted(WL_ERR_CUDA);
        return;
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, s->e0, s->e1);
    s->ws.ms_admit += ms;
}

// Requests whose every bucket is done: their lift (k_finish over the merged
// running products) is queued behind the step, and the step's end recorded.
static int serve_queue_finishes(wl_server* s, wl_server::Slot& sl) {
    wl_ctx* c = s->c;
    for (SReq* q : s->active) {
        if (q->finishing || q->cancel_seen) continue;
        bool done = true;
        for (uint32_t bid : q->bids) done &= s->sb[bid].done();
        if (!done) continue;
        launch_finish(q->L, as<Bucket>(s->pbuckets), as<RowInfo>(s->info), as<RowMod>(s->mods), nullptr, nullptr, 1,
                      nullptr, q->r0, q->nrows, q->qcap == 0 ? 1 : 0, as<RowOut>(s->out), c->st, as<uint4>(s->acc),
                      as<Deficit>(s->bdef), nullptr, nullptr);
        s->ws.launches++;
        q->finishing = true;
        sl.finishing.push_back(q);
    }
    cudaEventRecord(sl.e1, c->st);
    CK(cudaGetLastError());
    sl.inflight = true;
    return 0;
}

// One scheduler step, queued without waiting: every bucket with columns left
// advances by one chunk, then the lift of the requests that are done.
static int serve_step(wl_server* s) {
    wl_ctx* c = s->c;
    wl_server::Slot& sl = s->slot[s->cur];      // not in flight: the loop completes it first
    // kind 0: sparse columns of the resident table, 1: dense ones, 2: a chunk of
    // the number line above 2^32 (integers [c0, c0 + len), sieved this step)
    struct Work { uint32_t bid; uint64_t c0, len; int kind; };
    std::vector<Work> work;
    // The step's descriptor table covers every slot a merge may meet (a merge
    // over a span of rows may meet stale bucket ids of freed rows): slots
    // without work this step have nsplit = 0.  Slots are handed out lowest
    // first, so the active ones lie below `top`; the device table is written
    // up to max(top, what this set of buffers held before), so that no entry
    // above `top` keeps splits of an earlier step.
    uint32_t top = 0;
    for (SReq* q : s->active)
        for (uint32_t bid : q->bids) top = std::max(top, bid + 1);
    const uint32_t upload = std::min(s->bucket_cap, std::max(top, sl.dirty_top));
    size_t nact = 0;
    for (uint32_t bid = 0; bid < top; ++bid) nact += s->sb[bid].used && !s->sb[bid].idle();
    if (!nact) {                                 // only lifts to queue
        cudaEventRecord(sl.e0, c->st);
        return serve_queue_finishes(s, sl);
    }
    // each bucket's share of the step's cell budget.  Costs in cells: a dense
    // column about five (prefix fold + windowed buckets), an integer above 2^32
    // its share of the sieve plus a cell per prime.  Equal shares, or shares
    // weighted by 1 / sqrt(the request's work left), so that small requests
    // finish in a step or two while large ones keep a floor of a quarter of an
    // equal share; budget a bucket cannot use goes to the others.  (Measured
    // on the 2,000-request stream: weights 1 / sqrt(work) with a quarter floor
    // gave the steadiest tail; 1 / work with an eighth floor, or either with a
    // half floor, and equal shares gave longer ones.)
    auto work_left = [](const SBucket& b) {
        double r = 0;
        if (b.pos < b.ncols) {
            const uint64_t dl = b.pos < b.cdense ? b.cdense - b.pos : 0;
            const uint64_t sl = b.ncols - std::max(b.pos, b.cdense);
            r += (double)b.nrows * (5.0 * (double)dl + (double)sl);
        }
        if (b.bpos < b.bend)
            r += (double)(b.bend - b.bpos) * (BIG_SIEVE_CELLS + (double)b.nrows / std::log((double)b.bpos));
        return r;
    };
    const double budget = (double)s->step_cells;
    std::vector<double> wgt(top, 0.0), left(top, 0.0), share_of(top, 0.0);
    double wsum = 0;
    for (SReq* q : s->active) {
        double R = 0;
        for (uint32_t bid : q->bids) {
            if (bid >= top || !s->sb[bid].used || s->sb[bid].idle()) continue;
            left[bid] = work_left(s->sb[bid]);
            R += left[bid];
        }
        for (uint32_t bid : q->bids) {
            if (bid >= top || left[bid] <= 0) continue;
            wgt[bid] = s->shares == WL_SHARES_EQUAL ? 1.0 : 1.0 / std::sqrt(std::max(R, 1.0));
            wsum += wgt[bid];
        }
    }
    double spare = 0, wrest = 0;
    for (uint32_t bid = 0; bid < top; ++bid) {
        if (wgt[bid] <= 0) continue;
        share_of[bid] = std::max(budget * wgt[bid] / wsum, budget / (4.0 * (double)nact));
        if (left[bid] < share_of[bid]) { spare += share_of[bid] - left[bid]; share_of[bid] = left[bid]; }
        else wrest += wgt[bid];
    }
    for (uint32_t bid = 0; bid < top; ++bid)
        if (wgt[bid] > 0 && left[bid] > share_of[bid] && wrest > 0) share_of[bid] += spare * wgt[bid] / wrest;
    double W = 0;
    for (uint32_t bid = 0; bid < top; ++bid) {
        SBucket& b = s->sb[bid];
        if (!b.used || b.idle()) continue;
        const double share = std::max(share_of[bid], 1.0);
        Work w;
        w.bid = bid;
        double per, cost;
        if (b.pos < b.ncols) {
            w.c0 = b.pos;
            w.kind = b.pos < b.cdense ? 1 : 0;
            per = (double)b.nrows * (w.kind ? 5.0 : 1.0);
            const uint64_t want = (uint64_t)std::max(share / per, w.kind ? 1024.0 : 8192.0);
            const uint64_t end = w.kind ? b.cdense : b.ncols;
            w.len = std::min<uint64_t>(end - b.pos, want);
            // do not leave a sliver behind
            if (end - b.pos - w.len < w.len / 4) w.len = end - b.pos;
            cost = per * (double)w.len;
        } else {
            // whole sieve segments from bpos (a multiple of BIG_SPAN); the
            // sieve's per-CTA offsets (CTAs x sieving primes) stay below 1 GiB
            w.c0 = b.bpos;
            w.kind = 2;
            per = BIG_SIEVE_CELLS + (double)b.nrows / std::log((double)b.bpos);
            const uint64_t rest = (b.bend - b.bpos + BIG_SPAN - 1) / BIG_SPAN;     // segments left
            uint64_t nseg = (uint64_t)std::ceil(share / per / (double)BIG_SPAN);
            const uint64_t max_cta = std::max<uint64_t>(1, (1ull << 28) / std::max<uint32_t>(b.nroot, 1));
            nseg = std::max<uint64_t>(1, std::min<uint64_t>(nseg, 8 * max_cta));
            if (rest - std::min(rest, nseg) < nseg / 4) nseg = rest;
            nseg = std::min(nseg, rest);
            w.len = nseg * BIG_SPAN;
            cost = per * (double)w.len;
        }
        W += cost;
        work.push_back(w);
    }
    const double target_threads = (double)c->sms * 2048.0 * 4.0;
    std::vector<Bucket> sbk(upload);
    memset(sbk.data(), 0, sbk.size() * sizeof(Bucket));
    struct Grp { int L, rpt, kind; std::vector<SweepItem> items; };
    std::vector<Grp> groups;
    uint64_t part_total = 0, bwords = 0, boffs_need = 0, bseg_need = 0;
    uint32_t def_total = 0;
    std::vector<uint32_t> bucket_splits(top, 0);
    std::vector<uint64_t> bkeys, blos;
    for (const Work& w : work) {
        const SBucket& b = s->sb[w.bid];
        Bucket& x = sbk[w.bid];
        x = s->pdesc[w.bid];
        int rpt = 1;
        uint32_t min_tps = 1;
        uint64_t S;
        if (w.kind == 2) {
            // the chunk's bitmap region: its words from bwords on
            const uint64_t nseg = w.len / BIG_SPAN, nw = nseg * BIG_WORDS;
            if (bwords + nw >= (1ull << 32)) return WL_ERR_UNSUPPORTED;
            if (bkeys.empty()) { bkeys.assign(top, 0); blos.assign(top, 0); }
            bkeys[w.bid] = b.key;
            blos[w.bid] = w.c0;
            x.cbase = (uint32_t)bwords;
            x.ncols = (uint32_t)nw;
            bwords += nw;
            const uint64_t ncta = (nseg + 7) / 8;
            boffs_need = std::max(boffs_need, ncta * std::max<uint32_t>(b.nroot, 1));
            bseg_need = std::max(bseg_need, nseg);
            if (b.nrows >= 512) rpt = 2;
            // splits by the sweep's cells per row: the chunk's primes, about len / ln(c0)
            S = (uint64_t)std::ceil((double)rpt * ((double)w.len / std::log((double)w.c0)) * target_threads / W);
            S = std::max<uint64_t>(1, std::min<uint64_t>(S, std::max<uint64_t>(1, nw / 256)));
            x.cdense = 0;
            x.ndense = 0;
        } else {
            const bool dense = w.kind == 1;
            x.cbase = (uint32_t)w.c0;
            x.ncols = (uint32_t)w.len;
            if (dense) {
                uint32_t dtps;
                dense_shape(b.nrows, &rpt, &dtps);
                min_tps = 8;
            } else {
                rpt = sparse_rpt_for(c->tune.sparse_rpt[b.L - 2], b.nrows);
            }
            const double per = (double)b.nrows * (dense ? 5.0 : 1.0);
            S = (uint64_t)std::ceil((double)rpt * per / (double)b.nrows * (double)w.len * target_threads / W);
            const uint64_t minlen = dense ? 256 : 2048;
            S = std::max<uint64_t>(1, std::min<uint64_t>(S, std::max<uint64_t>(1, w.len / minlen)));
            if (dense) S = std::max<uint64_t>(S, std::min<uint64_t>((w.len + 1023) / 1024, w.len / 256 ? w.len / 256 : 1));
            x.cdense = dense ? (uint32_t)w.len : 0;
            x.ndense = dense ? (uint32_t)S : 0;
        }
        x.nsplit = (uint32_t)S;
        x.dstart = 0;
        x.part_base = part_total;
        x.def_base = def_total;
        part_total += S * b.nrows;
        def_total += (uint32_t)S;
        bucket_splits[w.bid] = (uint32_t)S;
        std::vector<RowTile> tiles;
        row_tiles(b.nrows, rpt, min_tps, tiles, w.kind == 1);
        for (const RowTile& t : tiles) {
            Grp* g = nullptr;
            for (auto& gg : groups)
                if (gg.L == (int)b.L && gg.rpt == t.rpt && gg.kind == w.kind) g = &gg;
            if (!g) {
                groups.push_back({ (int)b.L, t.rpt, w.kind, {} });
                g = &groups.back();
            }
            tile_items(t, 0, (uint32_t)S, [&](uint32_t r0, uint32_t s2, uint32_t tp) {
                g->items.push_back({ w.bid, r0, s2, tp });
            });
        }
    }
    std::vector<SweepItem> all;
    for (auto& g : groups) all.insert(all.end(), g.items.begin(), g.items.end());
    RC(ensure_step(s, sl.sbuckets, (size_t)s->bucket_cap * sizeof(Bucket)));
    RC(ensure_step(s, sl.items, all.size() * sizeof(SweepItem) + 16));
    RC(ensure_step(s, sl.part, part_total * 16 + 16));
    RC(ensure_step(s, sl.defs, (size_t)def_total * sizeof(Deficit) + 16));
    if (bwords) {
        RC(ensure_step(s, sl.bbitmap, bwords * 4));
        RC(ensure_step(s, sl.bsegcount, bseg_need * 4 + 16));
        RC(ensure_step(s, sl.boffs, boffs_need * 4 + 16));
        RC(ensure_step(s, sl.bkeys, (size_t)s->bucket_cap * 8));
        RC(ensure_step(s, sl.blos, (size_t)s->bucket_cap * 8));
    }
    cudaEventRecord(sl.e0, c->st);
    CK(cudaMemcpyAsync(sl.sbuckets.p, sbk.data(), sbk.size() * sizeof(Bucket), cudaMemcpyHostToDevice, c->st));
    sl.dirty_top = top;
    CK(cudaMemcpyAsync(sl.items.p, all.data(), all.size() * sizeof(SweepItem), cudaMemcpyHostToDevice, c->st));
    if (bwords) {
        CK(cudaMemcpyAsync(sl.bkeys.p, bkeys.data(), (size_t)top * 8, cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(sl.blos.p, blos.data(), (size_t)top * 8, cudaMemcpyHostToDevice, c->st));
        // sieve every chunk above 2^32 into its bitmap region (the sieving
        // primes 67 .. sqrt(key) come from the resident column table; one
        // launch after another on the stream, so they share the offsets)
        for (const Work& w : work) {
            if (w.kind != 2) continue;
            const SBucket& b = s->sb[w.bid];
            const uint32_t nseg = (uint32_t)(w.len / BIG_SPAN);
            launch_sieve_big(w.c0, std::min(w.c0 + w.len, b.bend), nseg, 8, as<uint32_t>(c->cols) + 18, b.nroot,
                             as<uint32_t>(sl.boffs), as<uint32_t>(sl.bbitmap) + sbk[w.bid].cbase,
                             as<uint32_t>(sl.bsegcount), c->st);
            s->ws.launches++;
        }
    }
    size_t ioff = 0;
    for (auto& g : groups) {
        if (g.kind == 2)
            launch_sweep_bits(g.L, g.rpt, (uint32_t)g.items.size(), as<Bucket>(sl.sbuckets),
                              as<SweepItem>(sl.items) + ioff, as<RowMod>(s->mods), as<uint32_t>(sl.bbitmap), 0,
                              as<uint64_t>(sl.bkeys), as<uint4>(sl.part), as<Deficit>(sl.defs), c->st,
                              as<uint64_t>(sl.blos));
        else if (g.kind == 1)
            launch_sweep_dense(g.L, g.rpt, (uint32_t)g.items.size(), as<Bucket>(sl.sbuckets), as<SweepItem>(sl.items) + ioff,
                               as<RowMod>(s->mods), as<uint32_t>(c->cols), nullptr, as<uint4>(sl.part),
                               as<Deficit>(sl.defs), c->st,
                               c->tune.dense_kernel[g.L - 2], (uint32_t)c->tune.dense_hstep[g.L - 2]);
        else
            launch_sweep(c->tune.sparse_variant[g.L - 2], g.L, g.rpt, (uint32_t)g.items.size(), as<Bucket>(sl.sbuckets),
                         as<SweepItem>(sl.items) + ioff, as<RowMod>(s->mods), as<uint32_t>(c->cols),
                         as<uint4>(sl.part), as<Deficit>(sl.defs), c->st, col_groups(c));
        s->ws.launches++;
        ioff += g.items.size();
    }
    // fold the chunk into the resident running products: one launch per limb
    // width over the span of the active requests' rows (rows of buckets
    // without splits this step, or not in use, are left alone by the kernel)
    for (int L = 2; L <= 4; ++L) {
        uint32_t lo = UINT32_MAX, hi = 0, maxs = 0;
        for (SReq* q : s->active) {
            if (q->L != L) continue;
            uint32_t m = 0;
            for (uint32_t bid : q->bids) if (bid < top) m = std::max(m, bucket_splits[bid]);
            if (!m) continue;
            maxs = std::max(maxs, m);
            lo = std::min(lo, q->r0);
            hi = std::max(hi, q->r0 + q->nrows);
        }
        if (!maxs) continue;
        if (maxs >= (uint32_t)c->tune.merge_cta_min)
            launch_merge_cta(L, as<Bucket>(sl.sbuckets), as<RowInfo>(s->info), as<RowMod>(s->mods),
                             as<uint4>(sl.part), as<Deficit>(sl.defs), lo, hi - lo, as<uint4>(s->acc),
                             as<Deficit>(s->bdef), c->st);
        else
            launch_merge(L, as<Bucket>(sl.sbuckets), as<RowInfo>(s->info), as<RowMod>(s->mods),
                         as<uint4>(sl.part), as<Deficit>(sl.defs), lo, hi - lo, as<uint4>(s->acc),
                         as<Deficit>(s->bdef), c->st);
        s->ws.launches++;
    }
    // positions advance now, so the next step is planned while this one runs
    for (const Work& w : work) {
        SBucket& b = s->sb[w.bid];
        if (w.kind == 2) b.bpos = std::min(w.c0 + w.len, b.bend);
        else b.pos += w.len;
    }
    return serve_queue_finishes(s, sl);
}

// The rows of a request whose lift has run (the step it followed is
// complete): read them back, in ascending p, with the checksum and the
// result lines (cl_wilson.cpp:872-900).
static int serve_read_rows(wl_server* s, SReq* q) {
    wl_ctx* c = s->c;
    const bool full = q->qcap == 0;
    std::vector<RowOut> ro(q->nrows);
    CK(cudaMemcpyAsync(ro.data(), as<RowOut>(s->out) + q->r0, (size_t)q->nrows * sizeof(RowOut),
                       cudaMemcpyDeviceToHost, c->st3));
    CK(cudaStreamSynchronize(c->st3));
    std::vector<uint32_t> ord(q->nrows);
    for (uint32_t k = 0; k < q->nrows; ++k) ord[k] = k;
    std::sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b) { return q->primes[a] < q->primes[b]; });
    uint64_t ck = 0;
    int err = 0;
    q->rows.resize(q->nrows);
    for (uint32_t j = 0; j < q->nrows; ++j) {
        const uint32_t k = ord[j];
        wl_row& w = q->rows[j];
        memset(&w, 0, sizeof(w));
        w.p = q->primes[k];
        w.s0 = ro[k].s0;
        w.s1 = ro[k].s1;
        w.rem = ro[k].rem;
        w.quot = ro[k].quot;
        w.type = q->types[k];
        w.status = ro[k].status;
        if (full) {
            ck += w.p + w.rem + w.quot;
            int32_t v;
            if (result_of(w, &v)) q->lines.push_back(wl_result{ w.p, v });
            if (w.status == 1 && !err) err = WL_ERR_WILSON_CHECK;
            if (w.status == 2 && !err) err = WL_ERR_NO_REPR;
        } else {
            ck += w.p + w.s0 + w.s1;
        }
    }
    q->checksum = ck;
    return err;
}

static void serve_end(wl_server* s, SReq* q, int state, int rc) {
    // called with s->mu held
    q->state = state;
    q->rc = rc;
    q->t_done = s->now_ms();
    if (state == WL_REQ_DONE) { s->ws.completed++; s->ws.rows_done += q->rows.size(); s->ws.cells += q->cells; }
    else if (state == WL_REQ_CANCELLED) s->ws.cancelled++;
    else s->ws.failed++;
    q->tested = state == WL_REQ_DONE ? q->rows.size() : 0;
    s->stats = s->ws;
    q->tps.clear();
    q->tps.shrink_to_fit();
    s->cv_done.notify_all();
}

// Ends a request that is in s->active: frees its rows and slots and removes it.
static void serve_retire(wl_server* s, SReq* q, int state, int rc) {
    std::lock_guard<std::mutex> lk(s->mu);
    serve_release(s, q);
    serve_end(s, q, state, rc);
    s->active.erase(std::find(s->active.begin(), s->active.end(), q));
}

// Waits for the step in `sl`, takes its device time, and completes the
// requests whose lift followed it.  err != 0 (a failed step) fails them.
static void serve_complete(wl_server* s, wl_server::Slot& sl, int err = 0) {
    if (!sl.inflight) return;
    const double t = s->now_ms();
    if (!err && cudaEventSynchronize(sl.e1) != cudaSuccess) err = WL_ERR_CUDA;
    if (!err) {
        float ms = 0;
        cudaEventElapsedTime(&ms, sl.e0, sl.e1);
        s->ws.ms_steps += ms;
        s->ws.steps++;
    }
    for (SReq* q : sl.finishing) {
        const int rc = err ? err : serve_read_rows(s, q);
        serve_retire(s, q, rc ? WL_REQ_FAILED : WL_REQ_DONE, rc);
    }
    sl.finishing.clear();
    sl.inflight = false;
    s->ws.ms_wall_finish += s->now_ms() - t;
}

// Completes every step in flight, the older first: the stream is then idle.
static void serve_drain(wl_server* s, int err = 0) {
    serve_complete(s, s->slot[s->cur], err);       // the older of the two, if both are in flight
    serve_complete(s, s->slot[s->cur ^ 1], err);
    if (err) cudaGetLastError();
}

static void serve_loop(wl_server* s) {
    cudaSetDevice(s->c->device);
    while (true) {
        // queued requests to admit (cancelled ones end here), and cancelled active ones
        std::vector<SReq*> cands, cancelled;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            while (!s->stop && s->active.empty() && !(s->admit_pending && !s->queue.empty())) s->cv_work.wait(lk);
            if (s->stop) break;
            const bool try_admit = s->admit_pending;
            s->admit_pending = false;
            for (auto it = s->queue.begin(); it != s->queue.end() && try_admit;) {
                if ((*it)->cancel) {
                    serve_end(s, *it, WL_REQ_CANCELLED, 0);
                    it = s->queue.erase(it);
                } else {
                    cands.push_back(*it);
                    ++it;
                }
            }
            for (SReq* q : s->active)
                if (q->cancel && !q->finishing && !q->cancel_seen) cancelled.push_back(q);
        }
        if (!cancelled.empty()) {
            // no step may still use their rows: drain, then free them
            serve_drain(s);
            for (SReq* q : cancelled) {
                q->cancel_seen = true;
                for (uint32_t bid : q->bids) s->sb[bid].stop = true;
                serve_retire(s, q, WL_REQ_CANCELLED, 0);
            }
        }
        if (!cands.empty()) {
            // admission synchronises the stream and may grow the column table
            serve_drain(s);
            std::vector<int> res;
            const double t = s->now_ms();
            serve_admit_batch(s, cands, res);
            s->ws.ms_wall_admit += s->now_ms() - t;
            std::lock_guard<std::mutex> lk(s->mu);
            for (size_t k = 0; k < cands.size(); ++k) {
                SReq* q = cands[k];
                if (res[k] == 1) continue;                  // waits for rows to free up
                s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
                if (res[k]) {
                    serve_release(s, q);
                    serve_end(s, q, WL_REQ_FAILED, res[k]);
                    continue;
                }
                q->state = WL_REQ_ACTIVE;
                q->t_admit = s->now_ms();
                s->active.push_back(q);
                q->tested = q->nrows;
                s->ws.admitted++;
            }
            s->ws.peak_rows = std::max(s->ws.peak_rows, s->pool.used);
            s->ws.peak_active = std::max<uint32_t>(s->ws.peak_active, (uint32_t)s->active.size());
            s->stats = s->ws;
        }
        // queue the next step into the free set of buffers, then complete the
        // previous step while this one runs
        bool work = false;                           // chunks to sweep or lifts to queue
        for (SReq* q : s->active) work |= !q->finishing && !q->cancel_seen;
        if (work) {
            serve_complete(s, s->slot[s->cur]);
            const double t = s->now_ms();
            const int e = serve_step(s);
            s->ws.ms_wall_steps += s->now_ms() - t;
            if (e) {
                // a failed step: every request still running fails with its code
                serve_drain(s, e);
                std::vector<SReq*> all(s->active);
                for (SReq* q : all) serve_retire(s, q, WL_REQ_FAILED, e);
                continue;
            }
        }
        serve_complete(s, s->slot[s->cur ^ 1]);
        if (work) s->cur ^= 1;
        else serve_complete(s, s->slot[s->cur]);
        std::lock_guard<std::mutex> lk(s->mu);
        s->stats = s->ws;
    }
    serve_drain(s);
}

extern "C" {

int wl_server_open(const wl_server_opts* opts, wl_server** out) {
    if (!out) return WL_ERR_ARG;
    *out = nullptr;
    wl_server_opts o;
    memset(&o, 0, sizeof(o));
    if (opts) o = *opts;
    const uint64_t bytes = o.pool_bytes ? o.pool_bytes : (1ull << 30);
    if (bytes / WL_SERVER_ROW_BYTES < 1024) return WL_ERR_ARG;
    wl_server* s = new wl_server();
    int rc = wl_open(o.device, &s->c);
    if (rc) { delete s; return rc; }
    if (o.tuning && (rc = wl_set_tuning(s->c, o.tuning))) {
        wl_close(s->c);
        delete s;
        return rc;
    }
    s->pool_cap = (uint32_t)std::min<uint64_t>(bytes / WL_SERVER_ROW_BYTES, 1u << 30);
    s->step_cells = o.step_cells ? o.step_cells : (1ull << 32);
    if (o.shares > WL_SHARES_EQUAL) {
        wl_close(s->c);
        delete s;
        return WL_ERR_ARG;
    }
    s->shares = o.shares;
    s->bucket_cap = 3 * 1024;
    s->sb.assign(s->bucket_cap, SBucket());
    s->pdesc.resize(s->bucket_cap);
    memset(s->pdesc.data(), 0, s->pdesc.size() * sizeof(Bucket));
    for (uint32_t b = 0; b < s->bucket_cap; ++b) s->free_bids.insert(b);
    s->pool.reset(s->pool_cap);
    if (ensure(s->info, (size_t)s->pool_cap * sizeof(RowInfo)) || ensure(s->mods, (size_t)s->pool_cap * sizeof(RowMod)) ||
        ensure(s->acc, (size_t)s->pool_cap * 16) || ensure(s->out, (size_t)s->pool_cap * sizeof(RowOut)) ||
        ensure(s->pbuckets, s->bucket_cap * sizeof(Bucket)) || ensure(s->bdef, s->bucket_cap * sizeof(Deficit)) ||
        cudaEventCreate(&s->e0) != cudaSuccess || cudaEventCreate(&s->e1) != cudaSuccess ||
        cudaEventCreate(&s->slot[0].e0) != cudaSuccess || cudaEventCreate(&s->slot[0].e1) != cudaSuccess ||
        cudaEventCreate(&s->slot[1].e0) != cudaSuccess || cudaEventCreate(&s->slot[1].e1) != cudaSuccess) {
        cudaGetLastError();
        DevBuf* bufs[] = { &s->info, &s->mods, &s->acc, &s->out, &s->pbuckets, &s->bdef };
        for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
        wl_close(s->c);
        delete s;
        return WL_ERR_NOMEM;
    }
    // the step buffers' pool, which keeps what is freed into it; each set of
    // step buffers starts at the size a step of the default budget takes
    // (about two rows of split products per thread of the sweep, a split
    // deficit per thread, a few thousand items)
    cudaMemPoolProps pp;
    memset(&pp, 0, sizeof(pp));
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = s->c->device;
    const uint64_t keep_all = ~0ull;
    bool ok = cudaMemPoolCreate(&s->mpool, &pp) == cudaSuccess &&
              cudaMemPoolSetAttribute(s->mpool, cudaMemPoolAttrReleaseThreshold, (void*)&keep_all) == cudaSuccess;
    const size_t threads = (size_t)s->c->sms * 2048 * 4;
    for (auto& sl : s->slot)
        ok = ok && !ensure_step(s, sl.sbuckets, (size_t)s->bucket_cap * sizeof(Bucket)) &&
             !ensure_step(s, sl.part, threads * 2 * 16) && !ensure_step(s, sl.items, 16384 * sizeof(SweepItem)) &&
             !ensure_step(s, sl.defs, threads * sizeof(Deficit));
    if (!ok) {
        cudaGetLastError();
        wl_server_close(s);                              // no worker yet: frees what there is
        return WL_ERR_NOMEM;
    }
    cudaMemset(s->pbuckets.p, 0, s->bucket_cap * sizeof(Bucket));
    cudaMemset(s->info.p, 0, (size_t)s->pool_cap * sizeof(RowInfo));   // bucket 0 for rows never admitted
    s->worker = std::thread(serve_loop, s);
    *out = s;
    return 0;
}

int wl_server_submit(wl_server* s, uint64_t pmin, uint64_t pmax, uint64_t q_cap, uint64_t* id) {
    if (!s) return WL_ERR_ARG;
    RC(wl_check_range(pmin, pmax));
    SReq* q = new SReq();
    q->pmin = pmin;
    q->pmax = pmax;
    q->qcap = q_cap;
    std::lock_guard<std::mutex> lk(s->mu);
    q->id = s->next_id++;
    q->t_submit = s->now_ms();
    s->reqs[q->id] = q;
    s->queue.push_back(q);
    s->admit_pending = true;
    if (id) *id = q->id;
    s->cv_work.notify_all();
    return 0;
}

static void fill_info(const SReq* q, wl_request_info* info) {
    if (!info) return;
    memset(info, 0, sizeof(*info));
    info->id = q->id;
    info->state = q->state;
    info->rc = q->rc;
    info->tested = q->tested;
    // the scheduler writes these before the state changes (under the mutex)
    if (q->state == WL_REQ_ACTIVE || q->state == WL_REQ_DONE) {
        for (int t = 0; t < 3; ++t) info->targets[t] = q->targets[t];
        info->cells = q->cells;
    }
    if (q->state == WL_REQ_DONE) {
        info->checksum = q->checksum;
        info->results = (uint32_t)q->lines.size();
    }
    info->ms_queued = q->t_admit > 0 ? q->t_admit - q->t_submit : 0;
    info->ms_latency = q->t_done > 0 ? q->t_done - q->t_submit : 0;
}

static SReq* find_req(wl_server* s, uint64_t id) {
    auto it = s->reqs.find(id);
    return it == s->reqs.end() ? nullptr : it->second;
}

int wl_server_poll(wl_server* s, uint64_t id, wl_request_info* info) {
    if (!s) return WL_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    SReq* q = find_req(s, id);
    if (!q) return WL_ERR_ARG;
    fill_info(q, info);
    return q->state >= WL_REQ_DONE ? 0 : 1;
}

int wl_server_wait(wl_server* s, uint64_t id, wl_request_info* info, double timeout_ms) {
    if (!s) return WL_ERR_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    SReq* q = find_req(s, id);
    if (!q) return WL_ERR_ARG;
    auto ended = [&] { return q->state >= WL_REQ_DONE; };
    if (timeout_ms < 0) s->cv_done.wait(lk, ended);
    else s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), ended);
    fill_info(q, info);
    return q->state >= WL_REQ_DONE ? 0 : 1;
}

int wl_server_results(wl_server* s, uint64_t id, wl_result* res, size_t cap, size_t* n) {
    if (!s) return WL_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    SReq* q = find_req(s, id);
    if (!q || q->state != WL_REQ_DONE) return WL_ERR_ARG;
    if (n) *n = q->lines.size();
    if (res) memcpy(res, q->lines.data(), std::min(cap, q->lines.size()) * sizeof(wl_result));
    return (res && cap < q->lines.size()) ? WL_ERR_CAPACITY : 0;
}

int wl_server_rows(wl_server* s, uint64_t id, wl_row* rows, size_t cap, size_t* n) {
    if (!s) return WL_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    SReq* q = find_req(s, id);
    if (!q || q->state != WL_REQ_DONE) return WL_ERR_ARG;
    if (n) *n = q->rows.size();
    if (rows) memcpy(rows, q->rows.data(), std::min(cap, q->rows.size()) * sizeof(wl_row));
    return (rows && cap < q->rows.size()) ? WL_ERR_CAPACITY : 0;
}

int wl_server_cancel(wl_server* s, uint64_t id) {
    if (!s) return WL_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    SReq* q = find_req(s, id);
    if (!q) return WL_ERR_ARG;
    q->cancel = true;
    s->admit_pending = true;
    s->cv_work.notify_all();
    return 0;
}

int wl_server_release(wl_server* s, uint64_t id) {
    if (!s) return WL_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    SReq* q = find_req(s, id);
    if (!q || q->state < WL_REQ_DONE) return WL_ERR_ARG;
    delete q;
    s->reqs.erase(id);
    return 0;
}

int wl_server_stats_get(wl_server* s, wl_server_stats* st) {
    if (!s || !st) return WL_ERR_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *st = s->stats;
    return 0;
}

void wl_server_close(wl_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->c->device);
    cudaStreamSynchronize(s->c->st);
    DevBuf* bufs[] = { &s->info, &s->mods, &s->acc, &s->out, &s->pbuckets, &s->bdef, &s->ipart };
    for (DevBuf* b : bufs) if (b->p) cudaFree(b->p);
    for (auto& sl : s->slot) {
        DevBuf* sb[] = { &sl.sbuckets, &sl.items, &sl.part, &sl.defs, &sl.bbitmap, &sl.bsegcount, &sl.boffs,
                         &sl.bkeys, &sl.blos };
        for (DevBuf* b : sb) if (b->p) cudaFreeAsync(b->p, s->c->st);
        if (sl.e0) cudaEventDestroy(sl.e0);
        if (sl.e1) cudaEventDestroy(sl.e1);
    }
    cudaStreamSynchronize(s->c->st);
    if (s->mpool) cudaMemPoolDestroy(s->mpool);
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    for (auto& kv : s->reqs) delete kv.second;
    wl_close(s->c);
    delete s;
}

}  // extern "C"
