// wl_plan.h -- split planning of the column sweeps: how many splits each
// bucket gets, and the cost model behind the dense sweep's split boundaries;
// the layout of the test-prime windows.  Host code only (no CUDA).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

// Cells per row that a dense column at prime q costs for class target T: one
// for the prefix product plus 7/8 of one per 3-bit window of the exponent's
// low part, s ~ log2(8 T ln(q) / q^2) bits when the high part changes every 8
// columns (k_sweep_dense), at most the exponent's length.
inline double dense_cells_at(double T, double q) {
    const double e = T / (q - 1.0);
    double sb = std::log2(std::max(1.0, 8.0 * T * std::log(q) / (q * q)));
    sb = std::min(sb, std::log2(std::max(e, 1.0)) + 1.0);
    return 1.0 + 0.875 * std::ceil(sb / 3.0);
}

// Cumulative dense cost over q in [2, qd] on a log grid: cum[k] for q = grid[k].
inline void dense_cost_grid(double T, double qd, std::vector<double>& grid, std::vector<double>& cum, double* cols_est) {
    const int N = 2048;
    grid.assign(N + 1, 0.0);
    cum.assign(N + 1, 0.0);
    const double u0 = std::log(2.0), u1 = std::log(std::max(qd, 3.0));
    const double du = (u1 - u0) / N;
    double c = 0, n = 0;
    grid[0] = 2.0;
    for (int k = 1; k <= N; ++k) {
        const double u = u0 + (k - 0.5) * du, q = std::exp(u);
        const double dn = q * du / u;            // primes in the step ~ dq / ln q
        n += dn;
        c += dn * dense_cells_at(T, q);
        grid[k] = std::exp(u0 + k * du);
        cum[k] = c;
    }
    *cols_est = n;
}

// Value of q where dense split k of Sd ends: the point of equal cumulative
// cost k/Sd, interpolated inside a grid step (there are more splits than grid
// points when the dense region is long, and a boundary snapped to the grid
// would leave empty splits next to ones many times too long).  Inside a step
// the cost per unit of ln q grows about like q, so the interpolation is linear
// in q between the grid points.
inline double dense_boundary(const std::vector<double>& grid, const std::vector<double>& cum, uint64_t k, uint64_t Sd) {
    const double target = cum.back() * (double)k / (double)Sd;
    size_t j = std::lower_bound(cum.begin(), cum.end(), target) - cum.begin();
    if (j >= cum.size()) j = cum.size() - 1;
    double q = grid[j];
    if (j > 0 && cum[j] > cum[j - 1]) {
        const double f = (target - cum[j - 1]) / (cum[j] - cum[j - 1]);
        q = grid[j - 1] + f * (grid[j] - grid[j - 1]);
    }
    return q;
}

// One bucket as the split planner sees it.
struct SplitBucket {
    uint32_t nrows = 0;     // test primes of the bucket
    int rpt = 1;            // rows per thread of its prefix-fold sweep
    uint64_t ndense = 0;    // columns of the dense regime
    uint64_t nsparse = 0;   // columns of the prefix-fold regime
    double dcost = 0;       // modelled cells per row of its dense columns
};

// Dense (Sd) and prefix-fold (Ss) splits of one bucket for work W (row x
// column cells of all buckets) spread over `threads` thread-splits; `scale`
// < 1 lengthens every split (memory budget).
//   dense: equal estimated cost, 256 to 1,024 columns each, so that the
//          per-split combination of window buckets stays small;
//   prefix-fold: at least 2,048 columns, at most 2^17 -- a bucket whose share
//          of the threads is small (few rows next to much dense work) would
//          otherwise run as a few very long CTAs that finish after the rest.
inline void plan_bucket_splits(const SplitBucket& b, double W, double threads, double scale, uint64_t* Sd_out,
                               uint64_t* Ss_out) {
    const uint64_t nd = b.ndense, ns = b.nsparse;
    uint64_t Sd = 0, Ss = 0;
    if (nd > 0) {
        Sd = (uint64_t)std::ceil(b.dcost * threads / W);
        Sd = std::max<uint64_t>(Sd, (nd + 1023) / 1024);
        Sd = std::max<uint64_t>(1, std::min<uint64_t>(Sd, std::max<uint64_t>(1, nd / 256)));
        Sd = std::max<uint64_t>(1, (uint64_t)((double)Sd * scale));
    }
    if (ns > 0) {
        Ss = (uint64_t)std::ceil((double)b.rpt * (double)ns * threads / W);
        Ss = std::max<uint64_t>(Ss, (ns + (1u << 17) - 1) >> 17);
        Ss = std::max<uint64_t>(1, std::min<uint64_t>(Ss, std::max<uint64_t>(1, ns / 2048)));
        Ss = std::max<uint64_t>(1, (uint64_t)((double)Ss * scale));
    }
    if (Sd + Ss == 0) Ss = 1;
    *Sd_out = Sd;
    *Ss_out = Ss;
}

// The split-length scale (<= 1) that keeps the split partials -- one per split
// and row -- within `budget` partials.
inline double split_scale(const std::vector<SplitBucket>& bs, double W, double threads, double budget) {
    double scale = 1.0;
    for (int it = 0; it < 8; ++it) {
        double tot = 0;
        for (const SplitBucket& b : bs) {
            uint64_t a, c;
            plan_bucket_splits(b, W, threads, scale, &a, &c);
            tot += (double)(a + c) * (double)b.nrows;
        }
        if (tot <= budget) break;
        scale *= 0.9 * budget / tot;
    }
    return scale;
}

// Test-prime windows of a batch of ranges, for one launch over all of them.
// Range i covers the odd numbers lo0 + 2j + 1 from lo0 = pmin rounded down to
// even, in nseg segments of `seg_span` integers (seg_span / 64 bitmap words
// and one prime counter each).  It owns ceil((pmax - lo0) / 512) blocks of
// 256 threads, one thread per odd number, so only its own integers are
// tested.  Its words, counters and blocks follow those of range i - 1.
struct WindowPlan {
    uint64_t lo0 = 0;
    uint32_t nseg = 0;
    uint64_t word_off = 0, seg_off = 0, block0 = 0, nblocks = 0;
};

inline void plan_windows(const uint64_t* pmin, const uint64_t* pmax, size_t nr, uint32_t seg_span,
                         std::vector<WindowPlan>& out, uint64_t* words, uint64_t* segs, uint64_t* blocks) {
    out.assign(nr, WindowPlan());
    uint64_t w = 0, s = 0, b = 0;
    for (size_t i = 0; i < nr; ++i) {
        WindowPlan& p = out[i];
        p.lo0 = pmin[i] & ~1ull;
        p.nseg = (uint32_t)((pmax[i] - p.lo0 + seg_span - 1) / seg_span);
        p.word_off = w;
        p.seg_off = s;
        p.block0 = b;
        p.nblocks = (pmax[i] - p.lo0 + 511) / 512;
        w += (uint64_t)p.nseg * (seg_span / 64);
        s += p.nseg;
        b += p.nblocks;
    }
    *words = w;
    *segs = s;
    *blocks = b;
}
