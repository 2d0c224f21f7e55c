// Test driver for clwilson_b200/csrc/wl_plan.h (split planning), used by
// tests/test_split_plan.py.  Commands:
//   bounds T qd Sd     the grid size and total modelled cost, then per dense
//                      boundary k = 1 .. Sd-1 its q and the cumulative cost at q
//   splits nrows rpt ndense nsparse dcost W threads scale     -> Sd Ss
//   scale W threads budget (nrows ndense nsparse dcost)...    -> scale and partials
//   windows seg_span (pmin pmax)...   test-prime window layout: totals (words
//                      segs blocks), then per range lo0 nseg word_off seg_off
//                      block0 nblocks
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "wl_plan.h"

int main(int argc, char** argv) {
    if (argc >= 3 && !strcmp(argv[1], "windows")) {
        const uint32_t span = (uint32_t)strtoul(argv[2], nullptr, 0);
        std::vector<uint64_t> lo, hi;
        for (int i = 3; i + 1 < argc; i += 2) {
            lo.push_back(strtoull(argv[i], nullptr, 0));
            hi.push_back(strtoull(argv[i + 1], nullptr, 0));
        }
        std::vector<WindowPlan> wp;
        uint64_t words = 0, segs = 0, blocks = 0;
        plan_windows(lo.data(), hi.data(), lo.size(), span, wp, &words, &segs, &blocks);
        printf("%" PRIu64 " %" PRIu64 " %" PRIu64 "\n", words, segs, blocks);
        for (const WindowPlan& p : wp)
            printf("%" PRIu64 " %u %" PRIu64 " %" PRIu64 " %" PRIu64 " %" PRIu64 "\n", p.lo0, p.nseg, p.word_off,
                   p.seg_off, p.block0, p.nblocks);
        return 0;
    }
    if (argc >= 5 && !strcmp(argv[1], "bounds")) {
        const double T = atof(argv[2]), qd = atof(argv[3]);
        const uint64_t Sd = strtoull(argv[4], nullptr, 0);
        std::vector<double> grid, cum;
        double cols = 0;
        dense_cost_grid(T, qd, grid, cum, &cols);
        printf("grid %zu total %.17g\n", grid.size(), cum.back());
        for (uint64_t k = 1; k < Sd; ++k) {
            const double q = dense_boundary(grid, cum, k, Sd);
            size_t j = std::upper_bound(grid.begin(), grid.end(), q) - grid.begin();
            double c = cum.back();
            if (j > 0 && j < grid.size())
                c = cum[j - 1] + (cum[j] - cum[j - 1]) * (q - grid[j - 1]) / (grid[j] - grid[j - 1]);
            printf("%.17g %.17g\n", q, c);
        }
        return 0;
    }
    if (argc >= 10 && !strcmp(argv[1], "splits")) {
        SplitBucket b;
        b.nrows = (uint32_t)atol(argv[2]);
        b.rpt = atoi(argv[3]);
        b.ndense = strtoull(argv[4], nullptr, 0);
        b.nsparse = strtoull(argv[5], nullptr, 0);
        b.dcost = atof(argv[6]);
        uint64_t Sd, Ss;
        plan_bucket_splits(b, atof(argv[7]), atof(argv[8]), atof(argv[9]), &Sd, &Ss);
        printf("%" PRIu64 " %" PRIu64 "\n", Sd, Ss);
        return 0;
    }
    if (argc >= 9 && !strcmp(argv[1], "scale") && (argc - 5) % 4 == 0) {
        const double W = atof(argv[2]), threads = atof(argv[3]), budget = atof(argv[4]);
        std::vector<SplitBucket> bs;
        for (int i = 5; i + 3 < argc; i += 4) {
            SplitBucket b;
            b.nrows = (uint32_t)atol(argv[i]);
            b.rpt = b.nrows >= 512 ? 2 : 1;
            b.ndense = strtoull(argv[i + 1], nullptr, 0);
            b.nsparse = strtoull(argv[i + 2], nullptr, 0);
            b.dcost = atof(argv[i + 3]);
            bs.push_back(b);
        }
        const double sc = split_scale(bs, W, threads, budget);
        double tot = 0;
        for (const SplitBucket& b : bs) {
            uint64_t Sd, Ss;
            plan_bucket_splits(b, W, threads, sc, &Sd, &Ss);
            tot += (double)(Sd + Ss) * b.nrows;
        }
        printf("%.17g %.17g\n", sc, tot);
        return 0;
    }
    return 2;
}
