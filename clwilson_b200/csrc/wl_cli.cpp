// wl_cli.cpp -- `clwilson`, the command-line program of the B200 Wilson-prime engine.
//
// Same surface as the reference program (main.cpp:27-159, cl_wilson.cpp:1146-1181,
// 1588-1595, 1959-1967, 1998-2139):
//   -p #   first prime to test      -P #   end of the range [p, P), P - p <= 1e7
//   -s     self test (the reference's seven known-answer ranges)
//   -r     verify results with |w_p/p| < 1/50000 against goodWilsonResults.txt (P <= 2e13)
//   -d #, --device #  accepted and ignored, as in the reference; the GPU comes from
//          init_data.xml (<gpu_device_num>) or defaults to 0
//   -h     help
// Writes results.txt (truncated at the start, one line per result, then the checksum
// line) exactly as the reference does.  Long searches run in pieces of columns and
// checkpoint every minute to stateA.ckp / stateB.ckp in the reference's format
// (cl_wilson.cpp:110-288), so a search resumes from its last checkpoint -- also one
// written by the reference program while its columns were below 2^32 (past
// that point the two programs' running products differ; see wl_ckpt.h).  All arithmetic runs in libwilson.so.
#include <getopt.h>
#include <algorithm>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "wilson.h"
#include "wl_ckpt.h"

static const char* RESULT_FILENAME = "results.txt";
static const char* GOOD_RES_FILENAME = "goodWilsonResults.txt";


struct Opts {
    uint64_t pmin = 0, pmax = 0;
    bool test = false, result_test = false;
};

static void help() {
    printf("Welcome to clwilson, a B200 CUDA program to search for Wilson Primes\n");
    printf("Program usage:\n");
    printf("-p #\tStarting prime to search p\n");
    printf("-P #\tEnd prime prime to search P, range [-p, -P) exclusive, 5 <= -p <= p < -P <= %" PRIu64 "\n",
           (uint64_t)WL_MAXP);
    printf("\tRequired range is <= 10e6\n");
    printf("-s \tPerform self test to verify proper operation of the program with the current GPU.\n");
    printf("-r \tVerify all results (up to 2e13) where |w_p/p| < 1/50000 with known good file %s\n", GOOD_RES_FILENAME);
    printf("\t-s and -r are for use in standalone testing.\n");
    printf("-h\tPrint this help\n");
    exit(EXIT_FAILURE);
}

static int gpu_from_init_data() {
    FILE* f = fopen("init_data.xml", "r");
    if (!f) return 0;
    char buf[4096];
    size_t n = fread(buf, 1, sizeof(buf) - 1, f);
    fclose(f);
    buf[n] = 0;
    const char* t = strstr(buf, "<gpu_device_num>");
    return t ? atoi(t + strlen("<gpu_device_num>")) : 0;
}

static void fail(const char* msg) {
    fprintf(stderr, "%s", msg);
    printf("%s", msg);
    exit(EXIT_FAILURE);
}

// setupSearch (cl_wilson.cpp:1146-1181)
static void setup_search(const Opts& o) {
    if (o.pmin == 0 || o.pmax == 0) {
        printf("-p and -P arguments are required\nuse -h for help\n");
        fprintf(stderr, "-p and -P arguments are required\n");
        exit(EXIT_FAILURE);
    }
    if (o.pmin > o.pmax) {
        printf("pmin <= pmax is required\nuse -h for help\n");
        fprintf(stderr, "pmin <= pmax is required\n");
        exit(EXIT_FAILURE);
    }
    if (o.pmax > o.pmin + 10000000) {
        printf("range <= 10000000 is required\nuse -h for help\n");
        fprintf(stderr, "range <= 10000000 is required\n");
        exit(EXIT_FAILURE);
    }
    if (o.result_test && o.pmax > 20000000000000ULL) {
        printf("pmax <= 2e13 is required when verifying results.\nuse -h for help\n");
        fprintf(stderr, "pmax < 2e13 is required when verifying results.\n");
        exit(EXIT_FAILURE);
    }
    fprintf(stderr, "Starting search at p: %" PRIu64 "\nStopping search at P: %" PRIu64 "\n", o.pmin, o.pmax);
    printf("Starting search at p: %" PRIu64 "\nStopping search at P: %" PRIu64 "\n", o.pmin, o.pmax);
}

struct GoodResult { uint64_t p; int32_t v; };

// readGoodResultFile (cl_wilson.cpp:936-1014)
static std::vector<GoodResult> read_good_results(uint64_t pmin, uint64_t pmax) {
    FILE* f = fopen(GOOD_RES_FILENAME, "r");
    if (!f) {
        fprintf(stderr, "Cannot open %s !!!\n", GOOD_RES_FILENAME);
        printf("Cannot open %s !!!\n", GOOD_RES_FILENAME);
        exit(EXIT_FAILURE);
    }
    char line[256];
    uint64_t sum = 0;
    std::vector<GoodResult> out;
    while (fgets(line, sizeof(line), f)) {
        uint64_t p;
        int32_t v;
        if (sscanf(line, "%" SCNu64 " %" SCNd32, &p, &v) != 2) {
            fclose(f);
            fail("Error reading goodWilsonResults.txt !!!\n");
        }
        sum += p + v;
        if (p >= pmin && p < pmax) out.push_back({ p, v });
    }
    fclose(f);
    if (sum != 0x6659912234F44428ULL) fail("Checksum error in goodWilsonResults.txt !!!\n");
    printf("Read %zu good results |w_p/p| < 1/50000 for search range from %s\n", out.size(), GOOD_RES_FILENAME);
    return out;
}

struct RunResult {
    uint64_t checksum = 0, pi_maxtarget = 0;
    std::vector<wl_result> results;
    int rc = 0;
};

// The search from column q_lo on (init: the rows' running products below q_lo,
// two digits per row; NULL with q_lo = 2 for a search from the start).
static RunResult run_search(wl_ctx* ctx, const Opts& o, bool verbose, uint64_t q_lo = 2,
                            const uint64_t* init = nullptr) {
    RunResult rr;
    // the whole row set (needed for -r) or just the result lines
    wl_stats st;
    std::vector<wl_row> rows;
    if (o.result_test) {
        size_t cap = (o.pmax - o.pmin) / 2 + 2, n = 0;
        rows.resize(cap);
        rr.rc = wl_rows_from(ctx, o.pmin, o.pmax, q_lo, 0, init, rows.data(), cap, &n, &st);
        rows.resize(n);
        for (const wl_row& r : rows) {
            const uint64_t negq = r.p - r.quot, sm = r.quot <= negq ? r.quot : negq;
            if (r.quot == 0) rr.results.push_back({ r.p, 0, 0 });
            else if (sm < 1000) rr.results.push_back({ r.p, sm == r.quot ? (int32_t)r.quot : -(int32_t)negq, 0 });
        }
    } else {
        std::vector<wl_result> res(1 << 16);
        rr.rc = wl_search_from(ctx, o.pmin, o.pmax, q_lo, init, res.data(), res.size(), &st);
        if (rr.rc == WL_ERR_CAPACITY) {
            res.resize(st.results);
            rr.rc = wl_search_from(ctx, o.pmin, o.pmax, q_lo, init, res.data(), res.size(), &st);
        }
        res.resize(st.results);
        rr.results = res;
    }
    if (rr.rc) return rr;
    rr.checksum = st.checksum;
    rr.pi_maxtarget = st.pi_maxtarget;
    if (verbose) {
        printf("Testing %" PRIu64 " primes.  There are %" PRIu64 " type 0 (1 mod 3) primes, %" PRIu64
               " type 1 (5 mod 12) primes, and %" PRIu64 " type 2 (11 mod 12) primes\n",
               st.tested, st.per_class[0], st.per_class[1], st.per_class[2]);
        printf("Factorial targets are %" PRIu64 ", %" PRIu64 ", %" PRIu64 "\n", st.targets[0], st.targets[1],
               st.targets[2]);
        printf("     Power limits are %" PRIu64 ", %" PRIu64 ", %" PRIu64 "\n", st.targets[0] / 2, st.targets[1] / 2,
               st.targets[2] / 2);
    }
    if (o.result_test) {
        std::vector<GoodResult> good = read_good_results(o.pmin, o.pmax);
        std::vector<bool> used(good.size(), false);
        size_t matched = 0;
        for (const wl_row& r : rows) {
            const uint64_t negq = r.p - r.quot, sm = r.quot <= negq ? r.quot : negq;
            if ((double)((long double)sm / (long double)r.p) >= 1.0 / 50000.0) continue;
            const int32_t dq = sm == r.quot ? (int32_t)r.quot : -(int32_t)negq;
            bool ok = false;
            for (size_t j = 0; j < good.size(); ++j) {
                if (good[j].p != r.p) continue;
                if (good[j].v != dq) {
                    fprintf(stderr, "error: result check failed! p: %" PRIu64 " %d, result file is %d\n", r.p, dq, good[j].v);
                    printf("error: result check failed! p: %" PRIu64 " %d, result file is %d\n", r.p, dq, good[j].v);
                    exit(EXIT_FAILURE);
                }
                printf("p: %" PRIu64 " has matching result %+d\n", r.p, dq);
                used[j] = true;
                ++matched;
                ok = true;
                break;
            }
            if (!ok) {
                fprintf(stderr, "error: result check failed! p: %" PRIu64 " is not in result file!\n", r.p);
                printf("error: result check failed! p: %" PRIu64 " is not in result file!\n", r.p);
                exit(EXIT_FAILURE);
            }
        }
        if (matched != good.size()) {
            for (size_t j = 0; j < good.size(); ++j)
                if (!used[j]) printf("error: result check failed! p: %" PRIu64 " was not found in results!\n", good[j].p);
            exit(EXIT_FAILURE);
        }
        printf("All results matched result file!\n");
        fprintf(stderr, "All results matched result file!\n");
    }
    return rr;
}

// writeResult + finalizeResults (cl_wilson.cpp:657-688, 1093-1143)
static void write_results_file(const RunResult& rr) {
    FILE* f = fopen(RESULT_FILENAME, "w");
    if (!f) fail("Cannot open results.txt !!!\n");
    for (const wl_result& r : rr.results) {
        if (r.value == 0) fprintf(f, "%" PRIu64 " is a Wilson prime\n", r.p);
        else fprintf(f, "%" PRIu64 " is a Near-Wilson prime %+d\n", r.p, r.value);
    }
    if (rr.results.empty()) fprintf(f, "no results\n%016" PRIX64 "\n", rr.checksum);
    else fprintf(f, "%016" PRIX64 "\n", rr.checksum);
    if (fclose(f) != 0) fail("Cannot close results.txt !!!\n");
}

static double prime_count_estimate(double x) { return x < 17 ? 7 : x / std::log(x); }

static int search(wl_ctx* ctx, const Opts& o) {
    setup_search(o);
    time_t t0 = time(nullptr);
    // the test primes and class targets: the rows with no columns multiplied in
    size_t cap = (o.pmax - o.pmin) / 2 + 2, n = 0;
    std::vector<wl_row> rows(cap);
    wl_stats st0;
    int rc = wl_rows(ctx, o.pmin, o.pmax, 2, rows.data(), cap, &n, &st0);
    if (rc) {
        fprintf(stderr, "error: %s\n", wl_strerror(rc));
        printf("error: %s\n", wl_strerror(rc));
        return EXIT_FAILURE;
    }
    rows.resize(n);
    const uint64_t maxtarget = std::max(st0.targets[0], std::max(st0.targets[1], st0.targets[2]));
    WorkStatus ws;
    memset(&ws, 0, sizeof(ws));
    ws.pmin = o.pmin;
    ws.pmax = o.pmax;
    ws.currp = 2;
    ws.tpcount = (uint32_t)n;
    std::vector<uint64_t> res(2 * n), ref(2 * n);
    for (size_t i = 0; i < n; ++i) { res[2 * i] = 1; res[2 * i + 1] = 0; }
    bool write_a_next = true;
    const int rsr = read_state(write_a_next, ws, ref);
    if (rsr == 3) return EXIT_FAILURE;   // a reference checkpoint past 2^32 (message printed)
    if (rsr == 2) {
        printf("Workunit complete.\n");
        fprintf(stderr, "Workunit complete.\n");
        return EXIT_SUCCESS;
    }
    if (rsr == 1) {
        printf("Resuming search from checkpoint. Current P: %" PRIu64 "\n", ws.currp);
        fprintf(stderr, "Resuming search from checkpoint. Current P: %" PRIu64 "\n", ws.currp);
        for (size_t i = 0; i < n; ++i) from_reference(rows[i].p, ref[2 * i], ref[2 * i + 1], &res[2 * i], &res[2 * i + 1]);
    } else {
        FILE* f = fopen(RESULT_FILENAME, "w");
        if (!f) fail("Cannot open results.txt !!!\n");
        fclose(f);
        ws.trickle = (uint64_t)time(nullptr);
    }

    // pieces of about 10 s of work while more than about 20 s remain, a
    // checkpoint at most once a minute, then the last piece (the remaining
    // columns, the tail and the lift).  For tests: WL_CKPT_PIECE fixes the
    // piece width (integers), WL_CKPT_INTERVAL the seconds between
    // checkpoints, and WL_CKPT_STOP=k ends the program (exit status 3) after
    // k pieces and a checkpoint, as an interrupted run would.
    const uint64_t fixed_piece = getenv("WL_CKPT_PIECE") ? strtoull(getenv("WL_CKPT_PIECE"), nullptr, 0) : 0;
    const int interval = getenv("WL_CKPT_INTERVAL") ? atoi(getenv("WL_CKPT_INTERVAL")) : 60;
    const int stop_after = getenv("WL_CKPT_STOP") ? atoi(getenv("WL_CKPT_STOP")) : 0;
    double rate = 1.0e11;   // column cells per second, refined by measurement
    time_t ckpt_last = time(nullptr);
    bool chunked = false;
    int pieces = 0;
    while (ws.currp <= maxtarget) {
        uint64_t stop;
        if (fixed_piece) {
            if (maxtarget + 1 - ws.currp <= fixed_piece) break;
            stop = ws.currp + fixed_piece;
        } else {
            const double left =
                (double)n * (prime_count_estimate((double)maxtarget) - prime_count_estimate((double)ws.currp));
            if (left <= rate * 20.0) break;
            const double want = rate * 10.0 / (double)n;   // primes per piece
            const double lnx = std::log(std::max((double)ws.currp, 17.0));
            stop = ws.currp + (uint64_t)std::max(1.0e6, want * lnx);
            if (stop > maxtarget) stop = maxtarget + 1;
        }
        const time_t tc = time(nullptr);
        wl_stats st;
        size_t got = 0;
        std::vector<wl_row> part(n);
        rc = wl_rows_from(ctx, o.pmin, o.pmax, ws.currp, stop, res.data(), part.data(), n, &got, &st);
        if (rc || got != n) {
            fprintf(stderr, "error: %s\n", wl_strerror(rc ? rc : WL_ERR_ARG));
            printf("error: %s\n", wl_strerror(rc ? rc : WL_ERR_ARG));
            return EXIT_FAILURE;
        }
        for (size_t i = 0; i < n; ++i) { res[2 * i] = part[i].s0; res[2 * i + 1] = part[i].s1; }
        const double secs = st.ms_device / 1e3;
        if (secs > 0.5 && st.cells) rate = std::min(rate * 4.0, (double)st.cells / secs);
        ws.currp = stop;
        ws.totalcount = st.pi_maxtarget;
        chunked = true;
        ++pieces;
        const bool stopping = stop_after > 0 && pieces >= stop_after;
        if ((int)(time(nullptr) - ckpt_last) >= interval || stopping) {
            ckpt_last = time(nullptr);
            for (size_t i = 0; i < n; ++i) to_reference(part[i].p, res[2 * i], res[2 * i + 1], &ref[2 * i], &ref[2 * i + 1]);
            write_state(write_a_next, ws, ref);
            printf("Checkpoint, Current P: %" PRIu64 "\n", ws.currp);
        }
        if (stopping) return 3;
    }
    RunResult rr = run_search(ctx, o, true, ws.currp, (chunked || rsr == 1) ? res.data() : nullptr);
    if (rr.rc) {
        fprintf(stderr, "error: %s\n", wl_strerror(rr.rc));
        printf("error: %s\n", wl_strerror(rr.rc));
        return EXIT_FAILURE;
    }
    // result lines go to stdout too, except when verifying (cl_wilson.cpp:876-891)
    for (const wl_result& r : rr.results) {
        if (o.result_test) break;
        if (r.value == 0) printf("%" PRIu64 " is a Wilson prime\n", r.p);
        else printf("%" PRIu64 " is a Near-Wilson prime %+d\n", r.p, r.value);
    }
    write_results_file(rr);
    // the finished workunit (read_state reports it complete)
    ws.done = 1;
    ws.currp = maxtarget + 1;
    for (size_t i = 0; i < n; ++i) to_reference(rows[i].p, res[2 * i], res[2 * i + 1], &ref[2 * i], &ref[2 * i + 1]);
    write_state(write_a_next, ws, ref);
    fprintf(stderr, "Search complete. Results: %zu, total power table primes generated %" PRIu64 ", removed 0 PRPs\n",
            rr.results.size(), rr.pi_maxtarget);
    printf("Search finished in %d sec.\n", (int)(time(nullptr) - t0));
    printf("results %zu, total power table primes generated %" PRIu64 ", checksum %016" PRIX64 ", removed 0 PRPs\n",
           rr.results.size(), rr.pi_maxtarget, rr.checksum);
    return EXIT_SUCCESS;
}

// run_test (cl_wilson.cpp:1998-2139): the seven known-answer ranges
static int self_test(wl_ctx* ctx) {
    struct Case { uint64_t pmin, pmax; uint32_t count; uint64_t checksum, pi; uint64_t prime; int32_t value; const char* note; };
    const Case cases[7] = {
        { 1239053554603ULL, 1239053554604ULL, 1, 0x00000240FAB1A752ULL, 8257082014ULL, 1239053554603ULL, -4, "1239053554603 is a type 0 prime" },
        { 1108967825921ULL, 1108967825922ULL, 1, 0x0000010233A2220DULL, 10956003002ULL, 1108967825921ULL, 12, "1108967825921 is a type 1 prime" },
        { 5609877309359ULL, 5609877309360ULL, 1, 0x00000A344D7D0F58ULL, 101542897873ULL, 5609877309359ULL, -6, "5609877309359 is a type 2 prime" },
        { 16556218163369ULL, 16556218163370ULL, 1, 0x00000F0ECB80A0ABULL, 147755473426ULL, 16556218163369ULL, 2, "16556218163369 is a type 1 prime" },
        { 200, 564, 57, 0x00000000000080A3ULL, 30, 563, 0, "Testing small iterations with Wilson prime 563" },
        { 86000000, 87467200, 1, 0x0000097C61AB0943ULL, 2604536, 87467099, -2, "Testing large iterations with type 2 prime 87467099" },
        { 17524177394450ULL, 17524177394618ULL, 1, 0x00005B54B4CBBC47ULL, 304620766446ULL, 17524177394617ULL, 256, "17524177394617 is a type 0 prime" },
    };
    printf("Beginning self test of 7 ranges.\n\n");
    time_t t0 = time(nullptr);
    int good = 0;
    for (int i = 0; i < 7; ++i) {
        const Case& c = cases[i];
        printf("%s\n", c.note);
        Opts o;
        o.pmin = c.pmin;
        o.pmax = c.pmax;
        RunResult rr = run_search(ctx, o, false);
        bool ok = rr.rc == 0 && rr.results.size() == c.count && rr.checksum == c.checksum && rr.pi_maxtarget == c.pi &&
                  !rr.results.empty() && rr.results.back().p == c.prime && rr.results.back().value == c.value;
        if (rr.rc) printf("  (%s)\n", wl_strerror(rr.rc));
        printf("test case %d %s.\n\n", i + 1, ok ? "passed" : "failed");
        fprintf(stderr, "test case %d %s.\n", i + 1, ok ? "passed" : "failed");
        good += ok;
    }
    if (good == 7) {
        printf("All test cases completed successfully!\n");
        fprintf(stderr, "All test cases completed successfully!\n");
    } else {
        printf("Self test FAILED!\n");
        fprintf(stderr, "Self test FAILED!\n");
    }
    printf("Elapsed time: %d sec.\n", (int)(time(nullptr) - t0));
    return good == 7 ? EXIT_SUCCESS : EXIT_FAILURE;
}

int main(int argc, char** argv) {
    Opts o;
    printf("\nclwilson (B200 CUDA engine)\n");
    fprintf(stderr, "Command line: ");
    for (int i = 0; i < argc; ++i) fprintf(stderr, "%s ", argv[i]);
    fprintf(stderr, "\n");
    static const struct option long_opts[] = { { "device", optional_argument, 0, 'd' }, { "test", no_argument, 0, 's' },
                                                { 0, 0, 0, 0 } };
    int opt, ind = -1;
    while ((opt = getopt_long(argc, argv, "p:P:srd:h", long_opts, &ind)) != -1) {
        int status = 0;
        switch (opt) {
            case 'p': status = wl_parse_uint64(&o.pmin, optarg, 5, WL_MAXP - 1); break;
            case 'P': status = wl_parse_uint64(&o.pmax, optarg, 6, WL_MAXP); break;
            case 's':
                o.test = true;
                fprintf(stderr, "Performing self test.\n");
                printf("Performing self test.\n");
                break;
            case 'r':
                o.result_test = true;
                fprintf(stderr, "Testing all results |w_p/p| < 1/50000 with known good result file %s\n", GOOD_RES_FILENAME);
                printf("Testing all results |w_p/p| < 1/50000 with known good result file %s\n", GOOD_RES_FILENAME);
                break;
            case 'd': break;
            default: help();
        }
        if (status == -1) {
            printf("%s: invalid argument -%c %s\n", argv[0], opt, optarg);
            fprintf(stderr, "%s: invalid argument -%c %s\n", argv[0], opt, optarg);
            return EXIT_FAILURE;
        }
        if (status == -2) {
            printf("%s: out of range argument -%c %s\n", argv[0], opt, optarg);
            fprintf(stderr, "%s: out of range argument -%c %s\n", argv[0], opt, optarg);
            return EXIT_FAILURE;
        }
        ind = -1;
    }
    wl_ctx* ctx = nullptr;
    int rc = wl_open(gpu_from_init_data(), &ctx);
    if (rc) {
        fprintf(stderr, "error: wl_open: %s\n", wl_strerror(rc));
        printf("error: wl_open: %s\n", wl_strerror(rc));
        return EXIT_FAILURE;
    }
    int ret = o.test ? self_test(ctx) : search(ctx, o);
    wl_close(ctx);
    return ret;
}
