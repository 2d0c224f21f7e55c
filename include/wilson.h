/*
 * wilson.h -- C ABI of the B200 Wilson-prime engine (libwilson.so).
 *
 * For every prime p in [pmin, pmax) the engine computes (p-1)! mod p^2 by the
 * three-class reduction of mfl0p/CLWilson and reports the Wilson quotient
 * w_p = ((p-1)! + 1)/p mod p, the results.txt lines and the checksum, bit for
 * bit as the reference does.
 *
 * Conventions: plain C types only; caller-owned host buffers; library-owned
 * device memory; every call returns 0 or a negative WL_ERR_* code (no exit()).
 * A context belongs to one GPU and one host thread at a time.
 *
 * Which reference interface each entry point replaces (paths inside the
 * reference project):
 *   wl_open / wl_close    OpenCL platform, context and queue setup and the
 *                         kernel builds (main.cpp:192-239, cl_wilson.cpp:1473-1485),
 *                         cleanup (cl_wilson.cpp:84-107)
 *   wl_search             one search run, cl_wilson() (cl_wilson.cpp:1442-1974,
 *                         declared cl_wilson.h:72): test primes, class targets,
 *                         the column sweep, iterate, getResults/processResult and
 *                         finalizeResults' checksum
 *   wl_rows               the per-prime residues the reference reads back before
 *                         finalising (getDataFromGPU, cl_wilson.cpp:320-350) plus
 *                         the per-prime quotient of processResult (691-900)
 *   wl_rows_from /        a search in pieces of columns with checkpoints (the
 *   wl_search_from        chunked main loop and resume, cl_wilson.cpp:1742-1776,
 *                         1856-1929)
 *   wl_rows_product       the fold of partial products into residues
 *                         (reduce.cl:11-44) across the column pieces of GPUs
 *   wl_batch              many ranges in one device pass (no counterpart: the
 *                         reference runs one range per process)
 *   wl_server_*           a resident serving session with continuous batching
 *                         (no counterpart: the reference is one range per process)
 *   wl_drop_columns       makes the next search sieve its columns again, as the
 *                         reference does on every run (getPrimes,
 *                         cl_wilson.cpp:1368-1397)
 *   wl_parse_uint64       the CLI number parser parse_uint64 (putil.c:34-116)
 *   wl_check_range        setupSearch's range rules (cl_wilson.cpp:1146-1181,
 *                         main.cpp:50-56)
 */
#ifndef WILSON_H
#define WILSON_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* error codes */
#define WL_OK                 0
#define WL_ERR_ARG          (-1)   /* bad argument / range rule violated */
#define WL_ERR_CUDA         (-2)   /* CUDA runtime error */
#define WL_ERR_NOPRIMES     (-3)   /* no primes in the range (cl_wilson.cpp:1532-1536) */
#define WL_ERR_UNSUPPORTED  (-4)   /* configuration not supported by this library */
#define WL_ERR_WILSON_CHECK (-5)   /* rem != 0 after the lift (cl_wilson.cpp:866-870) */
#define WL_ERR_NO_REPR      (-6)   /* a, c or u not found (cl_wilson.cpp:554-558) */
#define WL_ERR_CAPACITY     (-7)   /* caller buffer too small; *_needed tells the size */
#define WL_ERR_NOMEM        (-8)   /* device allocation failed */
#define WL_ERR_TOO_LARGE    (-9)   /* request exceeds the fixed scratch of wl_column_product_noalloc */

/* reference limits (cl_wilson.h:8, cl_wilson.cpp:1162) */
#define WL_MAXP      4611686018427387903ULL   /* (2^64-1)/4 */
#define WL_MAX_WIDTH 10000000ULL

typedef struct wl_ctx wl_ctx;

/* one results.txt line: value 0 = Wilson prime, else Near-Wilson +-value */
typedef struct {
    uint64_t p;
    int32_t value;
    uint32_t pad;
} wl_result;

/* per-test-prime output */
typedef struct {
    uint64_t p;
    uint64_t s0, s1;    /* T_p! mod p^2 = s0 + p*s1, T_p = (p-1)/6, /4 or /2;
                           capped runs: the partial product over q < q_cap */
    uint64_t rem, quot; /* ((p-1)! + 1) mod p^2 = rem + p*quot (full runs) */
    uint32_t type;      /* 0: p = 1 mod 3, 1: p = 5 mod 12, 2: p = 11 mod 12 */
    uint32_t status;    /* 0 ok, 1 rem != 0, 2 no representation */
} wl_row;

typedef struct {
    uint64_t pmin, pmax;
} wl_range;

typedef struct {
    uint64_t tested;        /* test primes in the range */
    uint64_t checksum;      /* full: sum p + rem + quot; capped: sum p + s0 + s1 (mod 2^64) */
    uint64_t targets[3];    /* class targets (0 if the class is empty) */
    uint32_t results;       /* result lines */
    uint32_t status;        /* 0 ok, else the first nonzero row status */
} wl_range_result;

typedef struct {
    uint64_t tested;            /* test primes */
    uint64_t per_class[3];      /* test primes per class */
    uint64_t targets[3];        /* class targets of the (first) range */
    uint64_t pi_maxtarget;      /* sieving primes <= the largest class target (first range) */
    uint64_t cells;             /* column multiplications: sum over rows of its columns */
    uint64_t tail_steps;        /* consecutive-integer multiplications */
    uint64_t checksum;          /* as wl_range_result.checksum, summed over ranges */
    uint32_t results;           /* result lines */
    uint32_t kernel_launches;   /* CUDA kernels launched by the call */
    double ms_device;           /* device time of the whole call (CUDA events) */
    double ms_primes;           /* test-prime generation */
    double ms_sieve;            /* column sieve (0 when the cache already covered it) */
    double ms_sweep;            /* column sweep kernels */
    double ms_iterate;          /* consecutive-integer tail */
    double ms_finish;           /* combine + lift */
    uint64_t h2d_bytes, d2h_bytes;
    double ms_big;              /* columns above 2^32 (window sieve + sweep + merge), own stream */
    uint64_t sieve_integers;    /* integers the column sieve covered (0 when the cache already held them) */
    uint64_t sieve_bytes;       /* its device-memory traffic: bitmap written and read back, counts,
                                   offsets, the column table written (4 B per prime) */
    uint64_t dense_column_cells; /* cells of the dense-regime sweep for the exponent's high part,
                                    one per (row, column); included in `cells` */
    uint64_t dense_window_cells; /* its further cells, one per nonzero window digit of the
                                    exponent's low part, summed over rows */
    uint64_t dense_products;    /* full Montgomery products it executed, summed over rows (about
                                   L cells each) */
    uint64_t graph_nodes;       /* nodes of the CUDA graph that carried the call's sweep, merges,
                                   tail and lift (wl_batch); 0 when they were launched one by one */
    double ms_graph_build;      /* host time to end that graph's capture and instantiate it */
} wl_stats;

/* Open a context on CUDA device `device`. */
int wl_open(int device, wl_ctx **out);
void wl_close(wl_ctx *ctx);
const char *wl_strerror(int code);
/* The CUDA stream all work of the context is issued on (a cudaStream_t). */
void *wl_stream(wl_ctx *ctx);

/* Range rules of the reference: 5 <= pmin < pmax <= WL_MAXP, pmax - pmin <= WL_MAX_WIDTH. */
int wl_check_range(uint64_t pmin, uint64_t pmax);

/* Search [pmin, pmax).  q_cap = 0: full search.  q_cap > 0: capped sweep over
 * sieving primes q < q_cap only (partial products; no tail, no lift, no
 * result lines).  Result lines go to `results` in ascending p (up to `cap`;
 * WL_ERR_CAPACITY when more exist, with stats->results set). */
int wl_search(wl_ctx *ctx, uint64_t pmin, uint64_t pmax, uint64_t q_cap,
              wl_result *results, size_t cap, wl_stats *stats);

/* As wl_search, returning every test prime's row (ascending p). */
int wl_rows(wl_ctx *ctx, uint64_t pmin, uint64_t pmax, uint64_t q_cap,
            wl_row *rows, size_t cap, size_t *nrows, wl_stats *stats);

/* Many ranges in one pass; out[i] describes ranges[i].  Result lines of all
 * ranges are appended to `results` (ascending p within each range, ranges in
 * order) when results != NULL. */
int wl_batch(wl_ctx *ctx, const wl_range *ranges, size_t n, uint64_t q_cap,
             wl_range_result *out, wl_result *results, size_t cap, size_t *nresults,
             wl_stats *stats);

/* A search in pieces (checkpoint and resume, as the reference's chunked main
 * loop, cl_wilson.cpp:1856-1929, resumed by read_state, 159-288).
 * wl_rows_from: as wl_rows with the column product restricted to the sieving
 * primes q in [q_lo, q_cap) (each class still stops at its target), times the
 * rows' running products over the primes below q_lo given in `init`: row i
 * (ascending p, as wl_rows returns them) starts from init[2i] + p*init[2i+1]
 * (both digits < p; init = NULL: 1).  q_cap = 0 runs to the class targets and
 * adds the tail and the lift, as wl_rows.  The returned (s0, s1) of a capped
 * call are the next call's init.  wl_search_from: the last piece, returning
 * result lines and checksum as wl_search. */
int wl_rows_from(wl_ctx *ctx, uint64_t pmin, uint64_t pmax, uint64_t q_lo, uint64_t q_cap, const uint64_t *init,
                 wl_row *rows, size_t cap, size_t *nrows, wl_stats *stats);
int wl_search_from(wl_ctx *ctx, uint64_t pmin, uint64_t pmax, uint64_t q_lo, const uint64_t *init,
                   wl_result *results, size_t cap, wl_stats *stats);

/* Row-wise product of partial column products, for a column interval split
 * between GPUs (each piece from wl_rows_from with init = NULL; the product is
 * the init of the finishing wl_search_from).  The reference has one device and
 * folds work-group partials into a residue with reduce.cl:11-44; this is that
 * fold across pieces.  parts holds nparts arrays of n rows:
 * parts[k*2n + 2i] + p[i]*parts[k*2n + 2i + 1] is row i's k-th partial (digits
 * < p[i], p[i] odd in [5, 2^62)); out[2i] + p[i]*out[2i+1] receives the product
 * mod p[i]^2.  Computed on the GPU; WL_ERR_ARG for a bad p or digit. */
int wl_rows_product(wl_ctx *ctx, size_t n, const uint64_t *p, size_t nparts, const uint64_t *parts,
                    uint64_t *out);

/* Forget the resident column table; the next call sieves it again. */
void wl_drop_columns(wl_ctx *ctx);

/* Column product of one class without any device allocation.
 *
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory while they run -- hosts that reserve all device memory in their own
 * pool at start-up and forbid cudaMalloc afterwards (cudaMalloc and cudaFree
 * synchronise the device and fail once the pool holds the memory), or paths
 * that must not take the driver's allocation lock.
 *
 * For each row i, with p = primes[i]:
 *     s0s1[2i] + p * s0s1[2i+1] = prod_{j < ncols} cols[j]^{v(cols[j], T!)}  mod p^2
 * where v(q, T!) is the exponent of q in T! -- the same partial product that
 * wl_rows() returns for one class with q_cap (cols = the primes q < q_cap, q <= T,
 * ascending; T = that class's target).
 *   primes  device array of nrows odd primes, 5 <= p < p_bound <= WL_MAXP + 1
 *   cols    device array of ncols ascending primes, each <= T and < 2^32
 *   s0s1    device array of 2 * nrows uint64_t (output)
 *   stream  the cudaStream_t to run on (NULL: the legacy default stream); the
 *           call returns once the work is queued, like a kernel launch
 * The inputs are checked on the device: a row whose prime is even, below 5
 * or not below p_bound gets s0 = s1 = UINT64_MAX (a real digit is < p), and
 * so does every row when a column is below 2, above T or not above the one
 * before it.  A CUDA error already pending in the calling thread is returned
 * as WL_ERR_CUDA before anything is launched (and left pending); a launch
 * that fails returns WL_ERR_CUDA at once.
 * All intermediate data lives in one fixed array of WL_NOALLOC_SCRATCH_BYTES
 * (5 MiB) of device memory that the CUDA runtime places on every GPU that
 * loads the library and keeps until the process exits.  Limits: nrows <=
 * WL_NOALLOC_MAX_ROWS and (column splits x nrows) <= WL_NOALLOC_MAX_PARTIALS;
 * larger requests return WL_ERR_TOO_LARGE.  The call uses the current CUDA
 * device; its first call on a device resolves the array's device address
 * (cudaGetSymbolAddress, once per device under a lock, so first calls from
 * several host threads are safe), so make that first call before any stream
 * capture.  Calls share the array; each call clears the one word that must
 * start at zero and overwrites everything else it reads before reading it; calls that overlap on the GPU
 * (different streams, or another host thread) race on it and must be
 * serialised by the caller. */
#define WL_NOALLOC_MAX_ROWS      4096u
#define WL_NOALLOC_MAX_PARTIALS  (1u << 18)
#define WL_NOALLOC_SCRATCH_BYTES (5u << 20)
int wl_column_product_noalloc(const uint64_t *primes, uint32_t nrows, uint64_t p_bound, uint64_t T,
                              const uint32_t *cols, uint32_t ncols, uint64_t *s0s1, void *stream);

/* ---- Kernel tuning ----------------------------------------------------------
 * No counterpart in the reference.  The sweep kernels have variants whose
 * speed depends on the GPU and the workload; a context keeps one choice per
 * limb width L (index L - 2: p < 2^31, < 2^47, < 2^62). */
#define WL_DENSE_SORTED_W3 0   /* digit-sorted windows, 3-bit, 3 CTAs/SM */
#define WL_DENSE_SORTED_W4 1   /* digit-sorted windows, 4-bit, 2 CTAs/SM */
#define WL_DENSE_SWITCH_W3 2   /* per-column bucket switch, 3-bit, 3 CTAs/SM */
#define WL_DENSE_SWITCH_W4 3   /* per-column bucket switch, 4-bit, 2 CTAs/SM */
#define WL_DENSE_SMEM_W3   4   /* digit-sorted, buckets in shared memory, 3-bit, 4 CTAs/SM (default) */
#define WL_DENSE_SMEM_W4   5   /* digit-sorted, buckets in shared memory, 4-bit, 2 CTAs/SM */
#define WL_DENSE_SORTED_W3_2CTA 6   /* digit-sorted windows, 3-bit, 2 CTAs/SM (no register spills) */
typedef struct {
    int32_t sparse_variant[3];   /* cell formulation of the prefix-fold sweep: 0 carry chain, 1 wide products,
                                    2 high half first, 3 wide products with each thread's last row on the carry chain */
    int32_t sparse_rpt[3];       /* rows per thread of the prefix-fold sweep for buckets of >= 512 rows (1, 2;
                                    4 from 1,024 rows) */
    int32_t dense_kernel[3];     /* WL_DENSE_* */
    int32_t dense_hstep[3];      /* columns per change of the exponent's high part in the dense sweep */
    int32_t merge_cta_min;       /* split count from which partials merge with one CTA per row (tree fan-in 256) */
    int32_t pad;
    double ms[3];                /* after wl_autotune: sweep time of the tuning sample per L (best choice) */
} wl_tuning;

int wl_get_tuning(wl_ctx *ctx, wl_tuning *out);
int wl_set_tuning(wl_ctx *ctx, const wl_tuning *t);
/* Time the variants and keep the fastest in the context, by coordinate
 * descent (prefix-fold sweep, dense sweep, merge fan-in; a candidate must be
 * more than 2% faster to replace the current choice).  ranges/n/q_cap: the
 * workload to tune on (one choice for all its limb widths); n = 0: built-in
 * samples, one per L with bit (L - 2) set in limbs_mask (0: all), a few
 * seconds each.  Every candidate must produce the same rows; a mismatch
 * returns WL_ERR_CUDA.  The choices are also written to *out when out != NULL. */
int wl_autotune(wl_ctx *ctx, const wl_range *ranges, size_t n, uint64_t q_cap, uint32_t limbs_mask,
                wl_tuning *out);

/* ---- Serving: a resident session with continuous batching ------------------
 *
 * No counterpart in the reference.  A server owns one GPU and a scheduler
 * thread.  Submitted ranges wait in a FIFO queue until the row pool (a device
 * memory budget for resident test primes: moduli, running partial products,
 * outputs) and the bucket table have room; then they are admitted between
 * scheduler steps.  Each step advances every admitted (range, class) bucket by
 * one chunk of its columns -- all buckets in the same sweep launches -- and
 * folds the chunk's products into the bucket rows' resident partial products.
 * Requests that finish their columns are completed (class lift, quotient,
 * result lines, checksum) and their rows freed for the next ones, so requests
 * that arrive while others run share the GPU with them.  Each request's
 * results are bit-identical to wl_search / wl_rows on the same range.
 *
 * Columns above 2^32 (full searches with p above about 8.5e9, or q_cap above
 * 2^32) are sieved in chunks of the number line inside the step loop, each
 * chunk sized to the bucket's share of the step.  A request larger than the
 * whole pool fails with WL_ERR_NOMEM.  All functions are thread-safe. */
typedef struct wl_server wl_server;

#define WL_SHARES_LEAST_WORK 0   /* shares weighted by 1/sqrt(work left): small requests first, large ones keep moving */
#define WL_SHARES_EQUAL      1   /* every active (request, class) bucket gets an equal share */
typedef struct {
    int device;
    uint32_t shares;       /* WL_SHARES_*: how a step's cell budget is split between requests */
    uint64_t pool_bytes;   /* device memory for resident rows (0: 1 GiB); WL_SERVER_ROW_BYTES each */
    uint64_t step_cells;   /* column-cell budget of one scheduler step (0: 2^32) */
    const wl_tuning *tuning;   /* kernel choices (NULL: the defaults) */
} wl_server_opts;

#define WL_SERVER_ROW_BYTES 160u

#define WL_REQ_QUEUED    0
#define WL_REQ_ACTIVE    1
#define WL_REQ_DONE      2
#define WL_REQ_CANCELLED 3
#define WL_REQ_FAILED    4

typedef struct {
    uint64_t id;
    int32_t state;         /* WL_REQ_* */
    int32_t rc;            /* 0, or the WL_ERR_* code of a failed request */
    uint64_t tested;       /* test primes (rows) */
    uint64_t checksum;     /* full: sum(p + rem + quot); capped: sum(p + s0 + s1), mod 2^64 */
    uint64_t targets[3];   /* class targets */
    uint64_t cells;        /* column cells + tail steps of the request */
    uint32_t results;      /* result lines (full searches) */
    uint32_t pad;
    double ms_queued;      /* submit -> admission */
    double ms_latency;     /* submit -> completion */
} wl_request_info;

typedef struct {
    uint64_t steps;        /* scheduler steps run */
    uint64_t admitted, completed, failed, cancelled;
    uint64_t rows_done;    /* rows of completed requests */
    uint64_t cells;        /* cells of completed requests */
    uint64_t launches;     /* kernel launches */
    double ms_steps;       /* device time of the steps (CUDA events) */
    double ms_admit;       /* device time of admissions */
    uint32_t peak_rows;    /* largest number of resident rows */
    uint32_t peak_active;  /* largest number of admitted requests at once */
    double ms_wall_steps;  /* scheduler wall time planning and queueing steps (overlaps the previous step) */
    double ms_wall_admit;  /* scheduler wall time in admissions (the pipeline drained first) */
    double ms_wall_finish; /* scheduler wall time waiting for steps to end and completing requests */
} wl_server_stats;

int wl_server_open(const wl_server_opts *opts, wl_server **out);
/* Queue [pmin, pmax) (q_cap as in wl_search); *id identifies the request. */
int wl_server_submit(wl_server *srv, uint64_t pmin, uint64_t pmax, uint64_t q_cap, uint64_t *id);
/* 0 if the request has ended (done, failed or cancelled), 1 if not; fills *info. */
int wl_server_poll(wl_server *srv, uint64_t id, wl_request_info *info);
/* As poll, waiting up to timeout_ms (< 0: no limit) for the request to end. */
int wl_server_wait(wl_server *srv, uint64_t id, wl_request_info *info, double timeout_ms);
/* Result lines of a finished full search, ascending p (WL_ERR_CAPACITY if cap is short). */
int wl_server_results(wl_server *srv, uint64_t id, wl_result *results, size_t cap, size_t *n);
/* Rows of a finished request, ascending p, as wl_rows. */
int wl_server_rows(wl_server *srv, uint64_t id, wl_row *rows, size_t cap, size_t *n);
/* Cancel a queued or running request; it ends in WL_REQ_CANCELLED. */
int wl_server_cancel(wl_server *srv, uint64_t id);
/* Forget an ended request (its id becomes invalid). */
int wl_server_release(wl_server *srv, uint64_t id);
int wl_server_stats_get(wl_server *srv, wl_server_stats *stats);
/* Stop the scheduler (running requests are abandoned) and free the server. */
void wl_server_close(wl_server *srv);

/* parse_uint64 of the reference CLI: returns 0, -1 (cannot parse) or -2 (out of range). */
int wl_parse_uint64(uint64_t *result, const char *str, uint64_t lo, uint64_t hi);

#ifdef __cplusplus
}
#endif

#endif /* WILSON_H */
