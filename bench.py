#!/usr/bin/env python
"""Wilson-prime search throughput on B200 (one JSON line on rank 0).

Workloads (--workload):
  plain-small   [default] every prime p in [1e9 + r*1e6, 1e9 + (r+1)*1e6) on rank r:
                the full search of the reference's CPU-runnable configuration
                ((p-1)! mod p^2, w_p, result lines, checksum), about 48k primes per GPU.
  plain-mid     every prime in [1e13, 1e13 + 1e7): column sweep capped at q < 2^32
                (the full run is about a day on one GPU); partial products per prime.
  plain-top     every prime in [2^62-1-1e7, 2^62-1): column sweep capped at q < 2^32.
  batched       256 ranges from numpy default_rng(0), log-uniform starts in
                [1e8, 2^62-1e7) and widths in [1e3, 1e7], each width truncated to
                --max-width integers (default 2000: the whole widths are about 9e6
                rows, 1.3e14 column cells, hours per step), column sweep capped at
                q < 2^28.  One wl_batch call per step; the same ranges as a loop of
                per-range wl_search calls (the plain form) are timed beside it.
  column-shard  the plain-small range [1e9, 1e9 + 1e6), full search, with its
                column interval split over the ranks (strong scaling): each rank
                computes its piece's per-row partial products, rank 0 gathers
                them (16 B per row and rank), multiplies them row-wise on its GPU
                and finishes (tail, lift, results, checksum).
  serving       a Poisson stream of --requests range requests (default 256) from
                numpy default_rng(1): exponential inter-arrival times at --rate
                requests/s, log-uniform starts in [1e8, 2^62-1e7), widths
                log-uniform in [1e4, 1e7] truncated to --max-width; q < 2^28.
                Submitted to a serving session (wl_server_*) at their arrival
                times; a step is the whole stream.  Reports p50/p99 latency.

A step is one call of the engine's C ABI on the workload (test primes, columns,
sweep, tail, lift, results).  `value` is device time (CUDA events on the
engine's stream, L2 flushed between steps); `e2e` is host wall time around the
same C-ABI call, which includes its host<->device copies.

The default run (plain-small) adds two records to its line, so that one run
measures the whole metric: `batched` (the 256 ranges, widths truncated to
--sub-batched-width, a warm-up call on 16 of them, --sub-batched-steps timed calls,
then the plain per-range form over the same ranges) and `serving` (the first
--sub-serving-requests requests of the default_rng(1) stream at
--sub-serving-rate per second, widths truncated to 2,000).  Every line also
carries `parity_sample`: the engine's rows at the CPU baseline's sample
indices, compared with the oracle's bit for bit.

--impl reference times the reference algorithm on the host cores instead (the
CPU restatement under oracle/, all threads) on a bounded sample of the same
workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PLAIN_SMALL = (10**9, 10**6)
OPS_PER_CELL = {2: 9, 3: 13, 4: 17}   # multiply-class PTX ops of one cell step (wl_arith.cuh)
HBM_FALLBACK_GBS = 6650.0             # copy bandwidth measured earlier on this kind of GPU


def hbm_peak():
    """(GB/s, source) of the HBM roofline: the measured copy bandwidth when a
    peaks file is present, else the earlier measurement."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            v = json.load(f).get("hbm_gbs")
        if v:
            return float(v), "of measured"
    except Exception:
        pass
    return HBM_FALLBACK_GBS, "of fallback"


def work_cells(st, L):
    """Cells the sweeps executed in cell-equivalents: one per (row, column)
    of every column, the dense sweep's window cells, and its full products
    (about L cells each); and the dense share of them."""
    extra = st.dense_window_cells + L * st.dense_products
    return st.cells + extra, st.dense_column_cells + extra


def parity_sample(eng, lo, hi, q_cap, want, sel):
    """The engine's rows of [lo, hi) at rows `sel` against the oracle's
    (`want`, the rows the CPU baseline computed): every field bit for bit."""
    got, _ = eng.rows(lo, hi, q_cap=q_cap)
    fields = ("p", "s0", "s1") + (() if q_cap else ("rem", "quot", "status"))
    ok = len(got) == len(want) and all(int(got[f][i]) == int(want[f][i]) for i in sel for f in fields)
    return {"ok": bool(ok), "rows_compared": len(sel), "range": [lo, hi], "fields": list(fields)}


def limbs_for(pmax_incl: int) -> int:
    return 2 if pmax_incl < 2**31 else (3 if pmax_incl < 2**47 else 4)


def batched_ranges(seed: int = 0, n: int = 256, max_width: int = 0):
    import numpy as np
    rng = np.random.default_rng(seed)
    lo, hi = np.log(1e8), np.log(2.0**62 - 1e7)
    starts = np.exp(rng.uniform(lo, hi, n))
    widths = np.round(np.exp(rng.uniform(np.log(1e3), np.log(1e7), n)))
    out = []
    for s, w in zip(starts, widths):
        a = int(s)
        w = int(w) if not max_width else min(int(w), max_width)
        b = min(a + w, 2**62 - 1)
        out.append((max(a, 5), b))
    return out


def serving_requests(seed: int = 1, n: int = 256, rate: float = 64.0, max_width: int = 0):
    """(arrival time in s, pmin, pmax) of a Poisson stream of range requests."""
    import numpy as np
    rng = np.random.default_rng(seed)
    lo, hi = np.log(1e8), np.log(2.0**62 - 1e7)
    starts = np.exp(rng.uniform(lo, hi, n))
    widths = np.round(np.exp(rng.uniform(np.log(1e4), np.log(1e7), n)))
    gaps = rng.exponential(1.0 / rate, n)
    t = np.cumsum(gaps) - gaps[0]
    out = []
    for ti, s, w in zip(t, starts, widths):
        a = max(int(s), 5)
        w = int(w) if not max_width else min(int(w), max_width)
        out.append((float(ti), a, min(a + w, 2**62 - 1)))
    return out


def workload(name: str, rank: int, world: int, width: int = 0, qcap: int = -1, max_width: int = 2000):
    """(ranges, q_cap, description) for this rank; width/qcap override the
    configuration (for profiling small cases only)."""
    if name == "plain-small":
        w = width or PLAIN_SMALL[1]
        q = 0 if qcap < 0 else qcap
        a = PLAIN_SMALL[0] + rank * w
        return [(a, a + w)], q, f"plain-small: every prime in [{a}, {a + w}), " + ("full search" if not q else f"columns q < {q}")
    if name == "column-shard":
        a, w = PLAIN_SMALL[0], width or PLAIN_SMALL[1]
        return [(a, a + w)], 0, f"column-shard: every prime in [{a}, {a + w}), full search, columns split over {world} ranks"
    if name == "plain-mid":
        w = width or 10**7
        q = 2**32 if qcap < 0 else qcap
        a = 10**13 + rank * w
        return [(a, a + w)], q, f"plain-mid: every prime in [{a}, {a + w}), columns q < {q}"
    if name == "plain-top":
        w = width or 10**7
        q = 2**32 if qcap < 0 else qcap
        b = 2**62 - 1 - rank * w
        return [(b - w, b)], q, f"plain-top: every prime in [{b - w}, {b}), columns q < {q}"
    if name == "batched":
        rs = batched_ranges(0, max_width=max_width)
        mine = rs[rank::world]
        q = 2**28 if qcap < 0 else qcap
        return mine, q, (f"batched: {len(mine)} of 256 ranges from default_rng(0), widths truncated to "
                         f"{max_width}, columns q < {q}")
    raise SystemExit(f"unknown workload {name}")


def merge_over_ranks(dist, times, counts, device="cuda"):
    """Whole-job figures: the max over ranks of each timing and the sum over
    ranks of each work count.  Every rank takes part, in the same order; with
    no process group the values are returned as they are."""
    if dist is None:
        return list(times), list(counts)
    import torch
    t = torch.tensor(list(times), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor(list(counts), dtype=torch.float64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return t.tolist(), c.tolist()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def host_threads() -> int:
    """Host threads this process may run on.  The CPU legs pass it to the
    oracle explicitly: torchrun sets OMP_NUM_THREADS=1 in every rank, which
    would otherwise leave the reference arm on one thread at N > 1."""
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except (AttributeError, OSError):
        return max(1, os.cpu_count() or 1)


CPU_COLUMNS = ("re-sieved every step in chunks of 2^24 integers; one thread sieves and builds the next chunk's "
               "columns while the others multiply the rows by the current one")


def cpu_baseline(lo: int, hi: int, q_cap: int, budget_s: float = 20.0):
    """The oracle (reference algorithm restated in C, all host threads) on a
    bounded sample of rows of [lo, hi): primes per second."""
    import oracle
    oracle.build()
    cores = host_threads()
    n = len(oracle.list_primes(lo, hi))
    k = max(1, cores)
    while True:
        step = max(1, n // k)
        sel = list(range(0, n, step))[:k]
        t0 = time.perf_counter()
        rows, targets = oracle.search(lo, hi, qcap=q_cap, threads=cores, rows=sel)
        dt = time.perf_counter() - t0
        if dt > budget_s / 3 or k >= n or k >= 512 * cores:
            break
        k *= 2
    return {"value": len(sel) / dt, "unit": "primes/s", "cores": cores, "kind": "port",
            "sample": f"{len(sel)} of {n} primes of [{lo}, {hi}) evenly spaced, q_cap={q_cap}, "
                      f"{dt:.1f} s incl. the column sieve",
            "columns": CPU_COLUMNS}, rows, sel


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    ranges, q_cap, desc = workload(args.workload, 0, 1, args.width, args.qcap, args.max_width)
    lo, hi = max(ranges, key=lambda r: r[1] - r[0])
    import oracle
    oracle.build()
    cores = host_threads()
    n = len(oracle.list_primes(lo, hi))
    # a step: `k` evenly spaced rows of the workload with all their columns,
    # k doubled from the core count until a step takes about 5 s, so that the
    # first column chunk, sieved before any row can start, does not dominate
    k = max(1, cores)
    while True:
        sel = list(range(0, n, max(1, n // k)))[:k]
        t0 = time.perf_counter()
        _, targets = oracle.search(lo, hi, qcap=q_cap, threads=cores, rows=sel)
        if time.perf_counter() - t0 > 5.0 or k >= n or k >= 512 * cores:
            break
        k *= 2
    times = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        rows, targets = oracle.search(lo, hi, qcap=q_cap, threads=cores, rows=sel)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
    tot = sum(times)
    if q_cap:
        # the capped sweep's unit: column cells (sieving primes q <= T, q < q_cap) of the sampled rows
        per_class = [oracle.count_primes_below(min(t, q_cap - 1) + 1) if t else 0 for t in targets]
        work = sum(per_class[int(rows["type"][i])] for i in sel)
        metric, unit = "128-bit mulmods/s (capped column sweep)", "mulmods/s"
    else:
        work, metric, unit = len(sel), "primes tested/s", "primes/s"
    value = work * len(times) / tot
    line = {
        "metric": metric, "value": value, "unit": unit, "impl": "reference",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "strong" if args.workload == "column-shard" else "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": desc, "sample_rows_per_step": len(sel), "rows_in_workload": n},
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port",
                         "sample": f"{len(sel)} of {n} primes per step, evenly spaced, q_cap={q_cap}",
                         "columns": CPU_COLUMNS},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def serving_record(local, rank, world, dist, requests, rate, max_width, q_cap, warmup, tuning=None,
                   shares="least-work"):
    """The serving stream through a serving session: every request submitted
    at its arrival time, all waited for.  Returns the record (throughput over
    the device-busy time, e2e over the stream's wall time, latencies)."""
    import numpy as np
    import clwilson_b200 as wl
    reqs = serving_requests(1, requests, rate, max_width)[rank::world]
    L = max(limbs_for(b - 1) for _, a, b in reqs)
    srv = wl.Server(local, tuning=tuning, shares=shares)

    late = []

    def stream(reqs):
        # submit each request at its arrival time; `late` records how far behind
        # its schedule each submission was (a stalled host thread shows up there
        # as a burst of submissions, not as server latency)
        ids = []
        del late[:]
        t0 = time.perf_counter()
        for t, a, b in reqs:
            dt = t - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            late.append(1e3 * max(0.0, time.perf_counter() - t0 - t))
            ids.append(srv.submit(a, b, q_cap))
        infos = [srv.wait(i, 3600e3) for i in ids]
        t1 = time.perf_counter()
        for i in ids:
            srv.release(i)
        return infos, t1 - t0

    # warm-up: a few requests through the session (column cache, first launches)
    for _ in range(warmup):
        stream(reqs[:4])
    st0 = srv.stats()
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        infos, wall = stream(reqs)
    st1 = srv.stats()
    srv.close()
    d = {k: st1[k] - st0[k] for k in ("steps", "admitted", "completed", "launches", "ms_steps", "ms_admit",
                                      "ms_wall_steps", "ms_wall_admit", "ms_wall_finish")}
    bad = [i for i in infos if i.state != "done"]
    cells = sum(i.cells for i in infos)
    rows = sum(i.tested for i in infos)
    busy_s = (d["ms_steps"] + d["ms_admit"]) / 1e3
    lat = [i.ms_latency for i in infos]
    queued = [i.ms_queued for i in infos]
    if dist:
        every = [None] * world
        dist.all_gather_object(every, (lat, queued))
        lat = [x for l, _ in every for x in l]
        queued = [x for _, qd in every for x in qd]
    lat = np.array(lat)
    (wall, busy_s), (cells, rows, nreq, nbad) = merge_over_ranks(dist, [wall, busy_s],
                                                                 [cells, rows, len(reqs), len(bad)])
    # host time planning and queueing a step; it overlaps the previous step on the GPU
    plan_us = 1e3 * d["ms_wall_steps"] / max(1, d["steps"])
    return {
        "metric": "128-bit mulmods/s (capped column sweep, serving)", "value": cells / busy_s,
        "unit": "mulmods/s", "higher_is_better": True, "n_gpus": world, "steps": 1, "warmup": warmup,
        "ms_per_step": 1e3 * wall,
        "config": {"workload": f"serving: {int(nreq)} requests from default_rng(1), Poisson at {rate}/s, "
                               f"widths truncated to {max_width}, columns q < {q_cap}",
                   "rate_per_s": rate, "requests": int(nreq), "q_cap": q_cap, "limbs_max": L, "shares": shares,
                   "test_primes": rows, "column_mulmods": cells,
                   "parallelism": f"requests sharded round-robin, dp{world}"},
        "e2e": {"value": cells / wall, "unit": "mulmods/s", "primes_per_s": rows / wall,
                "h2d_bytes_per_step": 16 * int(nreq), "d2h_bytes_per_step": 48 * int(rows)},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "mean": float(lat.mean()), "requests": int(lat.size)},
        "queue_ms_p50": float(np.percentile(queued, 50)),
        "submit_late_ms": {"p99": float(np.percentile(late, 99)), "max": float(max(late))},
        "failed": int(nbad),
        "server": {"steps": d["steps"], "admitted": d["admitted"], "completed": d["completed"],
                   "launches": d["launches"], "peak_active": st1["peak_active"], "busy_s": busy_s,
                   "plan_us_per_step": plan_us,
                   "device_us_per_step": 1e3 * d["ms_steps"] / max(1, d["steps"]),
                   "scheduler_wall_s": {"plan_and_queue": d["ms_wall_steps"] / 1e3,
                                        "admit": d["ms_wall_admit"] / 1e3,
                                        "wait_and_complete": d["ms_wall_finish"] / 1e3}},
        "gpu_launches": d["launches"],
        "clocks": clk.summary(),
    }


def run_serving(args, rank, world, local):
    """The serving stream as its own line."""
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    import clwilson_b200 as wl
    q_cap = 2**28 if args.qcap < 0 else args.qcap
    peak_mad = wl.probe("mad", local)
    # the default kernels unless asked: the tuner times the first requests as
    # one batch, whose best choice can lengthen the serving latency tail
    tuning = None
    if args.serving_autotune:
        reqs = serving_requests(1, args.requests, args.rate, args.max_width)[rank::world]
        eng = wl.Engine(local)
        tuning = eng.autotune([(a, b) for _, a, b in reqs[:64]], q_cap)
        eng.close()
    line = serving_record(local, rank, world, dist, args.requests, args.rate, args.max_width, q_cap,
                          max(3, args.warmup), tuning, args.serving_shares)
    line.update({"scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
                 "tuning": tuning if tuning is not None else "defaults",
                 "roofline": {"bound": "imad", "peak": peak_mad / 1e12, "unit": "TOP/s", "achieved": None,
                              "frac": None, "traffic": None,
                              "note": "device-busy throughput; see the batched and plain lines for the kernels",
                              "peak_source": "wl_probe mad.lo.u32 microbenchmark, this GPU, this run"}})
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def batched_record(eng, rank, world, dist, stream, flush, max_width, steps, plain_steps):
    """The batched workload (256 ranges from default_rng(0), widths truncated
    to max_width, q < 2^28) through wl_batch, one warm-up call on 16 of the
    ranges, `steps` timed calls, and the same ranges as a loop of per-range
    calls (the plain form)."""
    import torch
    ranges, q_cap, desc = workload("batched", rank, world, max_width=max_width)
    per_range_rows = []

    def timed(fn):
        flush.add_(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        out = fn()
        t1 = time.perf_counter()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1) / 1e3, t1 - t0

    def batch():
        eng.drop_columns()
        return eng.batch(ranges, q_cap=q_cap)

    def plain():
        eng.drop_columns()
        cks, cells = [], 0
        for a, b in ranges:
            rows, st = eng.rows(a, b, q_cap=q_cap)
            cks.append(int((rows["p"].astype(object) + rows["s0"].astype(object)
                            + rows["s1"].astype(object)).sum()) % (1 << 64))
            cells += st.cells
        return cks, cells

    eng.batch(ranges[:16], q_cap=q_cap)            # warm-up: first launches, on a few of the ranges
    if dist:
        dist.barrier()
    dev, wall, stats = [], [], []
    for _ in range(steps):
        (per_b, _, st), d, w = timed(batch)
        dev.append(d)
        wall.append(w)
        stats.append(st)
    per_range_rows = [pb["tested"] for pb in per_b]
    pdev, pwall, cks = [], [], None
    for _ in range(plain_steps):
        (cks, cells_p), d, w = timed(plain)
        pdev.append(d)
        pwall.append(w)
    cells = sum(s.cells for s in stats)
    rows = sum(s.tested for s in stats)
    sweep_s = sum(s.ms_sweep for s in stats) / 1e3
    work = [work_cells(s, 4) for s in stats]
    (tot_dev, tot_wall, sweep_s, pd, pw), (cells_all, rows_all, work_all, dense_all, pcells) = merge_over_ranks(
        dist, [sum(dev), sum(wall), sweep_s, sum(pdev), sum(pwall)],
        [cells, rows, sum(w for w, _ in work), sum(x for _, x in work), cells_p * len(pdev) if pdev else 0])
    rec = {
        "metric": "128-bit mulmods/s (capped column sweep, batched)", "value": cells_all / tot_dev,
        "unit": "mulmods/s", "steps": steps, "warmup": "1 call on 16 of the ranges", "ms_per_step": 1e3 * tot_dev / steps,
        "config": {"workload": desc, "q_cap": q_cap, "ranges": len(ranges),
                   "test_primes_per_step": rows_all / steps, "column_mulmods_per_step": cells_all / steps,
                   "rows_per_range": {"min": int(min(per_range_rows)), "max": int(max(per_range_rows))},
                   "l2": "256 MiB buffer written between steps", "columns": "re-sieved every step"},
        "e2e": {"value": cells_all / tot_wall, "unit": "mulmods/s"},
        "gpu_launches": sum(s.kernel_launches for s in stats),
        "cuda_graph": {"nodes_per_step": sum(s.graph_nodes for s in stats) / steps,
                       "host_ms_to_capture_end_and_instantiate": sum(s.ms_graph_build for s in stats) / steps,
                       "note": "the sweep, merge, tail and lift launches of a wl_batch call as one CUDA graph"},
        "work": {"cell_equivalents_per_step": work_all / steps, "dense_share": dense_all / max(1.0, work_all),
                 "cell_equivalents_per_s_in_sweep": work_all / max(sweep_s, 1e-9),
                 "note": "every column cell, plus the dense sweep's window cells and its full products at "
                         "L = 4 cells each"},
    }
    if pdev:
        rec["plain_form"] = {"value": pcells / pd, "unit": "mulmods/s", "e2e": pcells / pw,
                             "ms_per_pass": 1e3 * pd / len(pdev), "passes": len(pdev),
                             "calls_per_pass": len(ranges),
                             "per_range_checksums_equal": [pb["checksum"] for pb in per_b] == cks}
        rec["batched_over_plain"] = rec["value"] / rec["plain_form"]["value"]
    return rec


def run_column_shard(args, rank, world, local):
    """One range, its columns split over the ranks (clwilson_b200.colshard).
    Each step re-sieves the columns; rank 0's events span its piece, the
    gather and the finish, so the step time is the max over ranks."""
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    import clwilson_b200 as wl
    from clwilson_b200 import colshard
    eng = wl.Engine(local)
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", local))
    (lo, hi), = workload("column-shard", rank, world, args.width)[0]
    bounds = colshard.column_pieces(lo, hi, world)
    if dist:
        bounds = colshard.agree_on_bounds(bounds, rank)
    peak_mad = wl.probe("mad", local)
    L = limbs_for(hi - 1)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")   # 256 MiB > L2

    def step():
        eng.drop_columns()
        part, st = None, None
        if rank < len(bounds) - 1:
            part, st = eng.rows_from(lo, hi, bounds[rank], bounds[rank + 1])
        else:
            part, _ = eng.rows_from(lo, hi, 2, 2)       # no piece: the empty product
        if world == 1:
            parts = [part]
        else:
            mine = colshard.piece_digits(part, colshard.piece_interval(bounds, rank))
            parts = colshard.gather_to_rank0(mine, rank, world)
            parts = colshard.check_pieces(bounds, parts) if rank == 0 else None
        res = colshard.finish_pieces(eng, lo, hi, bounds, parts, p=part["p"]) if rank == 0 else None
        return st, res

    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    dev_ms, wall_s, out = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.add_(1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t0 = time.perf_counter()
            st, res = step()
            t1 = time.perf_counter()
            e1.record(stream)
            e1.synchronize()
            dev_ms.append(e0.elapsed_time(e1))
            wall_s.append(t1 - t0)
            out.append((st, res))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    pieces = [st for st, _ in out if st is not None]
    fins = [res for _, res in out if res is not None]
    tested = sum(r.stats.tested for r in fins)
    cells = sum(s.cells for s in pieces)
    sweep_s = sum(s.ms_sweep for s in pieces) / 1e3
    # the piece calls, the row-wise product (one kernel) and the finishing calls
    launches = sum(s.kernel_launches for s in pieces) + sum(r.stats.kernel_launches + 1 for r in fins)
    h2d = (pieces[-1].h2d_bytes if pieces else 0) + (fins[-1].stats.h2d_bytes if fins else 0)
    d2h = (pieces[-1].d2h_bytes if pieces else 0) + (fins[-1].stats.d2h_bytes if fins else 0)
    (tot_dev, tot_wall, _), (tested_all, cells_all, launches_all) = merge_over_ranks(
        dist, [sum(dev_ms) / 1e3, sum(wall_s), sweep_s], [tested, cells, launches])
    achieved = cells * OPS_PER_CELL[L] / max(sweep_s, 1e-9) / 1e12
    line = {
        "metric": "primes tested/s", "value": tested_all / tot_dev, "unit": "primes/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_dev / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"column-shard: every prime in [{lo}, {hi}), full search, columns split over "
                               f"{world} ranks", "column_bounds": bounds, "limbs": L,
                   "test_primes_per_step": tested_all / args.steps,
                   "column_mulmods_per_step": cells_all / args.steps,
                   "l2": "256 MiB buffer written between steps", "columns": "re-sieved every step",
                   "parallelism": f"columns sharded, {world} pieces; one gather of 16 B per row and rank to rank 0"},
        "roofline": {"bound": "imad", "achieved": achieved, "peak": peak_mad / 1e12, "unit": "TOP/s",
                     "frac": achieved * 1e12 / peak_mad, "traffic": None, "kernel": f"k_sweep<{L},*> (rank {rank})",
                     "ops_per_cell": OPS_PER_CELL[L],
                     "peak_source": "wl_probe mad.lo.u32 microbenchmark, this GPU, this run"},
        "e2e": {"value": tested_all / tot_wall, "unit": "primes/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches_all),
        "tuning": "defaults",
        "clocks": clk.summary(),
    }
    if rank == 0:
        one = eng.search(lo, hi)
        line["checksum_equal_one_call"] = all(r.checksum == one.checksum and r.results == one.results for r in fins)
        if not args.no_cpu_baseline:
            cb, want, sel = cpu_baseline(lo, hi, 0, 20.0 if world == 1 else 5.0)
            if world == 1:
                line["cpu_baseline"] = cb
            line["parity_sample"] = parity_sample(eng, lo, hi, 0, want, sel)
            line["parity_sample_ok"] = line["parity_sample"]["ok"]
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain-small",
                    choices=["plain-small", "plain-mid", "plain-top", "batched", "serving", "column-shard"])
    ap.add_argument("--max-width", type=int, default=2000,
                    help="batched/serving: truncate each range to this many integers (0: whole ranges)")
    ap.add_argument("--requests", type=int, default=256, help="serving: requests in the stream")
    ap.add_argument("--rate", type=float, default=64.0, help="serving: mean arrival rate, requests/s")
    ap.add_argument("--plain-steps", type=int, default=2, help="batched: timed passes of the plain per-range loop")
    ap.add_argument("--width", type=int, default=0,
                    help="range width per GPU (default: the configuration's; smaller only for profiling)")
    ap.add_argument("--qcap", type=int, default=-1,
                    help="column cap q < QCAP (default: the configuration's; only for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default kernel choices instead of timing the variants before the warm-up")
    ap.add_argument("--serving-autotune", action="store_true",
                    help="serving: tune the kernels on the first 64 requests run as one batch (batch throughput; "
                         "the default kernels are kept otherwise)")
    ap.add_argument("--serving-shares", default="least-work", choices=["least-work", "equal"],
                    help="serving: how a scheduler step's budget is split between requests")
    ap.add_argument("--no-sub-records", action="store_true",
                    help="plain-small: skip the batched and serving records that the default run adds")
    ap.add_argument("--sub-batched-width", type=int, default=50000,
                    help="batched record: truncate each of the 256 ranges to this many integers")
    ap.add_argument("--sub-batched-steps", type=int, default=1, help="batched record: timed calls")
    ap.add_argument("--sub-serving-requests", type=int, default=2000, help="serving record: requests in the stream")
    ap.add_argument("--sub-serving-rate", type=float, default=64.0, help="serving record: arrivals per second")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "serving":
        return run_serving(args, rank, world, local)
    if args.workload == "column-shard":
        return run_column_shard(args, rank, world, local)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))

    import clwilson_b200 as wl
    eng = wl.Engine(local)
    stream = torch.cuda.ExternalStream(eng.stream, device=torch.device("cuda", local))
    ranges, q_cap, desc = workload(args.workload, rank, world, args.width, args.qcap, args.max_width)
    L = max(limbs_for(b - 1) for a, b in ranges)
    t_tune = time.perf_counter()
    # tune on the workload itself; the capped plain workloads (over a minute per
    # step) on the first 1% of their range
    tune_ranges = ranges
    if args.workload in ("plain-mid", "plain-top"):
        tune_ranges = [(a, a + max(20000, (b - a) // 100)) for a, b in ranges]
    tuning = None if args.no_autotune else eng.autotune(tune_ranges, q_cap)
    t_tune = time.perf_counter() - t_tune
    peak_mad = wl.probe("mad", local)
    # the register-only rate of the cell formulation the sweeps run (wide products)
    peak_cell = wl.probe("cell%dw" % L, local)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")   # 256 MiB > L2

    def step():
        eng.drop_columns()
        if len(ranges) == 1:
            r = eng.search(ranges[0][0], ranges[0][1], q_cap=q_cap)
            return r.stats
        per, res, st = eng.batch(ranges, q_cap=q_cap)
        return st

    for _ in range(args.warmup):
        step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    dev_ms, wall_s, stats = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.add_(1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t0 = time.perf_counter()
            st = step()
            t1 = time.perf_counter()
            e1.record(stream)
            e1.synchronize()
            dev_ms.append(e0.elapsed_time(e1))
            wall_s.append(t1 - t0)
            stats.append(st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()

    tested = sum(s.tested for s in stats)
    tot_dev = sum(dev_ms) / 1e3
    tot_wall = sum(wall_s)
    sweep_s = sum(s.ms_sweep for s in stats) / 1e3
    cells = sum(s.cells for s in stats)
    launches = sum(s.kernel_launches for s in stats)
    h2d = stats[-1].h2d_bytes
    d2h = stats[-1].d2h_bytes
    (tot_dev, tot_wall, _), (tested_all, cells_all, _) = merge_over_ranks(
        dist, [tot_dev, tot_wall, sweep_s], [tested, cells, launches])

    full = q_cap == 0
    # cells the sweep kernels executed: every column cell, and in the dense
    # regime the window cells and full products counted on the device
    exec_cells = sum(work_cells(s, L)[0] for s in stats)
    dense_cells = sum(work_cells(s, L)[1] for s in stats)
    achieved = exec_cells * OPS_PER_CELL[L] / sweep_s / 1e12
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            traffic = json.load(open(tpath)).get(args.workload)
        except Exception:
            traffic = None
    line = {
        "metric": "primes tested/s" if full else "128-bit mulmods/s (capped column sweep)",
        "value": (tested_all / tot_dev) if full else (cells_all / tot_dev),
        "unit": "primes/s" if full else "mulmods/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot_dev / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic",
        "config": {"workload": desc, "q_cap": q_cap, "limbs": L, "test_primes_per_step": tested_all / args.steps,
                   "column_mulmods_per_step": cells_all / args.steps,
                   "tail_steps_per_step": sum(s.tail_steps for s in stats) / args.steps,
                   "l2": "256 MiB buffer written between steps", "columns": "re-sieved every step",
                   "parallelism": f"rows sharded by range, dp{world}"},
        "mulmods_per_s": cells_all / tot_dev,
        "roofline": {"bound": "imad", "achieved": achieved, "peak": peak_mad / 1e12, "unit": "TOP/s",
                     "frac": achieved * 1e12 / peak_mad, "traffic": traffic,
                     "traffic_source": ("dram__bytes_read.sum + dram__bytes_write.sum of the step's sweep launches of "
                                        "this workload, one ncu capture (profiles/traffic.json)") if traffic else None,
                     "kernel": f"k_sweep<{L},*>" if dense_cells < 0.5 * exec_cells else f"k_sweep_dense<{L},*>",
                     "ops_per_cell": OPS_PER_CELL[L],
                     "cells_executed_per_step": exec_cells / args.steps,
                     "dense_share_of_cells": dense_cells / max(1.0, exec_cells),
                     "dense_per_step": {k: sum(getattr(s, "dense_" + k) for s in stats) / args.steps
                                        for k in ("column_cells", "window_cells", "products")},
                     "cell_peak_per_s": peak_cell, "cell_frac": (exec_cells / sweep_s) / peak_cell,
                     "peak_source": "wl_probe mad.lo.u32 microbenchmark, this GPU, this run",
                     "count": "cells executed: one per (row, column), plus the dense sweep's window cells and "
                              "its full products at L cells each (device counters)"},
        "e2e": {"value": (tested_all / tot_wall) if full else (cells_all / tot_wall),
                "unit": "primes/s" if full else "mulmods/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "tuning": tuning if tuning is not None else "defaults",
        "autotune_s": round(t_tune, 2),
        "clocks": clk.summary(),
        "phase_ms_per_step": {k: sum(getattr(s, "ms_" + k) for s in stats) / args.steps
                              for k in ("primes", "sieve", "sweep", "iterate", "finish")},
    }
    # the column sieve (q < 2^32): its device-memory traffic over its event time
    sieve_ms = sum(s.ms_sieve for s in stats)
    if sieve_ms > 0:
        peak_gbs, src = hbm_peak()
        gbs = sum(s.sieve_bytes for s in stats) / (sieve_ms / 1e3) / 1e9
        line["sieve"] = {"ms_per_step": sieve_ms / args.steps,
                         "integers_per_step": sum(s.sieve_integers for s in stats) / args.steps,
                         "bytes_per_step": sum(s.sieve_bytes for s in stats) / args.steps,
                         "gbs": gbs, "hbm_peak_gbs": peak_gbs, "hbm_frac": gbs / peak_gbs, "peak_source": src,
                         "integers_per_s": sum(s.sieve_integers for s in stats) / (sieve_ms / 1e3),
                         "bound": "shared-memory marking (the bitmap is built in shared memory; HBM carries "
                                  "the bitmap, counts and the ordered column table)"}
    if len(ranges) > 1 and args.plain_steps > 0:
        # the plain form: one wl_search per range, same ranges, same column cap
        per_b, _, _ = eng.batch(ranges, q_cap=q_cap)

        def plain():
            eng.drop_columns()
            cks, cells_p = [], 0
            for a, b in ranges:
                if q_cap:
                    rows, st = eng.rows(a, b, q_cap=q_cap)
                    cks.append(int((rows["p"].astype(object) + rows["s0"].astype(object)
                                    + rows["s1"].astype(object)).sum()) % (1 << 64))
                else:
                    r = eng.search(a, b)
                    st = r.stats
                    cks.append(r.checksum)
                cells_p += st.cells
            return cks, cells_p
        cks, _ = plain()
        pdev, pwall = [], []
        for _ in range(args.plain_steps):
            flush.add_(1)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t0 = time.perf_counter()
            cks, cells_p = plain()
            t1 = time.perf_counter()
            e1.record(stream)
            e1.synchronize()
            pdev.append(e0.elapsed_time(e1) / 1e3)
            pwall.append(t1 - t0)
        line["plain_form"] = {
            "value": cells_p * len(pdev) / sum(pdev), "unit": line["unit"],
            "e2e": cells_p * len(pwall) / sum(pwall), "ms_per_pass": 1e3 * sum(pdev) / len(pdev),
            "passes": len(pdev), "calls_per_pass": len(ranges),
            "per_range_checksums_equal": [pb["checksum"] for pb in per_b] == cks,
        }
        line["batched_over_plain"] = line["value"] / line["plain_form"]["value"]
    if rank == 0 and not args.no_cpu_baseline:
        # the oracle on a sample of rows: the CPU baseline (one GPU), and in
        # every run the check of the engine's rows at the same indices
        lo, hi = max(ranges, key=lambda r: r[1] - r[0])
        cb, want, sel = cpu_baseline(lo, hi, q_cap, 20.0 if world == 1 else 5.0)
        if not full:
            cb["note"] = "capped sweep: value is primes/s of the capped partial products"
        if world == 1:
            line["cpu_baseline"] = cb
        line["parity_sample"] = parity_sample(eng, lo, hi, q_cap, want, sel)
        line["parity_sample_ok"] = line["parity_sample"]["ok"]
    if args.workload == "plain-small" and not args.no_sub_records:
        # the rest of the headline metric: batched against plain, and serving latency
        line["serving"] = serving_record(local, rank, world, dist, args.sub_serving_requests,
                                         args.sub_serving_rate, 2000, 2**28, 3)
        line["batched"] = batched_record(eng, rank, world, dist, stream, flush, args.sub_batched_width,
                                         args.sub_batched_steps, 1)
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
