"""clwilson_b200 -- B200-native Wilson-prime search engine.

Python host bindings over the C ABI of ``libwilson.so`` (include/wilson.h).
The computation runs only in the CUDA kernels of that library; importing this
package without the built library raises, and there is no CPU fallback.

Mirrors the reference program's surface (mfl0p/CLWilson):
  * ``search(pmin, pmax)``      one run of cl_wilson() (cl_wilson.cpp:1442-1974):
                                result lines and checksum
  * ``rows(pmin, pmax)``        per-prime residues and quotients
  * ``batch(ranges)``           many ranges in one device pass
  * ``Server``                  resident serving session with continuous batching
  * ``write_results(...)``      results.txt in the reference's byte format
                                (cl_wilson.cpp:657-688, 1093-1143)
  * ``parse_uint64``            the CLI number parser (putil.c:34-116)
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libwilson.so")

WL_MAXP = 4611686018427387903
WL_MAX_WIDTH = 10_000_000
ERRORS = {
    -1: "invalid argument or range", -2: "CUDA error", -3: "there are no primes to test in this range!",
    -4: "configuration not supported by this library", -5: "Wilson quotient check failed",
    -6: "representation a, c or u not found", -7: "result buffer too small", -8: "device allocation failed",
    -9: "request exceeds the fixed scratch of the no-allocation entry point",
}


class WilsonError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        super().__init__(f"{what}: {ERRORS.get(code, 'unknown error')} ({code})" if what else ERRORS.get(code, str(code)))


class _Result(ctypes.Structure):
    _fields_ = [("p", ctypes.c_uint64), ("value", ctypes.c_int32), ("pad", ctypes.c_uint32)]


class _Row(ctypes.Structure):
    _fields_ = [("p", ctypes.c_uint64), ("s0", ctypes.c_uint64), ("s1", ctypes.c_uint64),
                ("rem", ctypes.c_uint64), ("quot", ctypes.c_uint64), ("type", ctypes.c_uint32),
                ("status", ctypes.c_uint32)]


class _Range(ctypes.Structure):
    _fields_ = [("pmin", ctypes.c_uint64), ("pmax", ctypes.c_uint64)]


class _RangeResult(ctypes.Structure):
    _fields_ = [("tested", ctypes.c_uint64), ("checksum", ctypes.c_uint64), ("targets", ctypes.c_uint64 * 3),
                ("results", ctypes.c_uint32), ("status", ctypes.c_uint32)]


class _Stats(ctypes.Structure):
    _fields_ = [("tested", ctypes.c_uint64), ("per_class", ctypes.c_uint64 * 3), ("targets", ctypes.c_uint64 * 3),
                ("pi_maxtarget", ctypes.c_uint64), ("cells", ctypes.c_uint64), ("tail_steps", ctypes.c_uint64),
                ("checksum", ctypes.c_uint64), ("results", ctypes.c_uint32), ("kernel_launches", ctypes.c_uint32),
                ("ms_device", ctypes.c_double), ("ms_primes", ctypes.c_double), ("ms_sieve", ctypes.c_double),
                ("ms_sweep", ctypes.c_double), ("ms_iterate", ctypes.c_double), ("ms_finish", ctypes.c_double),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64), ("ms_big", ctypes.c_double),
                ("sieve_integers", ctypes.c_uint64), ("sieve_bytes", ctypes.c_uint64),
                ("dense_column_cells", ctypes.c_uint64), ("dense_window_cells", ctypes.c_uint64),
                ("dense_products", ctypes.c_uint64), ("graph_nodes", ctypes.c_uint64),
                ("ms_graph_build", ctypes.c_double)]


class _Tuning(ctypes.Structure):
    _fields_ = [("sparse_variant", ctypes.c_int32 * 3), ("sparse_rpt", ctypes.c_int32 * 3),
                ("dense_kernel", ctypes.c_int32 * 3), ("dense_hstep", ctypes.c_int32 * 3),
                ("merge_cta_min", ctypes.c_int32), ("pad", ctypes.c_int32), ("ms", ctypes.c_double * 3)]

    def to_dict(self) -> dict:
        return {k: (list(getattr(self, k)) if k in ("sparse_variant", "sparse_rpt", "dense_kernel", "dense_hstep", "ms")
                    else getattr(self, k)) for k, _ in self._fields_ if k != "pad"}

    @classmethod
    def from_dict(cls, d: dict) -> "_Tuning":
        t = cls()
        for k, v in d.items():
            if k in ("sparse_variant", "sparse_rpt", "dense_kernel", "dense_hstep"):
                setattr(t, k, (ctypes.c_int32 * 3)(*v))
            elif k == "ms":
                setattr(t, k, (ctypes.c_double * 3)(*v))
            elif k == "merge_cta_min":
                t.merge_cta_min = v
        return t


class _ServerOpts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("shares", ctypes.c_uint32), ("pool_bytes", ctypes.c_uint64),
                ("step_cells", ctypes.c_uint64), ("tuning", ctypes.c_void_p)]


class _RequestInfo(ctypes.Structure):
    _fields_ = [("id", ctypes.c_uint64), ("state", ctypes.c_int32), ("rc", ctypes.c_int32),
                ("tested", ctypes.c_uint64), ("checksum", ctypes.c_uint64), ("targets", ctypes.c_uint64 * 3),
                ("cells", ctypes.c_uint64), ("results", ctypes.c_uint32), ("pad", ctypes.c_uint32),
                ("ms_queued", ctypes.c_double), ("ms_latency", ctypes.c_double)]


class _ServerStats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_uint64), ("admitted", ctypes.c_uint64), ("completed", ctypes.c_uint64),
                ("failed", ctypes.c_uint64), ("cancelled", ctypes.c_uint64), ("rows_done", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("launches", ctypes.c_uint64), ("ms_steps", ctypes.c_double),
                ("ms_admit", ctypes.c_double), ("peak_rows", ctypes.c_uint32), ("peak_active", ctypes.c_uint32),
                ("ms_wall_steps", ctypes.c_double), ("ms_wall_admit", ctypes.c_double),
                ("ms_wall_finish", ctypes.c_double)]


REQ_STATES = {0: "queued", 1: "active", 2: "done", 3: "cancelled", 4: "failed"}
SERVER_ROW_BYTES = 160

ROW_DTYPE = np.dtype([("p", "<u8"), ("s0", "<u8"), ("s1", "<u8"), ("rem", "<u8"), ("quot", "<u8"),
                      ("type", "<u4"), ("status", "<u4")])
assert ROW_DTYPE.itemsize == ctypes.sizeof(_Row)

# exported symbols of include/wilson.h
SYMBOLS = ("wl_open", "wl_close", "wl_strerror", "wl_stream", "wl_check_range", "wl_search", "wl_rows",
           "wl_batch", "wl_rows_from", "wl_search_from", "wl_rows_product", "wl_drop_columns", "wl_parse_uint64",
           "wl_probe",
           "wl_column_product_noalloc", "wl_get_tuning", "wl_set_tuning", "wl_autotune",
           "wl_server_open", "wl_server_submit", "wl_server_poll", "wl_server_wait", "wl_server_results",
           "wl_server_rows", "wl_server_cancel", "wl_server_release", "wl_server_stats_get", "wl_server_close")
# cellL: the carry-chain cell; cellLw: the wide-product cell the sweeps run by default
PROBES = {"mad": 0, "madhi": 1, "cell2": 2, "cell3": 3, "cell4": 4, "madwide": 5,
          "cell2w": 101, "cell3w": 111, "cell4w": 121}

_lib = None


def load_library(path: str = LIB_PATH):
    """Load libwilson.so and declare its C signatures.  Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"libwilson.so not built ({path}); run `python -m clwilson_b200.build`")
    L = ctypes.CDLL(path)
    u64, vp, sz = ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t
    L.wl_open.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.wl_open.restype = ctypes.c_int
    L.wl_close.argtypes = [vp]
    L.wl_close.restype = None
    L.wl_strerror.argtypes = [ctypes.c_int]
    L.wl_strerror.restype = ctypes.c_char_p
    L.wl_stream.argtypes = [vp]
    L.wl_stream.restype = vp
    L.wl_check_range.argtypes = [u64, u64]
    L.wl_check_range.restype = ctypes.c_int
    L.wl_search.argtypes = [vp, u64, u64, u64, ctypes.POINTER(_Result), sz, ctypes.POINTER(_Stats)]
    L.wl_search.restype = ctypes.c_int
    L.wl_rows.argtypes = [vp, u64, u64, u64, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(_Stats)]
    L.wl_rows.restype = ctypes.c_int
    L.wl_batch.argtypes = [vp, ctypes.POINTER(_Range), sz, u64, ctypes.POINTER(_RangeResult),
                           ctypes.POINTER(_Result), sz, ctypes.POINTER(sz), ctypes.POINTER(_Stats)]
    L.wl_batch.restype = ctypes.c_int
    L.wl_rows_from.argtypes = [vp, u64, u64, u64, u64, vp, vp, sz, ctypes.POINTER(sz), ctypes.POINTER(_Stats)]
    L.wl_rows_from.restype = ctypes.c_int
    L.wl_search_from.argtypes = [vp, u64, u64, u64, vp, ctypes.POINTER(_Result), sz, ctypes.POINTER(_Stats)]
    L.wl_search_from.restype = ctypes.c_int
    L.wl_rows_product.argtypes = [vp, sz, vp, sz, vp, vp]
    L.wl_rows_product.restype = ctypes.c_int
    L.wl_parse_uint64.argtypes = [ctypes.POINTER(u64), ctypes.c_char_p, u64, u64]
    L.wl_parse_uint64.restype = ctypes.c_int
    L.wl_drop_columns.argtypes = [vp]
    L.wl_drop_columns.restype = None
    L.wl_probe.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    L.wl_probe.restype = ctypes.c_int
    L.wl_column_product_noalloc.argtypes = [vp, ctypes.c_uint32, u64, u64, vp, ctypes.c_uint32, vp, vp]
    L.wl_column_product_noalloc.restype = ctypes.c_int
    L.wl_get_tuning.argtypes = [vp, ctypes.POINTER(_Tuning)]
    L.wl_set_tuning.argtypes = [vp, ctypes.POINTER(_Tuning)]
    L.wl_autotune.argtypes = [vp, ctypes.POINTER(_Range), sz, u64, ctypes.c_uint32, ctypes.POINTER(_Tuning)]
    for fn in ("wl_get_tuning", "wl_set_tuning", "wl_autotune"):
        getattr(L, fn).restype = ctypes.c_int
    L.wl_server_open.argtypes = [ctypes.POINTER(_ServerOpts), ctypes.POINTER(vp)]
    L.wl_server_submit.argtypes = [vp, u64, u64, u64, ctypes.POINTER(u64)]
    L.wl_server_poll.argtypes = [vp, u64, ctypes.POINTER(_RequestInfo)]
    L.wl_server_wait.argtypes = [vp, u64, ctypes.POINTER(_RequestInfo), ctypes.c_double]
    L.wl_server_results.argtypes = [vp, u64, ctypes.POINTER(_Result), sz, ctypes.POINTER(sz)]
    L.wl_server_rows.argtypes = [vp, u64, vp, sz, ctypes.POINTER(sz)]
    L.wl_server_cancel.argtypes = [vp, u64]
    L.wl_server_release.argtypes = [vp, u64]
    L.wl_server_stats_get.argtypes = [vp, ctypes.POINTER(_ServerStats)]
    for fn in ("wl_server_open", "wl_server_submit", "wl_server_poll", "wl_server_wait", "wl_server_results",
               "wl_server_rows", "wl_server_cancel", "wl_server_release", "wl_server_stats_get"):
        getattr(L, fn).restype = ctypes.c_int
    L.wl_server_close.argtypes = [vp]
    L.wl_server_close.restype = None
    _lib = L
    return L


def parse_uint64(text: str, lo: int, hi: int) -> Tuple[int, int]:
    """(status, value): status 0 ok, -1 cannot parse, -2 out of range (putil.c:34-116)."""
    L = load_library()
    v = ctypes.c_uint64(0)
    rc = L.wl_parse_uint64(ctypes.byref(v), text.encode(), lo, hi)
    return rc, v.value


def probe(which: str, device: int = 0) -> float:
    """Integer-pipe microbenchmark (include/wilson_probe.h): operations or cells per second."""
    L = load_library()
    r = ctypes.c_double(0)
    rc = L.wl_probe(device, PROBES[which], ctypes.byref(r))
    if rc:
        raise WilsonError(rc, "wl_probe")
    return r.value


def check_range(pmin: int, pmax: int) -> int:
    return load_library().wl_check_range(pmin, pmax)


@dataclass
class Stats:
    tested: int = 0
    per_class: Tuple[int, int, int] = (0, 0, 0)
    targets: Tuple[int, int, int] = (0, 0, 0)
    pi_maxtarget: int = 0
    cells: int = 0
    tail_steps: int = 0
    checksum: int = 0
    results: int = 0
    kernel_launches: int = 0
    ms_device: float = 0.0
    ms_primes: float = 0.0
    ms_sieve: float = 0.0
    ms_sweep: float = 0.0
    ms_iterate: float = 0.0
    ms_finish: float = 0.0
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    ms_big: float = 0.0
    sieve_integers: int = 0
    sieve_bytes: int = 0
    dense_column_cells: int = 0
    dense_window_cells: int = 0
    dense_products: int = 0
    graph_nodes: int = 0
    ms_graph_build: float = 0.0

    @classmethod
    def from_c(cls, s: _Stats) -> "Stats":
        return cls(s.tested, tuple(s.per_class), tuple(s.targets), s.pi_maxtarget, s.cells, s.tail_steps,
                   s.checksum, s.results, s.kernel_launches, s.ms_device, s.ms_primes, s.ms_sieve, s.ms_sweep,
                   s.ms_iterate, s.ms_finish, s.h2d_bytes, s.d2h_bytes, s.ms_big, s.sieve_integers, s.sieve_bytes,
                   s.dense_column_cells, s.dense_window_cells, s.dense_products, s.graph_nodes, s.ms_graph_build)


@dataclass
class SearchResult:
    results: List[Tuple[int, int]]   # (p, value): value 0 = Wilson prime, else Near-Wilson +-value
    checksum: int
    stats: Stats = field(default_factory=Stats)

    def lines(self) -> List[str]:
        return [result_line(p, v) for p, v in self.results]


def result_line(p: int, value: int) -> str:
    """One results.txt line (cl_wilson.cpp:665-676)."""
    if value == 0:
        return f"{p} is a Wilson prime"
    return f"{p} is a Near-Wilson prime {value:+d}"


def write_results(path: str, results: Sequence[Tuple[int, int]], checksum: int, append: bool = False) -> None:
    """results.txt: the lines in ascending p, then the checksum line
    (finalizeResults, cl_wilson.cpp:1126-1137)."""
    with open(path, "a" if append else "w") as f:
        for p, v in results:
            f.write(result_line(p, v) + "\n")
        if results:
            f.write("%016X\n" % checksum)
        else:
            f.write("no results\n%016X\n" % checksum)


class Engine:
    """One context on one GPU (wl_open / wl_close)."""

    def __init__(self, device: int = 0):
        self._L = load_library()
        self._ctx = ctypes.c_void_p()
        rc = self._L.wl_open(device, ctypes.byref(self._ctx))
        if rc:
            raise WilsonError(rc, "wl_open")

    def close(self) -> None:
        if self._ctx:
            self._L.wl_close(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def drop_columns(self) -> None:
        self._L.wl_drop_columns(self._ctx)

    @property
    def tuning(self) -> dict:
        t = _Tuning()
        rc = self._L.wl_get_tuning(self._ctx, ctypes.byref(t))
        if rc:
            raise WilsonError(rc, "wl_get_tuning")
        return t.to_dict()

    @tuning.setter
    def tuning(self, d: dict) -> None:
        """Set some or all choices (keys of the `tuning` dict)."""
        cur = self.tuning
        cur.update(d)
        t = _Tuning.from_dict(cur)
        rc = self._L.wl_set_tuning(self._ctx, ctypes.byref(t))
        if rc:
            raise WilsonError(rc, "wl_set_tuning")

    def autotune(self, ranges: Optional[Sequence[Tuple[int, int]]] = None, q_cap: int = 0, limbs=(2, 3, 4)) -> dict:
        """Time the sweep kernel variants and keep the fastest in this context
        (wl_autotune): on the given ranges (the workload), or on built-in
        samples for the given limb widths."""
        mask = 0
        for L in limbs:
            mask |= 1 << (L - 2)
        t = _Tuning()
        n = len(ranges) if ranges else 0
        rr = (_Range * max(n, 1))(*[_Range(a, b) for a, b in (ranges or [])])
        rc = self._L.wl_autotune(self._ctx, rr if n else None, n, q_cap, mask, ctypes.byref(t))
        if rc:
            raise WilsonError(rc, "wl_autotune")
        return t.to_dict()

    @property
    def stream(self) -> int:
        return self._L.wl_stream(self._ctx) or 0

    def search(self, pmin: int, pmax: int, q_cap: int = 0, cap: int = 1 << 16) -> SearchResult:
        res = (_Result * cap)()
        st = _Stats()
        rc = self._L.wl_search(self._ctx, pmin, pmax, q_cap, res, cap, ctypes.byref(st))
        if rc:
            raise WilsonError(rc, "wl_search")
        out = [(res[i].p, res[i].value) for i in range(min(st.results, cap))]
        return SearchResult(out, st.checksum, Stats.from_c(st))

    def rows(self, pmin: int, pmax: int, q_cap: int = 0) -> Tuple[np.ndarray, Stats]:
        n = ctypes.c_size_t(0)
        st = _Stats()
        # size the buffer generously: primes in the window are < width/2 + 2
        cap = (pmax - pmin) // 2 + 2
        buf = np.zeros(cap, dtype=ROW_DTYPE)
        rc = self._L.wl_rows(self._ctx, pmin, pmax, q_cap, buf.ctypes.data, cap, ctypes.byref(n), ctypes.byref(st))
        if rc and rc not in (-5, -6):
            raise WilsonError(rc, "wl_rows")
        return buf[: n.value].copy(), Stats.from_c(st)

    @staticmethod
    def _init_array(init):
        if init is None:
            return None, None
        a = np.ascontiguousarray(np.stack([np.asarray(init["s0"], dtype=np.uint64),
                                           np.asarray(init["s1"], dtype=np.uint64)], axis=1))
        return a, a.ctypes.data

    def rows_from(self, pmin: int, pmax: int, q_lo: int, q_cap: int = 0, init=None) -> Tuple[np.ndarray, Stats]:
        """Rows over the sieving primes q in [q_lo, q_cap), continuing from the
        running products `init` (rows of an earlier capped call, or None)."""
        keep, ptr = self._init_array(init)
        n = ctypes.c_size_t(0)
        st = _Stats()
        cap = (pmax - pmin) // 2 + 2
        buf = np.zeros(cap, dtype=ROW_DTYPE)
        rc = self._L.wl_rows_from(self._ctx, pmin, pmax, q_lo, q_cap, ptr, buf.ctypes.data, cap, ctypes.byref(n),
                                  ctypes.byref(st))
        if rc and rc not in (-5, -6):
            raise WilsonError(rc, "wl_rows_from")
        return buf[: n.value].copy(), Stats.from_c(st)

    def search_from(self, pmin: int, pmax: int, q_lo: int, init=None, cap: int = 1 << 16) -> SearchResult:
        keep, ptr = self._init_array(init)
        res = (_Result * cap)()
        st = _Stats()
        rc = self._L.wl_search_from(self._ctx, pmin, pmax, q_lo, ptr, res, cap, ctypes.byref(st))
        if rc:
            raise WilsonError(rc, "wl_search_from")
        out = [(res[i].p, res[i].value) for i in range(min(st.results, cap))]
        return SearchResult(out, st.checksum, Stats.from_c(st))

    def rows_product(self, parts, p=None) -> np.ndarray:
        """Row-wise product of partial column products (wl_rows_product).

        `parts`: pieces of one range over disjoint column intervals (same
        primes, same order), each either rows (wl_rows_from) or an (n, 2)
        array of digits (s0, s1).  `p`: the primes, when no part is rows.
        Returns rows with p and the digits (s0, s1) of the product mod p^2,
        the init of the finishing search_from."""
        parts = list(parts)
        if not parts:
            raise ValueError("rows_product needs at least one part")
        rows_parts = [x for x in parts if x.dtype.names]
        if p is None:
            if not rows_parts:
                raise ValueError("rows_product: give p or at least one part as rows")
            p = rows_parts[0]["p"]
        p = np.ascontiguousarray(p, dtype=np.uint64)
        n = p.size
        digits = np.empty((len(parts), n, 2), dtype=np.uint64)
        for k, x in enumerate(parts):
            if x.dtype.names:
                if not np.array_equal(x["p"], p):
                    raise ValueError("rows_product: the parts hold different primes")
                digits[k, :, 0] = x["s0"]
                digits[k, :, 1] = x["s1"]
            else:
                if x.shape != (n, 2):
                    raise ValueError("rows_product: a digit part must have shape (%d, 2)" % n)
                digits[k] = x
        out = np.zeros((max(n, 1), 2), dtype=np.uint64)
        rc = self._L.wl_rows_product(self._ctx, n, p.ctypes.data, len(parts), digits.ctypes.data, out.ctypes.data)
        if rc:
            raise WilsonError(rc, "wl_rows_product")
        rows = np.zeros(n, dtype=ROW_DTYPE)
        rows["p"] = p
        rows["s0"] = out[:n, 0]
        rows["s1"] = out[:n, 1]
        if rows_parts:
            rows["type"] = rows_parts[0]["type"]
        return rows

    def batch(self, ranges: Sequence[Tuple[int, int]], q_cap: int = 0, cap: int = 1 << 20):
        n = len(ranges)
        rr = (_Range * n)(*[_Range(a, b) for a, b in ranges])
        out = (_RangeResult * n)()
        res = (_Result * cap)()
        nres = ctypes.c_size_t(0)
        st = _Stats()
        rc = self._L.wl_batch(self._ctx, rr, n, q_cap, out, res, cap, ctypes.byref(nres), ctypes.byref(st))
        if rc:
            raise WilsonError(rc, "wl_batch")
        per_range = [dict(tested=o.tested, checksum=o.checksum, targets=tuple(o.targets), results=o.results,
                          status=o.status) for o in out]
        results = [(res[i].p, res[i].value) for i in range(min(nres.value, cap))]
        return per_range, results, Stats.from_c(st)


@dataclass
class RequestInfo:
    id: int
    state: str
    rc: int
    tested: int
    checksum: int
    targets: Tuple[int, int, int]
    cells: int
    results: int
    ms_queued: float
    ms_latency: float

    @classmethod
    def from_c(cls, r: _RequestInfo) -> "RequestInfo":
        return cls(r.id, REQ_STATES.get(r.state, str(r.state)), r.rc, r.tested, r.checksum, tuple(r.targets),
                   r.cells, r.results, r.ms_queued, r.ms_latency)


class Server:
    """Resident serving session (wl_server_*): ranges submitted at any time
    are admitted into a device row pool as it frees up and share the GPU's
    column sweeps with the requests already running; each request's results
    equal those of ``Engine.search`` / ``Engine.rows`` on its range."""

    def __init__(self, device: int = 0, pool_bytes: int = 0, step_cells: int = 0, tuning: Optional[dict] = None,
                 shares: str = "least-work"):
        self._L = load_library()
        self._srv = ctypes.c_void_p()
        self._tune = _Tuning.from_dict(tuning) if tuning else None
        policy = {"least-work": 0, "equal": 1}[shares]
        o = _ServerOpts(device, policy, pool_bytes, step_cells,
                        ctypes.cast(ctypes.pointer(self._tune), ctypes.c_void_p) if tuning else None)
        rc = self._L.wl_server_open(ctypes.byref(o), ctypes.byref(self._srv))
        if rc:
            raise WilsonError(rc, "wl_server_open")

    def close(self) -> None:
        if self._srv:
            self._L.wl_server_close(self._srv)
            self._srv = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, pmin: int, pmax: int, q_cap: int = 0) -> int:
        rid = ctypes.c_uint64(0)
        rc = self._L.wl_server_submit(self._srv, pmin, pmax, q_cap, ctypes.byref(rid))
        if rc:
            raise WilsonError(rc, "wl_server_submit")
        return rid.value

    def poll(self, rid: int) -> RequestInfo:
        info = _RequestInfo()
        rc = self._L.wl_server_poll(self._srv, rid, ctypes.byref(info))
        if rc < 0:
            raise WilsonError(rc, "wl_server_poll")
        return RequestInfo.from_c(info)

    def wait(self, rid: int, timeout_ms: float = -1.0) -> RequestInfo:
        info = _RequestInfo()
        rc = self._L.wl_server_wait(self._srv, rid, ctypes.byref(info), timeout_ms)
        if rc < 0:
            raise WilsonError(rc, "wl_server_wait")
        return RequestInfo.from_c(info)

    def results(self, rid: int) -> List[Tuple[int, int]]:
        n = ctypes.c_size_t(0)
        rc = self._L.wl_server_results(self._srv, rid, None, 0, ctypes.byref(n))
        if rc:
            raise WilsonError(rc, "wl_server_results")
        res = (_Result * max(n.value, 1))()
        rc = self._L.wl_server_results(self._srv, rid, res, n.value, ctypes.byref(n))
        if rc:
            raise WilsonError(rc, "wl_server_results")
        return [(res[i].p, res[i].value) for i in range(n.value)]

    def rows(self, rid: int) -> np.ndarray:
        n = ctypes.c_size_t(0)
        rc = self._L.wl_server_rows(self._srv, rid, None, 0, ctypes.byref(n))
        if rc:
            raise WilsonError(rc, "wl_server_rows")
        buf = np.zeros(max(n.value, 1), dtype=ROW_DTYPE)
        rc = self._L.wl_server_rows(self._srv, rid, buf.ctypes.data, n.value, ctypes.byref(n))
        if rc:
            raise WilsonError(rc, "wl_server_rows")
        return buf[: n.value]

    def cancel(self, rid: int) -> None:
        rc = self._L.wl_server_cancel(self._srv, rid)
        if rc:
            raise WilsonError(rc, "wl_server_cancel")

    def release(self, rid: int) -> None:
        rc = self._L.wl_server_release(self._srv, rid)
        if rc:
            raise WilsonError(rc, "wl_server_release")

    def stats(self) -> dict:
        st = _ServerStats()
        rc = self._L.wl_server_stats_get(self._srv, ctypes.byref(st))
        if rc:
            raise WilsonError(rc, "wl_server_stats_get")
        return {k: getattr(st, k) for k, _ in _ServerStats._fields_}
