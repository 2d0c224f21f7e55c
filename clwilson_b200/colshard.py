"""Column sharding: the sieving-prime interval of one range split between GPUs.

The reference runs a range on one device.  It sweeps the columns (sieving
primes q <= T, the class target) chunk by chunk and folds each chunk's
work-group partial products into the residues (cl_wilson.cpp:1856-1929,
reduce.cl:11-44).  Here the column interval [2, q_end) of one range is cut
into one piece per rank, at boundaries that balance the modelled work (cells
and column sieve; rank 0 is charged the finish it also runs).

* Each rank computes its piece's per-row partial products with
  wl_rows_from, starting from 1.
* Rank 0 gathers the pieces and multiplies them row-wise on its GPU with
  wl_rows_product.
* Rank 0 then finishes the search from q_end with wl_search_from: no column
  is left, so only the tail, the class lift, the result lines and the
  checksum remain.

The rows, result lines and checksum are those of a one-GPU wl_search of the
range.  The pieces partition the columns, and products mod p^2 do not depend
on order.  The exchange is one tensor gather of 16 bytes per row and rank,
after a 16-byte header that names the piece's column interval.

The row-wise product and the finish run only on rank 0.  Every rank uses
rank 0's piece boundaries (one broadcast), so the pieces partition the
columns however each rank would have planned them; rank 0 also checks every
gathered header against its boundaries and raises on a mismatch, which
covers a caller-supplied gather too.  With the NCCL backend every rank must
have selected its CUDA device (torch.cuda.set_device) before the collectives.

The consecutive-integer tail stays in rank 0's finish.  The planner charges
rank 0 for it (a smaller first piece), so the ranks' work is balanced with
the tail where it is.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence

import numpy as np

# share of test primes per class: p = 1 mod 3, p = 5 mod 12, p = 11 mod 12
CLASS_SHARE = (0.5, 0.25, 0.25)
# class target T = (p - 1) / k per class (cl_wilson.cpp:1549-1586)
CLASS_DIV = (6, 4, 2)
# ranges up to this width are planned from their actual test primes
EXACT_PLAN_WIDTH = 1 << 14

# Costs in cells of the sparse sweep (about 1.4e12 cells/s on B200):
# sieving the columns costs about 1.1e-12 s per integer below and above 2^32
# (the resident column sieve; the windowed sieve with its bitmap sweep), and
# the finishing call about 6.5 ms besides its tail (test primes, row setup,
# the row-wise product, the lift), both measured on B200.
SIEVE_CELLS_PER_INTEGER = 1.6
FINISH_FIXED_CELLS = 9.0e9


def column_end(pmax: int) -> int:
    """First column above every class target of a range below pmax.

    The largest target is (p - 1) / 2 of a class-2 prime p < pmax."""
    return (pmax - 2) // 2 + 1


def _is_prime(n: int) -> bool:
    """Miller-Rabin with the first 12 prime bases (exact below 3.3e24)."""
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for q in small:
        if n % q == 0:
            return n == q
    d, r = n - 1, 0
    while d % 2 == 0:
        d //= 2
        r += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(r - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def _class_of(p: int) -> int:
    return 0 if p % 3 == 1 else (1 if p % 12 == 5 else 2)


class RangeModel:
    """What the planner knows of a range: the number of test primes, each
    class's share of them and its shared target (the target of the class's
    first prime).  Exact for ranges up to EXACT_PLAN_WIDTH integers (host
    primality test; planning only, the engine finds the primes itself),
    otherwise the asymptotic shares with targets (pmin - 1) / k."""

    def __init__(self, pmin: int, pmax: int):
        self.pmin, self.pmax = pmin, pmax
        if pmax - pmin <= EXACT_PLAN_WIDTH:
            first = [0, 0, 0]
            count = [0, 0, 0]
            for p in range(max(pmin, 5), pmax):
                if _is_prime(p):
                    t = _class_of(p)
                    if not count[t]:
                        first[t] = p
                    count[t] += 1
            n = sum(count)
            self.rows = float(max(n, 1))
            self.share = tuple(c / max(n, 1) for c in count)
            self.targets = tuple((first[t] - 1) // CLASS_DIV[t] if count[t] else 0 for t in range(3))
        else:
            self.rows = max(1.0, (pmax - pmin) / math.log(max(pmin, 3)))
            self.share = CLASS_SHARE
            self.targets = tuple((pmin - 1) / k for k in CLASS_DIV)

    def cells(self, q: float) -> float:
        """Modelled cells per test prime of the columns below q: each class
        sweeps about li(min(q, T)) primes, weighted by its share."""
        return sum(w * _li(min(q, T)) for w, T in zip(self.share, self.targets) if w)

    def work(self, q: float) -> float:
        """Modelled cost of the columns below q, in cells: every test prime's
        cells plus the sieve of the integers up to the largest target."""
        sieved = max(0.0, min(q, max(self.targets)) - 2)
        return self.rows * self.cells(q) + SIEVE_CELLS_PER_INTEGER * sieved

    def finish(self) -> float:
        """Modelled cost of rank 0's finish, in cells: the consecutive-integer
        tail T_type+1 .. T_p of each row (iterate.cl), on average
        (pmax - pmin) / (2k) integers for class divisor k, plus the call's
        fixed cost."""
        width = self.pmax - self.pmin
        tail = sum(w * width / (2.0 * k) for w, k in zip(self.share, CLASS_DIV))
        return self.rows * tail + FINISH_FIXED_CELLS


def _li(x: float) -> float:
    """Integral of dq / ln q from 2 to x (Simpson's rule in u = ln q)."""
    if x <= 2.0:
        return 0.0
    a, b = math.log(2.0), math.log(x)
    m = 256
    h = (b - a) / m
    s = 0.0
    for i in range(m + 1):
        u = a + i * h
        w = 1 if i in (0, m) else (4 if i % 2 else 2)
        s += w * math.exp(u) / u
    return s * h / 3


def column_pieces(pmin: int, pmax: int, world: int, rank0_extra: Optional[float] = None,
                  model: Optional[RangeModel] = None) -> List[int]:
    """Boundaries 2 = b_0 < b_1 < ... < b_m = column_end(pmax) of m <= world
    pieces [b_r, b_{r+1}).  Rank 0 also finishes the search, so its piece plus
    `rank0_extra` (cells; default the model's finish) and every other piece
    have about equal modelled work; when the finish alone outweighs a piece,
    rank 0's piece is one column.  m < world only when there are fewer
    columns than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    model = model or RangeModel(pmin, pmax)
    q_end = column_end(pmax)
    m = max(1, min(world, q_end - 2))
    total = model.work(q_end)
    extra = 0.0 if m == 1 else (model.finish() if rank0_extra is None else rank0_extra)
    # rank 0's share; when the finish alone outweighs a piece, rank 0 keeps
    # one column and the other ranks share the rest equally
    first = max(0.0, (total + extra) / m - extra)
    other = (total - first) / (m - 1) if m > 1 else total
    bounds = [2]
    for r in range(1, m):
        goal = first + other * (r - 1)
        lo, hi = bounds[-1] + 1, q_end - (m - r)
        # the first integer x in [lo, hi] with work(x) >= goal
        a, b = lo, hi
        while a < b:
            mid = (a + b) // 2
            if model.work(mid) >= goal:
                b = mid
            else:
                a = mid + 1
        bounds.append(a)
    bounds.append(q_end)
    return bounds


def search_piece(engine, pmin: int, pmax: int, bounds: Sequence[int], rank: int):
    """Rank `rank`'s partial products (rows).  A rank beyond the last piece
    (a range with fewer columns than ranks) holds the empty product: every
    row's digits (1, 0), from a call with no column (q_cap = 2)."""
    if rank >= len(bounds) - 1:
        rows, _ = engine.rows_from(pmin, pmax, 2, 2)
        return rows
    rows, _ = engine.rows_from(pmin, pmax, bounds[rank], bounds[rank + 1])
    return rows


def piece_interval(bounds: Sequence[int], rank: int):
    """The column interval [lo, hi) of rank `rank`'s piece; (0, 0) for none."""
    return (bounds[rank], bounds[rank + 1]) if rank < len(bounds) - 1 else (0, 0)


def piece_digits(rows, interval=None):
    """What crosses to rank 0 for one piece, as an (n + 1, 2) uint64 array:
    the piece's column interval [lo, hi) in the first row, then the digits
    (s0, s1) of every row, 16 bytes each.  Without `interval`, the (n, 2)
    digits alone."""
    if rows is None:
        return None
    head = 0 if interval is None else 1
    out = np.empty((rows.size + head, 2), dtype=np.uint64)
    if head:
        out[0] = interval
    out[head:, 0] = rows["s0"]
    out[head:, 1] = rows["s1"]
    return out


def check_pieces(bounds: Sequence[int], parts: Sequence) -> List:
    """The digit arrays of gathered pieces after checking each header against
    rank 0's boundaries: piece r must cover [bounds[r], bounds[r + 1]), ranks
    beyond the last piece hold (0, 0).  Raises ValueError on a mismatch (pieces
    that overlap or leave a gap would give wrong quotients with no error)."""
    out = []
    for r, x in enumerate(parts):
        want = piece_interval(bounds, r)
        got = (int(x[0, 0]), int(x[0, 1]))
        if got != tuple(want):
            raise ValueError("column pieces disagree: rank %d swept [%d, %d), rank 0 planned [%d, %d)"
                             % (r, got[0], got[1], want[0], want[1]))
        if r < len(bounds) - 1:
            out.append(x[1:])
    return out


def finish_pieces(engine, pmin: int, pmax: int, bounds: Sequence[int], parts: Sequence, p=None):
    """The search result from the pieces of all ranks (in rank order): rows,
    or digit arrays with the primes `p` (or with one part as rows)."""
    held = [x for x in parts if x is not None]
    if len(held) != len(bounds) - 1:
        raise ValueError("finish_pieces: %d pieces for %d column intervals" % (len(held), len(bounds) - 1))
    init = engine.rows_product(held, p=p)
    return engine.search_from(pmin, pmax, bounds[-1], init=init)


def agree_on_bounds(bounds: List[int], rank: int, group=None) -> List[int]:
    """Rank 0's piece boundaries on every rank (torch.distributed broadcast)."""
    import torch.distributed as dist
    box = [list(bounds) if rank == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    return box[0]


def gather_to_rank0(arr, rank: int, world: int, group=None):
    """Every rank's (n + 1, 2) uint64 array, in rank order, on rank 0 (None
    elsewhere): one torch.distributed.gather of a tensor of 16 (n + 1) bytes
    per rank, on the GPU for the NCCL backend and on the CPU otherwise.  All
    ranks hold the same rows, so the shapes agree."""
    import torch
    import torch.distributed as dist
    on_gpu = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_gpu else torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(arr).view(np.int64)).to(dev)
    bufs = [torch.empty_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, bufs, dst=0, group=group)
    if rank != 0:
        return None
    return [b.cpu().numpy().view(np.uint64) for b in bufs]


def search_columns_sharded(engine, pmin: int, pmax: int, rank: int = 0, world: int = 1, group=None,
                           gather: Optional[Callable] = None):
    """One range searched with its columns split over `world` ranks.

    Every rank calls this with its own engine (one GPU each).  Rank 0 returns
    the SearchResult; the other ranks return None.  `gather(arr)` collects
    one array per rank on rank 0 in rank order.  By default it is a tensor
    gather over `group` (gather_to_rank0), and the boundaries are rank 0's,
    broadcast over `group`.  With a caller's gather each rank plans its own
    boundaries; rank 0 raises if any rank's piece differs from its plan."""
    bounds = column_pieces(pmin, pmax, world)
    if world > 1 and gather is None:
        bounds = agree_on_bounds(bounds, rank, group)
    part = search_piece(engine, pmin, pmax, bounds, rank)
    if world == 1:
        return finish_pieces(engine, pmin, pmax, bounds, [part])
    mine = piece_digits(part, piece_interval(bounds, rank))
    parts = gather(mine) if gather is not None else gather_to_rank0(mine, rank, world, group)
    if rank != 0:
        return None
    # rank 0 always holds the first piece, whose rows carry the primes
    return finish_pieces(engine, pmin, pmax, bounds, check_pieces(bounds, parts), p=part["p"])
