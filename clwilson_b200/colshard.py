"""Column sharding: the sieving-prime interval of one range split between GPUs.

The reference runs a range on one device.  It sweeps the columns (sieving
primes q <= T, the class target) chunk by chunk and folds each chunk's
work-group partial products into the residues (cl_wilson.cpp:1856-1929,
reduce.cl:11-44).  Here the column interval [2, q_end) of one range is cut
into one piece per rank, at boundaries that balance the modelled cell count.

* Each rank computes its piece's per-row partial products with
  wl_rows_from, starting from 1.
* Rank 0 gathers the pieces and multiplies them row-wise on its GPU with
  wl_rows_product.
* Rank 0 then finishes the search from q_end with wl_search_from: no column
  is left, so only the tail, the class lift, the result lines and the
  checksum remain.

The rows, result lines and checksum are those of a one-GPU wl_search of the
range.  The pieces partition the columns, and products mod p^2 do not depend
on order.  The exchange is one gather of 16 bytes per row and rank.

Multiply-rows and finish run only on rank 0.  With the NCCL backend every rank
must have selected its CUDA device (torch.cuda.set_device) before the gather.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence

# share of test primes per class: p = 1 mod 3, p = 5 mod 12, p = 11 mod 12
CLASS_SHARE = (0.5, 0.25, 0.25)
# class target T = (p - 1) / k per class (cl_wilson.cpp:1549-1586)
CLASS_DIV = (6, 4, 2)


def column_end(pmax: int) -> int:
    """First column above every class target of a range below pmax.

    The largest target is (p - 1) / 2 of a class-2 prime p < pmax."""
    return (pmax - 2) // 2 + 1


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


def modelled_cells(pmin: int, q: float) -> float:
    """Modelled cells of the columns below q, per test prime of the range.

    Each class sweeps the primes up to its target, about li(min(q, T)) of
    them, weighted by its share of the test primes."""
    return sum(w * _li(min(q, (pmin - 1) / k)) for w, k in zip(CLASS_SHARE, CLASS_DIV))


def finish_cells(pmin: int, pmax: int) -> float:
    """Modelled cost of rank 0's finish per test prime, in cells: the
    consecutive-integer tail T_type+1 .. T_p of each row (iterate.cl), on
    average (pmax - pmin) / (2k) integers for class divisor k.  The finish
    also has a fixed cost (about 6.5 ms on B200: test primes, row setup, the
    row-wise product, the lift); it is left out of the model, which counts
    cells and not the column sieve, and would overrate it for ranges with
    few test primes."""
    width = pmax - pmin
    return sum(w * width / (2.0 * k) for w, k in zip(CLASS_SHARE, CLASS_DIV))


def column_pieces(pmin: int, pmax: int, world: int, rank0_extra: Optional[float] = None) -> List[int]:
    """Boundaries 2 = b_0 < b_1 < ... < b_m = column_end(pmax) of m <= world
    pieces [b_r, b_{r+1}).  Rank 0 also finishes the search, so its piece plus
    `rank0_extra` (cells per test prime; default finish_cells) and every other
    piece have about equal modelled cells.  m < world only when there are
    fewer columns than ranks."""
    if world < 1:
        raise ValueError("world must be >= 1")
    q_end = column_end(pmax)
    m = max(1, min(world, q_end - 2))
    total = modelled_cells(pmin, q_end)
    extra = 0.0 if m == 1 else (finish_cells(pmin, pmax) if rank0_extra is None else rank0_extra)
    each = (total + extra) / m
    bounds = [2]
    for r in range(1, m):
        goal = max(0.0, each * r - extra)
        lo, hi = bounds[-1] + 1, q_end - (m - r)
        # the first integer x in [lo, hi] with modelled_cells(x) >= goal
        a, b = lo, hi
        while a < b:
            mid = (a + b) // 2
            if modelled_cells(pmin, mid) >= goal:
                b = mid
            else:
                a = mid + 1
        bounds.append(a)
    bounds.append(q_end)
    return bounds


def search_piece(engine, pmin: int, pmax: int, bounds: Sequence[int], rank: int):
    """Rank `rank`'s partial products (rows), or None when it holds no piece."""
    if rank >= len(bounds) - 1:
        return None
    rows, _ = engine.rows_from(pmin, pmax, bounds[rank], bounds[rank + 1])
    return rows


def finish_pieces(engine, pmin: int, pmax: int, bounds: Sequence[int], parts: Sequence):
    """The search result from the pieces of all ranks (in rank order)."""
    held = [x for x in parts if x is not None]
    if len(held) != len(bounds) - 1:
        raise ValueError("finish_pieces: %d pieces for %d column intervals" % (len(held), len(bounds) - 1))
    init = engine.rows_product(held)
    return engine.search_from(pmin, pmax, bounds[-1], init=init)


def gather_to_rank0(obj, rank: int, world: int, group=None):
    """One object per rank, in rank order, on rank 0 (None elsewhere):
    torch.distributed.gather_object over `group`."""
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(obj, out, dst=0, group=group)
    return out


def search_columns_sharded(engine, pmin: int, pmax: int, rank: int = 0, world: int = 1, group=None,
                           gather: Optional[Callable] = None):
    """One range searched with its columns split over `world` ranks.

    Every rank calls this with its own engine (one GPU each).  Rank 0 returns
    the SearchResult; the other ranks return None.  `gather(obj)` collects
    one object per rank on rank 0 in rank order.  By default it is
    torch.distributed.gather_object over `group`."""
    bounds = column_pieces(pmin, pmax, world)
    part = search_piece(engine, pmin, pmax, bounds, rank)
    if world == 1:
        parts = [part]
    elif gather is not None:
        parts = gather(part)
    else:
        parts = gather_to_rank0(part, rank, world, group)
    if rank != 0:
        return None
    return finish_pieces(engine, pmin, pmax, bounds, parts)
