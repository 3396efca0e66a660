"""One process per GPU: how the independent-per-s work is split over ranks.

The squaring, the deep scan and the serving work are independent per s (the
reference scans one s at a time, trinomial_scan.cu:648-689), so ranks take
disjoint s values and exchange nothing on the data path; the only
collectives are the barrier and small host-level reductions (max of the
timed region, gather of result lines).  The sieve shards by degree and has
one real exchange: the elementwise minimum of every rank's best[] (the
reference's multi-GPU merge, coarse_sieve.cu:466-507), one all-reduce of
8 (smax + 1) bytes.  The functions here hold that host logic so it can be
tested with `gloo` ranks on CPU.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


def rank_s_values(r: int, n: int, rank: int, seed: int = 1000) -> np.ndarray:
    """n seeded s values in [3, r/2) for one rank (each rank its own stream)."""
    rng = np.random.default_rng(seed + rank)
    return rng.integers(3, r // 2, size=n).astype(np.uint64)


def shard(items: Sequence, rank: int, world: int) -> list:
    """Round-robin share of `items` for `rank` (every item on exactly one rank)."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside 0..{world - 1}")
    return list(items)[rank::world]


def max_over_ranks(x: float, dist=None, device: Optional[str] = None) -> float:
    """Largest value of x over all ranks (x itself without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def scan_sharded(r: int, survivors: Sequence[int], k0: int, maxd: int, rank: int, world: int,
                 dist=None, scan_fn: Optional[Callable] = None, **kw) -> list:
    """Deep scan of `survivors` split over ranks; every rank returns all
    result lines in the order of `survivors` (gathered on the host)."""
    if scan_fn is None:
        from .engine import scan as scan_fn
    mine = shard(survivors, rank, world)
    lines = scan_fn(r, mine, k0, maxd, **kw) if mine else []
    if len(lines) != len(mine):
        raise RuntimeError(f"rank {rank}: {len(lines)} results for {len(mine)} s values")
    if dist is None or not dist.is_initialized() or world == 1:
        parts = [lines]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, lines)
    out = [None] * len(survivors)
    for rk, part in enumerate(parts):
        for j, line in enumerate(part):
            out[rk + j * world] = line
    if any(x is None for x in out):
        raise RuntimeError("missing results after gather")
    return out


def sieve_degrees(dmin: int, dmax: int, rank: int, world: int) -> list:
    """Degrees of [dmin, dmax] for `rank`: costs grow as 2^d, so degrees are
    dealt largest first to the least-loaded rank (every degree on exactly
    one rank)."""
    if not (0 <= rank < world):
        raise ValueError(f"rank {rank} outside 0..{world - 1}")
    load = [0] * world
    mine = {k: [] for k in range(world)}
    for d in range(dmax, dmin - 1, -1):
        k = min(range(world), key=lambda i: (load[i], i))
        load[k] += 1 << d
        mine[k].append(d)
    return sorted(mine[rank])


def _sieve_degrees_engine(r: int, degrees: Sequence[int], smax: int) -> np.ndarray:
    from .engine import run_sieve
    best = None
    for d in sorted(degrees):
        best = run_sieve(r, d, smax, dmin=d, preload=best)
    if best is None:
        best = np.full(smax + 1, np.uint64(0xFFFFFFFFFFFFFFFF), dtype=np.uint64)
    return best


def min_merge(best: np.ndarray, dist=None, device: Optional[str] = None) -> np.ndarray:
    """Elementwise minimum of every rank's best[] (all-ones = no factor)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return best
    import torch
    v = np.ascontiguousarray(best, dtype=np.uint64).view(np.int64).copy()
    none = v == -1                               # UINT64_MAX as int64
    v[none] = np.iinfo(np.int64).max             # keys are below 2^63
    t = torch.from_numpy(v).to(device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    out = t.cpu().numpy()
    out[out == np.iinfo(np.int64).max] = -1
    return out.view(np.uint64)


def sieve_sharded(r: int, dmin: int, dmax: int, smax: int, rank: int, world: int, dist=None,
                  sieve_fn: Optional[Callable] = None, device: Optional[str] = None) -> np.ndarray:
    """best[0..smax] for degrees dmin..dmax with the degrees split over ranks
    and the keys merged by minimum; every rank returns the full result."""
    fn = sieve_fn or _sieve_degrees_engine
    best = fn(r, sieve_degrees(dmin, dmax, rank, world), smax)
    return min_merge(best, dist, device)
