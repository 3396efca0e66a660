"""One process per GPU: how the independent-per-s work is split over ranks.

The squaring, the deep scan and the serving work are independent per s (the
reference scans one s at a time, trinomial_scan.cu:648-689), so ranks take
disjoint s values and exchange nothing on the data path; the only
collectives are the barrier and small host-level reductions (max of the
timed region, gather of result lines).  The functions here hold that host
logic so it can be tested with `gloo` ranks on CPU.
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
