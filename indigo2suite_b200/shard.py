"""Work split across GPUs for independent traversals.

One traversal does not shard (its frontier exchange would be a collective per
level); independent units do: the sources of a multi-source run, or the graphs
of a batch. Each rank takes a contiguous share of the units, runs them on its
own GPU, and only host-side bookkeeping crosses ranks: the per-rank timings
(max over ranks is the job time) and, when wanted, the gathered results.
`torch.distributed` carries that bookkeeping (NCCL on GPUs, gloo on CPUs).
"""
from __future__ import annotations

from typing import Callable, Sequence


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous share [lo, hi) of n units for `rank`; shares differ by at most one unit."""
    if world < 1 or not 0 <= rank < world or n < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def run_shard(units: Sequence, rank: int, world: int, run: Callable[[object], tuple[float, object]]):
    """Run this rank's share; `run(unit)` returns (seconds, result)."""
    lo, hi = shard_range(len(units), rank, world)
    secs, results = 0.0, []
    for u in units[lo:hi]:
        t, r = run(u)
        secs += t
        results.append(r)
    return secs, results


def max_over_ranks(x: float, world: int, device=None) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_results(results: list, world: int) -> list:
    """Concatenate every rank's results in rank order (the order of the units)."""
    if world == 1:
        return list(results)
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, results)
    return [r for p in parts for r in p]
