"""Splitting independent hafnians across GPUs (one process per GPU).

The hot paths shard only by instance: every hafnian of a batch is independent, so N GPUs run N
replicas with no data-path collective.  Instances differ widely in cost (a degree-32 DP is ~8x a
degree-28 one; a sieve's cost is its term count times the term size), so contiguous splits would
leave ranks idle.  `balanced_shards` assigns instances to ranks by longest-processing-time-first on
a cost estimate, deterministically, so every rank computes the same assignment without
communicating.
"""
from __future__ import annotations

import heapq

from . import policy as pol
from . import roofline as R


def dp_cost(N: int) -> float:
    """Transitions of the degree-N plan (the DP's work per instance)."""
    return float(pol._dp_counts(N)[1])


def sieve_cost(edge_reps, glynn: bool, cplx: bool = False) -> float:
    """Algorithmic flops of one sieve (roofline.sieve_flops)."""
    return R.sieve_flops(edge_reps, glynn, cplx)


def shard_range(n: int, world: int, rank: int) -> range:
    """Contiguous, near-equal split of range(n) (for equal-cost instances)."""
    lo = (rank * n) // world
    hi = ((rank + 1) * n) // world
    return range(lo, hi)


def balanced_shards(costs, world: int) -> list[list[int]]:
    """Instances per rank, largest first onto the least-loaded rank; ties by index, so the result
    is the same on every rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in out]
