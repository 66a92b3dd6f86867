"""Splitting one list of independent read sets over several GPUs.

Read sets are independent jobs (each is one extend_graph over its reads,
src/lib.rs:184-204), so a batch shards across devices with no exchange on
the data path: every rank aligns its share on its own GPU and the results
are gathered on the host. Shares are balanced by estimated work with the
longest-processing-time greedy rule: sets in decreasing order of estimated
band cells, each to the rank with the least work so far (ties to the lower
rank). The split is deterministic, so every rank computes the same one
without communicating.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def set_work(reads: Sequence[bytes], b: int = 100, f: int = 40) -> float:
    """Estimated band cells of aligning one read set with static band b + m/f:
    reads x rows (growing with the reads fused) x band width."""
    if not reads:
        return 0.0
    L = max(len(r) for r in reads)
    w = min(2.0 * (b + (L / f if f else L)) + 16.0, L + 16.0)
    return sum(len(r) for r in reads) * w * (1.0 + 0.03 * len(reads))


def partition(works: Sequence[float], n_ranks: int) -> List[List[int]]:
    """Indices of the sets each rank runs (each list in increasing index
    order, so outputs gather back in set order)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be positive")
    order = sorted(range(len(works)), key=lambda s: (-works[s], s))
    heap = [(0.0, r) for r in range(n_ranks)]
    heapq.heapify(heap)
    shares: List[List[int]] = [[] for _ in range(n_ranks)]
    for s in order:
        load, r = heapq.heappop(heap)
        shares[r].append(s)
        heapq.heappush(heap, (load + works[s], r))
    return [sorted(x) for x in shares]


def gather(n_sets: int, shares: List[List[int]], per_rank: List[List[object]]) -> List[object]:
    """Per-set results back in set order from each rank's results (in the
    order of its share)."""
    out: List[object] = [None] * n_sets
    for idx, res in zip(shares, per_rank):
        if len(idx) != len(res):
            raise ValueError("a rank returned a different number of results than its share")
        for s, x in zip(idx, res):
            out[s] = x
    return out
