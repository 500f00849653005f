"""Cloth sharding across ranks (one process per GPU) for batched workloads.

Cloths are independent, so a batch splits by cloth with no exchange inside a step; each rank packs its own cloths into
its own context. The per-frame cost of a cloth is proportional to its constraint count (every pass reads each
constraint once and solves it), so shards are balanced by constraints: the longest-processing-time rule — cloths in
decreasing constraint count, each to the rank with the fewest constraints so far (lowest rank on ties).
"""
from __future__ import annotations

import heapq


def shard_by_constraints(constraint_counts, world: int) -> list[list[int]]:
    """Cloth indices per rank (each list ascending). Deterministic: every rank computes the same assignment."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(constraint_counts)), key=lambda k: (-int(constraint_counts[k]), k))
    heap = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        out[r].append(k)
        heapq.heappush(heap, (load + int(constraint_counts[k]), r))
    return [sorted(s) for s in out]
