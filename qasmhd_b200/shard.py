"""Sharding of a batched ensemble over ranks (one process per GPU).

Instances are independent, so the ensemble partitions with no collective in the
data path: each rank steps its own shard with one qas_batch; only the final
per-rank metrics are gathered.  The partition is a greedy longest-processing-
time balance on interior cell counts (work per step is proportional to cells).
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def partition(cells: Sequence[int], world: int) -> List[List[int]]:
    """Indices of the instances each rank owns; largest first onto the least loaded rank.
    Ties go to the lower rank, so the result is deterministic on every rank."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(cells)), key=lambda q: (-cells[q], q))
    heap = [(0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for q in order:
        load, r = heapq.heappop(heap)
        out[r].append(q)
        heapq.heappush(heap, (load + cells[q], r))
    for r in range(world):
        out[r].sort()
    return out


def imbalance(cells: Sequence[int], parts: List[List[int]]) -> float:
    """max rank load / mean rank load (1.0 = perfect)."""
    loads = [sum(cells[q] for q in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


def run_shard(probs, rank: int, world: int, steps: int, device: int = -1):
    """Advance this rank's shard of the ensemble `steps` steps on its GPU; returns
    (instance indices, list of (steps, tim, dt))."""
    from . import lib
    parts = partition([p.interior_cells for p in probs], world)
    mine = parts[rank]
    if not mine:
        return mine, []
    with lib.Batch([probs[q] for q in mine], device=device) as b:
        for k, q in enumerate(mine):
            b.upload(k, probs[q].state)
        info = b.run(max_steps=steps, flg=1, stop_rule=0, cfl=0.4)
    return mine, info
