"""Splitting a batch of independent problems across ranks (one process per GPU).

The batched convection-diffusion workload is a set of independent solves, so it shards with no
data-path communication: each rank solves its own share, and one collective at the end brings the
per-problem results to rank 0.  The reference is single-device (crates/backend-hip/src/backend.rs:112,
hipSetDevice(0)); this is the library's own multi-GPU layer for the batch.

- `partition_by_points`: longest-processing-time-first assignment of problems to ranks by their
  point counts (deterministic: ties break by problem index, then by rank), which bounds every
  rank's load by the average plus the largest problem.
- `gather_results`: one `all_gather_object` of each rank's (problem index, result) pairs; every
  rank returns the results in problem order.
"""
from __future__ import annotations

import heapq
from typing import Any, Dict, List, Sequence, Tuple


def partition_by_points(points: Sequence[int], world: int) -> List[List[int]]:
    """Problem indices per rank, each list in ascending order."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    order = sorted(range(len(points)), key=lambda i: (-int(points[i]), i))
    heap: List[Tuple[int, int]] = [(0, r) for r in range(world)]  # (load, rank)
    heapq.heapify(heap)
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(points[i]), r))
    return [sorted(p) for p in parts]


def loads(points: Sequence[int], parts: Sequence[Sequence[int]]) -> List[int]:
    return [sum(int(points[i]) for i in p) for p in parts]


def gather_results(local: Dict[int, Any], n_problems: int, group=None) -> List[Any]:
    """All ranks' {problem index: result} merged in problem order (one collective).  Raises if a
    problem is missing or was solved twice."""
    import torch.distributed as dist

    world = dist.get_world_size(group)
    gathered: List[Any] = [None] * world
    dist.all_gather_object(gathered, sorted(local.items()), group=group)
    out: List[Any] = [None] * n_problems
    seen = [False] * n_problems
    for part in gathered:
        for i, res in part:
            if seen[i]:
                raise RuntimeError(f"problem {i} was solved on two ranks")
            seen[i] = True
            out[i] = res
    missing = [i for i, s in enumerate(seen) if not s]
    if missing:
        raise RuntimeError(f"problems without a result: {missing[:8]}")
    return out
