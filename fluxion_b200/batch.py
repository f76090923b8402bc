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


class BatchSolver:
    """Many independent steady convection-diffusion problems solved together on one GPU
    (fx_batch_*; new): -nu Lap u + v.grad u = f (first-order upwind, Dirichlet 0) on square grids of
    side 2^k + 1, each by right-preconditioned BiCGSTAB with the conv-diff V(2,2)-cycle, every
    phase one launch over the whole batch (see fx_batch.cu).  Batch vectors are F64 `CudaBuffer`s
    with every problem's grid one after the other (`offsets`)."""

    def __init__(self, device, grid_sides: Sequence[int], nu: float, vx, vy, cycle_dtype=None,
                 n_pre: int = 2, n_post: int = 2, omega: float = 0.8, coarse_max: int = 15,
                 coarse_sweeps: int = 200, sigma: float = 0.0, coeff: float = 1.0):
        import ctypes as C

        from . import _lib as L
        from .backend import check
        from .core import DType
        self._L, self._check, self._C = L, check, C
        self.device = device
        self.count = len(grid_sides)
        sides = (C.c_size_t * self.count)(*[int(s) for s in grid_sides])
        dt = DType.F64 if cycle_dtype is None else DType(cycle_dtype)
        self._keep = (vx, vy)
        out = C.c_void_p()
        check(L.lib().fx_batch_create(device.backend().ctx, self.count, sides, float(nu), float(sigma), float(coeff),
                                      vx.handle, vy.handle, int(dt), int(n_pre), int(n_post), float(omega),
                                      int(coarse_max), int(coarse_sweeps), C.byref(out)))
        self.h = out.value
        offs = (C.c_size_t * (self.count + 1))()
        lev = (C.c_size_t * self.count)()
        check(L.lib().fx_batch_layout(self.h, offs, lev))
        self.offsets = [offs[i] for i in range(self.count + 1)]
        self.depths = [lev[i] for i in range(self.count)]

    def set_chunk(self, elements: int) -> None:
        """Elements per flat work item of the batch's launches (no effect on the values)."""
        self._check(self._L.lib().fx_batch_set_chunk(self.h, int(elements)))

    def apply(self, v, out) -> None:
        self._check(self._L.lib().fx_batch_apply(self.h, v.handle, out.handle))

    def residual_norms(self, x, b):
        """||b_p - A x_p|| of every problem (computed on the device)."""
        out = (self._C.c_double * self.count)()
        self._check(self._L.lib().fx_batch_residual_norms(self.h, x.handle, b.handle, out))
        return [out[i] for i in range(self.count)]

    def precondition(self, z, r) -> None:
        self._check(self._L.lib().fx_batch_precondition(self.h, z.handle, r.handle))

    def bicgstab(self, x, b, rel_tol: float = 1e-10, max_iter: int = 200, use_graph: bool = True):
        """Solve every problem; returns (per-problem SolveStats, batch iterations launched)."""
        C = self._C
        from ._lib import FxStats
        from .solvers import _stats
        st = (FxStats * self.count)()
        run = C.c_size_t()
        self._check(self._L.lib().fx_batch_bicgstab(self.h, x.handle, b.handle, float(rel_tol), int(max_iter),
                                                    1 if use_graph else 0, st, C.byref(run)))
        return [_stats(st[i]) for i in range(self.count)], run.value

    def __del__(self):
        try:
            if self.h:
                self._L.lib().fx_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass
