"""Autotuning of the library's free launch and algorithm parameters, with a JSON cache (new; the
reference has no tuner).

- `tune_vertex_mg`: the fused Poisson V-cycle's layout (row chunks per launch, first tail level),
  via fx_mg_autotune; every candidate computes the same values.
- `tune_batch`: the batched convection-diffusion solver's work-item size (elements per chunk),
  smoothing sweep counts (n_pre = n_post) and cycle precision, by timing whole BiCGSTAB solves of a
  sample of the batch.  Sweep counts and precision change the iterations, so a candidate counts
  only if every sampled problem converges to the requested tolerance on its true residual; the
  fastest such candidate wins.

A `TuneCache` keeps results in a JSON file keyed by what the choice depends on (kind, sizes,
parameters, device name), so a second run with the same key reads the choice instead of timing.
"""
from __future__ import annotations

import json
import os
import tempfile
from typing import Dict, Optional, Sequence

import numpy as np


class TuneCache:
    """A JSON file of {key: choice}; keys are canonical JSON strings of dicts."""

    def __init__(self, path: Optional[str] = None):
        self.path = path
        self.data: Dict[str, dict] = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.data = json.load(f)

    @staticmethod
    def key(**kw) -> str:
        return json.dumps(kw, sort_keys=True)

    def get(self, key: str) -> Optional[dict]:
        return self.data.get(key)

    def put(self, key: str, value: dict) -> None:
        self.data[key] = value
        if not self.path:
            return
        d = os.path.dirname(os.path.abspath(self.path))
        os.makedirs(d, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=d, suffix=".json")
        with os.fdopen(fd, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def device_name(device) -> str:
    import torch
    return torch.cuda.get_device_properties(device.ordinal).name


def tune_vertex_mg(mg, z, r, cache: Optional[TuneCache] = None, reps: int = 5, **key_extra) -> dict:
    """Apply the cached or measured layout of a fused vertex multigrid; returns the choice.
    key_extra: what else the choice depends on (dtype, coarse_max, coarse_sweeps, ...)."""
    cache = cache or TuneCache()
    g = mg.grid
    key = TuneCache.key(kind="vertex_mg", rows=g.rows, cols=g.cols, device=device_name(mg.device), **key_extra)
    hit = cache.get(key)
    if hit is not None:
        mg.set_tuning(int(hit["chunk_pct"]), int(hit["tail_top_points"]))
        return dict(hit, cached=True)
    best = mg.autotune(z, r, reps=reps)
    cache.put(key, {"chunk_pct": best["chunk_pct"], "tail_top_points": best["tail_top_points"], "ms": best["ms"]})
    return dict(best, cached=False)


def _sample(sides: Sequence[int], n: int, seed: int = 0) -> list:
    """Up to n problem indices keeping the batch's mix of sizes (round-robin over the sizes)."""
    by = {}
    for i, s in enumerate(sides):
        by.setdefault(int(s), []).append(i)
    rng = np.random.default_rng(seed)
    for v in by.values():
        rng.shuffle(v)
    out, k = [], 0
    keys = sorted(by)
    while len(out) < min(n, len(sides)):
        for s in keys:
            if k < len(by[s]) and len(out) < n:
                out.append(by[s][k])
        k += 1
    return sorted(out)


def tune_batch(device, sides: Sequence[int], nu: float, vx: Sequence[np.ndarray], vy: Sequence[np.ndarray],
               f: Sequence[np.ndarray], rel_tol: float = 1e-10, sample: int = 96,
               chunks=(1024, 2048, 4096), sweeps=(1, 2, 3), dtypes=("f64", "f32"), omega: float = 0.8,
               coarse_max: int = 15, coarse_sweeps: int = 200, cache: Optional[TuneCache] = None) -> dict:
    """Choose (chunk, sweeps, cycle dtype) for the batched solver from timed solves of a sample of the
    batch (per-problem host arrays vx, vy, f).  Returns {"chunk", "sweeps", "cycle_dtype", "ms",
    "candidates": [...], "cached"}."""
    import torch
    from .batch import BatchSolver
    from .core import DType
    cache = cache or TuneCache()
    idx = _sample(sides, sample)
    hist = {str(s): int(sum(1 for i in idx if sides[i] == s)) for s in sorted(set(int(sides[i]) for i in idx))}
    key = TuneCache.key(kind="batch_convdiff", nu=nu, tol=rel_tol, sample_sizes=hist, omega=omega,
                        coarse_max=coarse_max, coarse_sweeps=coarse_sweeps, device=device_name(device),
                        space=[list(chunks), list(sweeps), list(dtypes)])
    hit = cache.get(key)
    if hit is not None:
        return dict(hit, cached=True)
    be = device.backend()
    s_sides = [int(sides[i]) for i in idx]
    VX = be.upload_f64(np.concatenate([vx[i] for i in idx]))
    VY = be.upload_f64(np.concatenate([vy[i] for i in idx]))
    F = be.upload_f64(np.concatenate([f[i] for i in idx]))
    fnorm = [float(np.linalg.norm(f[i])) for i in idx]
    sp = be.stream()  # the library's stream: the events must be recorded where its kernels run
    stream = torch.cuda.ExternalStream(sp) if sp else torch.cuda.current_stream()
    cands = []
    for dt in dtypes:
        for sw in sweeps:
            B = BatchSolver(device, s_sides, nu, VX, VY, cycle_dtype=DType.F32 if dt == "f32" else DType.F64,
                            n_pre=sw, n_post=sw, omega=omega, coarse_max=coarse_max, coarse_sweeps=coarse_sweeps)
            for ch in chunks:
                B.set_chunk(int(ch))
                X = be.allocate(B.offsets[-1], DType.F64)
                B.bicgstab(X, F, rel_tol, 300)  # records the iteration graph
                be.fill(X, 0.0)
                be.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                stats, _ = B.bicgstab(X, F, rel_tol, 300)
                e1.record(stream)
                torch.cuda.synchronize()
                rn = B.residual_norms(X, F)
                ok = all(s.converged() for s in stats) and all(r <= 1.01 * rel_tol * fn for r, fn in zip(rn, fnorm))
                cands.append({"chunk": int(ch), "sweeps": int(sw), "cycle_dtype": dt, "ms": e0.elapsed_time(e1),
                              "ok": bool(ok), "iterations_max": int(max(s.iterations for s in stats))})
            del B
    good = [c for c in cands if c["ok"]]
    if not good:
        raise RuntimeError("batch autotune: no candidate converged on the sample")
    best = min(good, key=lambda c: c["ms"])
    out = {"chunk": best["chunk"], "sweeps": best["sweeps"], "cycle_dtype": best["cycle_dtype"], "ms": best["ms"],
           "sample": len(idx), "candidates": cands}
    cache.put(key, out)
    return dict(out, cached=False)
