#!/usr/bin/env python
"""Benchmark: time to relative residual 1e-10 for the 4095^2 Poisson solve on one B200.

Workload (one "step"): -Lap u = f on the unit square, 4095 x 4095 interior nodes (4097^2 grid
with the Dirichlet ring), f = 32 seeded sin-sin modes (k, l in 1..64, N(0,1) amplitudes) plus
1e-3 * U[-1,1] noise, u0 = 0, CG preconditioned by one V(2,2)-cycle per iteration (full
weighting, bilinear prolongation, weighted Jacobi omega = 0.8, coarsest 15^2 with 200 sweeps)
to ||r|| < 1e-10 ||f|| (verified in FP64 against the plain operator and against the exact
DST-I solve).  `value` and `e2e` are the plain FP64 solve, the same arithmetic as the reference
arm; the mixed solve (FP64 CG, residual, update and inner products; FP32 V-cycle) and the other
variants are reported beside it under their own keys.

Also reported: e2e time through the public API with the source and the solution in pinned host
memory; the live roofline of the dominant kernel (CUDA events on its launching stream over the
timed region); stencil / AXPY / dual-dot microbenchmarks on a 16384^2 grid; the CPU oracle on
the host cores; SM clocks sampled during the timed region; the number of our kernel launches.

`--impl reference` times the reference algorithm's CPU restatement (the oracle: the reference
itself is Rust and cannot be built here) on all host cores, on a bounded sample of the same
workload.  Under torchrun (N > 1) every rank solves its own replica (no data-path exchange).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time to rel-resid 1e-10: learned/mixed vs plain (1 B200); stencil GB/s"
N_INTERIOR = 4095
SEED = 2024
# V(2,2)-cycle parameters of the configuration: weighted Jacobi 0.8, coarsen while the interior
# exceeds 15 x 15, 200 Jacobi sweeps on the coarsest grid
OMEGA = 0.8
COARSE_MAX = 15
COARSE_SWEEPS = 200
SOLVER = (f"V(2,2) full weighting / bilinear / weighted Jacobi {OMEGA}, coarsest interior <= "
          f"{COARSE_MAX}^2 x {COARSE_SWEEPS} sweeps")

# algorithmic bytes per grid point of each kernel (F64 sizes; F32 kernels carry a _f32 tag)
BYTES_PER_POINT = {
    "mg_sweep": 3, "mg_residual": 3, "mg_prolong_bilinear": 2.25, "mg_restrict_fw": 5, "mg_zero": 1,
    "pcg_dir": 3, "pcg_update": 5, "pcg_rz": 2, "pcg_init": 3,
}
# element-size multiplier is applied per dtype: F64 -> 8 bytes, F32 -> 4 bytes (see roofline())


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--n", type=int, default=N_INTERIOR, help="interior nodes per direction")
    p.add_argument("--no-micro", action="store_true")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--batch", type=int, default=1024, help="problems in --mode batch")
    p.add_argument("--lanes", type=int, default=8, help="--mode batch: concurrent contexts (host threads)")
    p.add_argument("--pdl", type=int, default=1, choices=[0, 1],
                   help="--mode batch: programmatic dependent launch in the lanes' contexts")
    p.add_argument("--autotune", action="store_true",
                   help="--mode vcycle: autotune the cycle's layout first; --mode batch: choose the batched "
                        "solver's chunk size, sweep counts and cycle precision first (timed on a sample)")
    p.add_argument("--tune-cache", default=None, help="JSON file that keeps autotuner choices between runs")
    p.add_argument("--mode", default="solve", choices=["solve", "vcycle", "batch", "convdiff", "learned", "lsm_step", "micro"],
                   help="solve: the headline MG-PCG solve; vcycle: preconditioner applications alone "
                        "(the F32 V(2,2)-cycle on FP64 vectors), e.g. as a profiling target; batch: "
                        "1024 conv-diff problems; convdiff: convection-dominated conv-diff at --n; "
                        "learned: train the learned smoother, then FGMRES(30) with the learned vs the plain "
                        "conv-diff cycle at --n; lsm_step: learned smoothing steps alone at --n (a profiling "
                        "target of the network kernel); micro: the stencil / AXPY / dual-dot microbenchmarks "
                        "alone on an --n x --n grid")
    p.add_argument("--nu", default="1e-3,1e-4", help="--mode convdiff: viscosities, comma-separated")
    p.add_argument("--k-range", default="6,10",
                   help="--mode batch: interior sizes 2^k - 1 for k uniform in this inclusive range")
    p.add_argument("--replay", type=int, default=0, choices=[0, 1],
                   help="--mode batch: record each hierarchy's cycle into a CUDA graph and replay it")
    p.add_argument("--pipeline", type=int, default=2,
                   help="--mode batch --batched 1: sub-batches (balanced by points) whose uploads, solves and "
                        "read-backs overlap (1: upload all, solve all, read back all)")
    p.add_argument("--batched", type=int, default=1, choices=[0, 1],
                   help="--mode batch: 1 = the batched solver (every phase one launch over all problems, "
                        "graph-replayed iterations); 0 = independent solves on --lanes host threads")
    p.add_argument("--mg-dtype", default="f64", choices=["f64", "f32"],
                   help="--mode batch / vcycle: arithmetic of the V-cycle (the Krylov solver stays FP64)")
    return p.parse_args()


NOMINAL_HBM_GBS = 7700.0  # B200 HBM3e, the nominal (HGX) figure, reported beside the measured one


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ clocks

_CLOCK_POLL = r"""
import sys, time
import pynvml
pynvml.nvmlInit()
sel, period = sys.argv[1], float(sys.argv[2])
h = pynvml.nvmlDeviceGetHandleByUUID(sel) if sel.startswith("GPU-") else pynvml.nvmlDeviceGetHandleByIndex(int(sel))
get = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
print("ready", pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM), flush=True)
while True:
    print(time.time(), pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), get(h), flush=True)
    time.sleep(period)
"""


class ClockSampler:
    """SM clock and clock-event reasons sampled every ~1 ms through NVML, in a separate process
    (so the launch loop's interpreter lock cannot starve it), while the timed region runs; a solve
    takes a few ms, far below nvidia-smi's sampling interval.  Reads settings only, changes none."""

    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, gpu_index: int, uuid: str = "", period_s: float = 0.001):
        self.sel = (uuid if uuid.startswith("GPU-") else "GPU-" + uuid) if uuid else str(gpu_index)
        self.period = period_s
        self.samples = []  # (time, sm_mhz, reasons bitmask), every sample the poller sent
        self.max_mhz = None
        self.proc = None
        self.t = None
        self.ready = threading.Event()
        self.window = (0.0, 0.0)  # the timed region, on the poller's clock (time.time())

    def __enter__(self):
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", _CLOCK_POLL, self.sel, str(self.period)],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            self.ready.wait(timeout=30)
        except Exception:
            self.proc = None
        self.window = (time.time(), 0.0)
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = line.split()
            if not parts:
                continue
            if parts[0] == "ready":
                self.max_mhz = float(parts[1])
                self.ready.set()
            elif len(parts) == 3:
                self.samples.append((float(parts[0]), float(parts[1]), int(parts[2])))
        self.ready.set()  # the poller exited (e.g. no NVML): do not wait for it

    def __exit__(self, *a):
        self.window = (self.window[0], time.time())
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            if self.t is not None:
                self.t.join(timeout=5)  # drain what the poller sent before it stopped

    def summary(self):
        t0, t1 = self.window
        inside = [(m, bits) for t, m, bits in self.samples if t0 <= t <= t1]
        sm = [m for m, _ in inside]
        reasons = sorted({nm for _, bits in inside for nm, bit in self.REASONS.items() if bits & bit})
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "source": "nvml"}


# ------------------------------------------------------------------ CPU oracle timing

def oracle_solve(n: int, f: np.ndarray):
    """One full MG-PCG solve of the n^2 problem by the oracle (the same algorithm and parameters
    as the GPU solve, FP64 throughout) on all host threads: (seconds, iterations, threads)."""
    from oracle import oracle as O
    from fluxion_b200.workloads import poisson_problem

    O.set_threads(os.cpu_count() or 1)
    P = poisson_problem(n)
    N = n + 2
    mg = O.Multigrid(N, N, P.h, P.h, 2, 2, OMEGA, mode=1, op_coeff=1.0, entries=P.stencil.as_triples(),
                     coarse_max=COARSE_MAX, coarse_sweeps=COARSE_SWEEPS)
    tol = 1e-10 * float(np.linalg.norm(f))
    x = np.zeros(N * N)
    t0 = time.perf_counter()
    iters, _, _ = O.cg_solve(x, f, N, N, 1.0, P.stencil.as_triples(), tol, 200, pc=mg)
    return time.perf_counter() - t0, int(iters), O.get_threads()


def headline_config(n: int, world: int) -> dict:
    """The `config` both arms print for the headline solve: identical keys and strings."""
    N = n + 2
    return {"workload": f"poisson_{n}sq_mg_pcg_rel1e-10", "grid": f"{N}x{N} incl. Dirichlet ring",
            "solver": f"CG + {SOLVER}", "precision": "fp64 throughout",
            "tolerance": "||r||_2 < 1e-10 ||f||_2", "coarse": f"{COARSE_MAX}^2 interior x {COARSE_SWEEPS} sweeps",
            "rhs": "32 sin-sin modes, k,l in 1..64, N(0,1) amplitudes, + 1e-3 U[-1,1] noise", "seed": SEED,
            "l2": "inputs larger than L2 (134 MB per vector)",
            "parallelism": "replicas" if world > 1 else "single device"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from fluxion_b200.workloads import poisson_modes_rhs

    n = args.n
    N = n + 2
    f = poisson_modes_rhs(n, SEED)
    samples, iters, threads = [], 0, 1
    for step in range(args.warmup + args.steps):
        t, iters, threads = oracle_solve(n, f)
        if step >= args.warmup:
            samples.append(t)
    v = float(np.mean(samples))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(n, int(os.environ.get("WORLD_SIZE", "1"))),
        "iterations": iters,
        "cpu_baseline": {"value": v, "unit": "s", "cores": threads, "kind": "port",
                         "sample": f"per step: one full {n}^2 MG-PCG solve to 1e-10 ({iters} iterations)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference is Rust (no cargo/rustc here); its CPU backend is timed as the C restatement",
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ our arm

def run_vcycle(args):
    """Time `steps` applications z = M^-1 r of the V(2,2)-cycle in `--mg-dtype` (after `warmup` untimed ones)
    on the n^2 problem, and report each level kernel's device time from the timing records."""
    import ctypes as C

    import torch
    from fluxion_b200 import DType, Device, Field, Multigrid
    from fluxion_b200 import _lib as L
    from fluxion_b200.workloads import poisson_modes_rhs, poisson_problem

    n = args.n
    dev = Device.Cuda(0)
    be = dev.backend()
    stream = torch.cuda.Stream()
    be.set_stream(stream.cuda_stream)
    P = poisson_problem(n)
    r = Field.from_f64(P.grid, poisson_modes_rhs(n, SEED), dev)
    z = Field.zeros(P.grid, DType.F64, dev)
    mg = Multigrid.vertex(P.grid, None, dev, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS,
                          DType.F32 if args.mg_dtype == "f32" else DType.F64)
    tuned = mg.autotune(z, r, reps=max(3, args.steps)) if args.autotune else None
    for _ in range(args.warmup):
        mg.precondition(z, r)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        mg.precondition(z, r)
    e1.record(stream)
    torch.cuda.synchronize()
    per = {}
    for k in ("mg_down", "mg_up", "mg_tail"):
        L.lib().fx_ctx_timing_begin(be.ctx, k.encode())
        mg.precondition(z, r)
        cap = 64
        ms, pts, byt, cnt = (C.c_double * cap)(), (C.c_double * cap)(), (C.c_double * cap)(), C.c_size_t()
        L.lib().fx_ctx_timing_end_records(be.ctx, ms, pts, byt, cap, C.byref(cnt))
        per[k] = [{"points": pts[i], "us": ms[i] * 1e3, "GBps": byt[i] / (ms[i] * 1e-3) / 1e9 if byt[i] else None}
                  for i in range(cnt.value)]
    print(json.dumps({"mode": "vcycle", "workload": f"poisson_{n}sq_{args.mg_dtype}_vcycle", "steps": args.steps,
                      "warmup": args.warmup, "ms_per_vcycle": e0.elapsed_time(e1) / args.steps,
                      "levels": mg.depth(), "autotune": tuned, "per_launch_with_events": per}), flush=True)
    return 0


LSM_FLOPS_PER_POINT = 2 * (3 * 16 * 9 + 16 * 16 * 9 + 16 * 9)  # the network's MACs x 2, halos not counted


def run_lsm_step(args):
    """Time `steps` learned smoothing steps (the q / scale pass and the network with the update) on the
    n^2 conv-diff problem after `warmup` untimed ones, with CUDA events on the library's stream, and
    report the network pass's device time and its tensor roofline (5760 flop per point)."""
    import ctypes as C

    import torch
    from fluxion_b200 import ConvDiffOperator, DType, Device, Field, Grid
    from fluxion_b200 import _lib as L
    from fluxion_b200.learned import LearnedSmoother
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity

    n = args.n
    dev = Device.Cuda(0)
    be = dev.backend()
    stream = torch.cuda.Stream()
    be.set_stream(stream.cuda_stream)
    N, h = n + 2, 1.0 / (n + 1)
    g = Grid.square(N, h)
    vx, vy = stream_velocity(n, SEED + 3)
    f = poisson_uniform_rhs(n, SEED + 4)
    op = ConvDiffOperator(g, Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev), -1e-3, sigma=0.0, coeff=1.0)
    lsm = LearnedSmoother(dev, seed=1)
    p = lsm.params
    p[-145:-1] = np.random.default_rng(SEED).normal(0.0, 0.2, 144)  # a non-zero last layer
    lsm.params = p
    x = Field.zeros(g, DType.F64, dev)
    b = Field.from_f64(g, f, dev)
    lsm.smooth(op, x, b, OMEGA, max(1, args.warmup))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    lsm.smooth(op, x, b, OMEGA, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    step_ms = e0.elapsed_time(e1) / args.steps
    L.lib().fx_ctx_timing_begin(be.ctx, b"lsm_apply")
    lsm.smooth(op, x, b, OMEGA, 3)
    cap = 8
    ms, pts, byt, cnt = (C.c_double * cap)(), (C.c_double * cap)(), (C.c_double * cap)(), C.c_size_t()
    L.lib().fx_ctx_timing_end_records(be.ctx, ms, pts, byt, cap, C.byref(cnt))
    apply_ms = float(np.mean([ms[i] for i in range(cnt.value)])) if cnt.value else None
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = float(json.load(fh)["bf16_tflops"])
    except Exception:
        peak = 1590.0
    flops = LSM_FLOPS_PER_POINT * float(n) * float(n)
    tf = flops / (apply_ms * 1e-3) / 1e12 if apply_ms else None
    print(json.dumps({"mode": "lsm_step", "workload": f"learned_smoother_step_{n}sq", "steps": args.steps,
                      "warmup": args.warmup, "ms_per_step": step_ms, "network_pass_ms": apply_ms,
                      "roofline": {"kernel": "k_lsm_apply", "bound": "tensor", "achieved": tf, "peak": peak,
                                   "unit": "TFLOP/s", "frac": tf / peak if tf else None,
                                   "flops_per_point": LSM_FLOPS_PER_POINT}}), flush=True)
    return 0


def run_batch_batched(args, ks, mine, host, world, rank, local_rank, dist):
    """The batch through the batched solver, as a pipeline of --pipeline sub-batches (balanced by
    points): the first sub-batch's f, vx and vy are uploaded from page-locked host memory on a
    copy stream, the others' once the first is built (its small table copies would otherwise
    queue behind them on the copy engine); sub-batch k is built (hierarchies and work tables) and solved by
    BiCGSTAB with the conv-diff V-cycle (every phase one launch over the sub-batch, each
    iteration replayed from a CUDA graph) once its upload has landed, while the later uploads
    continue; its true residuals are computed on the device and its solutions read back on a
    second copy stream while sub-batch k + 1 solves.  All of it is timed; the host data
    generation is not."""
    import torch
    from fluxion_b200 import DType, Device
    from fluxion_b200.batch import BatchSolver, partition_by_points

    dev = Device.Cuda(local_rank)
    be = dev.backend()
    stream = torch.cuda.Stream()
    be.set_stream(stream.cuda_stream)
    nu = 1e-2
    sides = [int(2 ** ks[i] + 1) for i in mine]
    nsub = max(1, min(int(args.pipeline), len(sides)))
    parts = [p_ for p_ in partition_by_points([s_ * s_ for s_ in sides], nsub) if p_]
    subs = []  # (local indices, sides, f, vx, vy, out) per sub-batch, host arrays page-locked
    for part in parts:
        sd = [sides[j] for j in part]
        tot = sum(s_ * s_ for s_ in sd)
        pin = torch.empty(4 * tot, dtype=torch.float64, pin_memory=True).numpy()
        fv, xv, yv, out = pin[:tot], pin[tot:2 * tot], pin[2 * tot:3 * tot], pin[3 * tot:]
        o = 0
        for j, s_ in zip(part, sd):
            _, vx, vy, f, _ = host[mine[j]]
            fv[o:o + s_ * s_], xv[o:o + s_ * s_], yv[o:o + s_ * s_] = f, vx, vy
            o += s_ * s_
        subs.append((part, sd, fv, xv, yv, out))
    mg_dtype = DType.F32 if args.mg_dtype == "f32" else DType.F64
    chunk, sweeps, tuned = 2048, 2, None
    if args.autotune:  # before the timed region: work-item size, sweep counts and cycle precision
        from fluxion_b200.autotune import TuneCache, tune_batch
        t_tune = time.perf_counter()
        tuned = tune_batch(dev, sides, nu, [host[i][1] for i in mine], [host[i][2] for i in mine],
                           [host[i][3] for i in mine], sample=96, omega=OMEGA, coarse_max=COARSE_MAX,
                           coarse_sweeps=COARSE_SWEEPS, cache=TuneCache(args.tune_cache))
        tuned["tuning_s"] = time.perf_counter() - t_tune
        chunk, sweeps = tuned["chunk"], tuned["sweeps"]
        mg_dtype = DType.F32 if tuned["cycle_dtype"] == "f32" else DType.F64
    up, down = torch.cuda.Stream(), torch.cuda.Stream()

    def once():
        bufs = []
        for (_, sd, _, _, _, _) in subs:
            tot = sum(s_ * s_ for s_ in sd)
            bufs.append(tuple(be.allocate(tot, DType.F64) for _ in range(4)))  # VX, VY, F, X
        up.wait_stream(stream)  # the buffers' allocation and zero fill come first
        landed = []

        def upload(k):
            (_, _, fv, xv, yv, _), (VX, VY, F, _) = subs[k], bufs[k]
            VX.write_async(xv, up.cuda_stream)
            VY.write_async(yv, up.cuda_stream)
            F.write_async(fv, up.cuda_stream)
            e_ = torch.cuda.Event()
            e_.record(up)
            landed.append(e_)

        solve_ms, run_tot, per = 0.0, 0, []
        keep = []
        host_ms = {"build": 0.0, "solve_and_check": 0.0}
        upload(0)
        for k, ((part, sd, _, _, _, out), (VX, VY, F, X)) in enumerate(zip(subs, bufs)):
            stream.wait_event(landed[k])
            tb = time.perf_counter()
            B = BatchSolver(dev, sd, nu, VX, VY, cycle_dtype=mg_dtype, n_pre=sweeps, n_post=sweeps, omega=OMEGA,
                            coarse_max=COARSE_MAX, coarse_sweeps=COARSE_SWEEPS)
            host_ms["build"] += (time.perf_counter() - tb) * 1e3
            if chunk != 2048:
                B.set_chunk(chunk)
            if k == 0:  # the other uploads go after the first build, whose small table copies would
                for j in range(1, len(subs)):  # otherwise queue behind them on the copy engine
                    upload(j)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ts = time.perf_counter()
            e0.record(stream)
            stats, run = B.bicgstab(X, F, 1e-10, 200)
            e1.record(stream)
            rn = B.residual_norms(X, F)  # every true residual, on the device (synchronises)
            host_ms["solve_and_check"] += (time.perf_counter() - ts) * 1e3
            solve_ms += e0.elapsed_time(e1)
            run_tot += run
            down.wait_stream(stream)
            X.copy_to_host_async(out, down.cuda_stream)
            per.append((part, stats, rn))
            keep.append(B)
        down.synchronize()
        return per, run_tot, solve_ms, host_ms

    once()  # warm-up (first-use costs of the library, the pool and the copy streams)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    per, run, solve_ms, host_ms = once()
    wall = time.perf_counter() - t0
    res = {}
    for part, stats, rn in per:
        for q, j in enumerate(part):
            i = mine[j]
            rel = float(rn[q] / max(host[i][4], 1e-300))
            res[i] = (sides[j] - 2, int(stats[q].iterations), bool(stats[q].converged()), solve_ms, rel, wall)
    return res, wall, {"batch_iterations_launched": run, "device_solve_ms": solve_ms,
                       "points": sum(s_ * s_ for s_ in sides), "launch_per_iteration": "one CUDA graph",
                       "pipeline_sub_batches": len(subs),
                       "host_wall_ms": {k_: round(v_, 1) for k_, v_ in host_ms.items()},
                       "tuning": {"chunk": chunk, "sweeps": sweeps, "cycle_dtype": "f32" if mg_dtype == DType.F32 else
                                  "f64", "autotuned": tuned}}


def run_batch(args):
    """The batched convection-diffusion workload, through the public API: `--batch` problems
    -nu Lap u + v.grad u = f, N x N interior with N = 2^k - 1, k ~ U{6..10}, nu = 1e-2, v from a
    stream function of 8 modes (k, l <= 4, N(0, 1) amplitudes) scaled to max|v| = 1, first-order
    upwind, Dirichlet 0, f ~ U[-1, 1], all seeded per problem; BiCGSTAB preconditioned by the
    conv-diff V(2,2)-cycle (omega 0.8, coarsest 15^2 x 200 sweeps) to ||b - A x|| < 1e-10 ||f||,
    FP64.  Every problem's host arrays are generated before the timed region, into page-locked
    host memory.  `--lanes K` host threads each drive their own context and stream on the GPU
    (Device.Cuda(0, lane=k)) and take problems from a shared counter, so up to K independent
    solves run side by side.  Timed per problem (wall clock): upload of f and the velocity
    fields, operator and hierarchy set-up, the solve (also timed with CUDA events on the lane's
    stream), the true residual b - A x recomputed on the device with the library's operator and
    its norm read back, and the solution read back into the lane's page-locked host array.  Each
    lane keeps one BiCGSTAB object per grid size, created while warming up on one problem of
    every size.  Reports solves/s = problems / wall time of the whole batch, p50 / p99 of the
    per-problem time and of the device solve time.  `--batched 1` (the default) runs the batched
    solver instead (run_batch_batched)."""
    import threading

    import torch
    from fluxion_b200 import (BiCgStabSolver, ConvDiffMultigrid, ConvDiffOperator, DType, Device, Field,
                              Grid)
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity

    from fluxion_b200.batch import gather_results, partition_by_points

    nu = 1e-2
    lanes = max(1, int(args.lanes))
    mg_dtype = DType.F32 if args.mg_dtype == "f32" else DType.F64
    rng = np.random.default_rng(SEED)
    k_lo, k_hi = (int(v) for v in args.k_range.split(","))
    ks = rng.integers(k_lo, k_hi + 1, size=args.batch)
    sizes = [int(2 ** k + 1) ** 2 for k in ks]
    # one process per GPU: each rank solves its share of the problems (split by points), no
    # data-path exchange; one gather of the per-problem results at the end
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    mine = partition_by_points(sizes, world)[rank]
    pinned = torch.empty(3 * sum(sizes[i] for i in mine), dtype=torch.float64, pin_memory=True).numpy()
    host, off = {}, 0
    for i in mine:
        n = int(2 ** ks[i] - 1)
        vx, vy = stream_velocity(n, SEED + 2 * i)
        arrs = []
        for a in (vx, vy, poisson_uniform_rhs(n, SEED + 2 * i + 1)):
            dst = pinned[off:off + a.size]
            dst[:] = a.ravel()
            arrs.append(dst)
            off += a.size
        host[i] = (n, *arrs, float(np.linalg.norm(arrs[2])))
    first_of_size = sorted({int(ks[i]): i for i in reversed(mine)}.values())
    extra = {}
    if args.batched:
        res, wall, extra = run_batch_batched(args, ks, mine, host, world, rank, local_rank, dist)
        lanes = 0
        return _batch_report(args, ks, k_lo, k_hi, res, wall, world, rank, local_rank, dist, lanes, extra, host)

    def make_lane(k):
        dev = Device.Cuda(local_rank, lane=k)
        stream = torch.cuda.Stream()
        dev.backend().set_stream(stream.cuda_stream)
        dev.backend().set_pdl(args.pdl)
        out = torch.empty(max(sizes), dtype=torch.float64, pin_memory=True).numpy()
        return dev, stream, {}, out

    def one(lane, i):
        dev, stream, solvers, out = lane
        n, vx, vy, f, fnorm = host[i]
        N, h = n + 2, 1.0 / (n + 1)
        g = Grid.square(N, h)
        stream.synchronize()
        t0 = time.perf_counter()  # from here: upload, set-up, solve, check, read-back
        VX, VY, b = Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev), Field.from_f64(g, f, dev)
        x = Field.zeros(g, DType.F64, dev)
        op = ConvDiffOperator(g, VX, VY, -nu, sigma=0.0, coeff=1.0)
        mg = ConvDiffMultigrid(op, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS, mg_dtype)
        if args.replay:
            mg.set_replay(True)
        solver = solvers.get(N)  # one solver (and its work vectors) per grid size, reused
        if solver is None:
            solver = solvers[N] = BiCgStabSolver(g, dev, 1.0, 200)
        solver.tol = 1e-10 * fnorm
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = solver.solve_op(x, b, op, mg)
        e1.record(stream)
        ax = Field.zeros(g, DType.F64, dev)
        op.apply(x, ax)
        ax.axpy(-1.0, b)
        rel = ax.norm_l2() / fnorm
        x.copy_to_host(out[:N * N])
        stream.synchronize()
        return n, st, e0.elapsed_time(e1), rel, time.perf_counter() - t0

    lane_state = [make_lane(k) for k in range(lanes)]
    for lane in lane_state:  # warm-up: one problem of every size on every lane
        for i in first_of_size:
            one(lane, i)
    torch.cuda.synchronize()
    res = {}
    nxt = [0]
    mu = threading.Lock()
    errors = []
    start = threading.Barrier(lanes + 1)

    def work(lane):
        try:
            start.wait()
            while True:
                with mu:
                    j = nxt[0]
                    nxt[0] += 1
                if j >= len(mine):
                    return
                i = mine[j]
                r = one(lane, i)
                res[i] = (r[0], int(r[1].iterations), bool(r[1].converged()), r[2], r[3], r[4])
        except Exception as e:  # reported after the join
            errors.append(e)

    threads = [threading.Thread(target=work, args=(lane,)) for lane in lane_state]
    if dist:
        dist.barrier()
    for t in threads:
        t.start()
    start.wait()
    t_begin = time.perf_counter()
    for t in threads:
        t.join()
    wall = time.perf_counter() - t_begin
    if errors:
        raise errors[0]
    return _batch_report(args, ks, k_lo, k_hi, res, wall, world, rank, local_rank, dist, lanes, extra, host)


# Algorithmic bytes per grid point of one BiCGSTAB iteration with the conv-diff V(2,2)-cycle in
# FP64 (fields x, b, vx, vy streamed once per pass): per cycle, level 0 = sweep pair 40 + residual
# 40 + restriction 10 + prolongation 18 + sweep pair 40 = 148, x 4/3 for the coarser levels; two
# cycles per iteration; the vector passes p 32, v = A p_hat 40, s 24, t = A s_hat 40, the update 64
# and the two zero fills 16.
BATCH_BYTES_PER_POINT_ITER = 2 * 148 * 4 / 3 + 216


def batch_cpu_baseline(ks, host, sample_n=16):
    """The oracle's BiCGSTAB + conv-diff V(2,2)-cycle (FP64, the same algorithm) on a sample of the
    batch keeping its size mix, on all host threads; solves/s extrapolated to the whole batch by
    points."""
    from oracle import oracle as O
    from fluxion_b200.autotune import _sample
    O.set_threads(os.cpu_count() or 1)
    sides = [int(2 ** k + 1) for k in ks]
    idx = [i for i in _sample(sides, sample_n) if i in host]
    t_tot, pts = 0.0, 0
    for i in idx:
        n, vx, vy, f, fnorm = host[i]
        N, h = n + 2, 1.0 / (n + 1)
        op = O.cd_op(N, N, h, h, np.ascontiguousarray(vx), np.ascontiguousarray(vy), kappa=None, kappa_s=-1e-2,
                     sigma=0.0, coeff=1.0)
        x = np.zeros(N * N)
        t0 = time.perf_counter()
        O.bicgstab_solve_op(x, np.ascontiguousarray(f), op, 1e-10 * fnorm, 200,
                            O.CdMultigrid(op, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS))
        t_tot += time.perf_counter() - t0
        pts += N * N
    all_pts = sum(s * s for s in sides)
    per_point_s = t_tot / max(1, pts)
    return {"value": len(sides) / (per_point_s * all_pts), "unit": "solves/s", "cores": O.get_threads(),
            "kind": "port", "sample": f"{len(idx)} problems keeping the batch's size mix ({t_tot:.1f} s), "
                                      "extrapolated to the whole batch by grid points"}


def _batch_report(args, ks, k_lo, k_hi, res, wall, world, rank, local_rank, dist, lanes, extra, host=None):
    import torch
    from fluxion_b200.batch import gather_results
    if dist:  # the job's wall time is the slowest rank's; then one gather of the results
        t = torch.tensor([wall], device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        wall = float(t.item())
        allres = gather_results(res, args.batch)
        dist.barrier()
        dist.destroy_process_group()
    else:
        allres = [res[i] for i in range(args.batch)]
    if rank != 0:
        return 0
    res = allres
    ms = np.array([r[3] for r in res])
    its = np.array([r[1] for r in res])
    ok = all(r[2] for r in res)
    peak, peak_kind = measured_peaks()
    roof = None
    if args.batched and extra.get("device_solve_ms"):
        # solve level: the algorithmic bytes of every problem's iterations over the batch's device time
        byts = sum(BATCH_BYTES_PER_POINT_ITER * (r[1] + 1) * (r[0] + 2) ** 2 for r in res)
        ach = byts / (extra["device_solve_ms"] * 1e-3) / 1e9
        roof = {"kernel": "whole batched solve (all phases)", "bound": "hbm", "achieved": ach, "peak": peak,
                "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind, "traffic": None,
                "nominal_peak": NOMINAL_HBM_GBS, "frac_of_nominal": ach / NOMINAL_HBM_GBS,
                "bytes_per_point_iteration": BATCH_BYTES_PER_POINT_ITER}
    cpu = None
    if not args.no_cpu and host is not None:
        try:
            cpu = batch_cpu_baseline(ks, host)
        except Exception as e:  # reported, never required
            cpu = {"value": None, "unit": "solves/s", "kind": "port", "sample": f"failed: {e}"}
    print(json.dumps({
        "mode": "batch", "workload": f"convdiff_batch_{args.batch}_k{k_lo}-{k_hi}_nu1e-2_bicgstab_cdmg",
        "solver": "batched (one launch per phase over the batch)" if args.batched else "lanes",
        "problems": args.batch, "n_gpus": world, "scaling": "strong", "lanes": lanes, "pdl": bool(args.pdl),
        **extra,
        "vcycle_dtype": extra.get("tuning", {}).get("cycle_dtype", args.mg_dtype), "vcycle_replay": bool(args.replay),
        "interior_sizes": {str(2 ** k - 1): int((ks == k).sum()) for k in range(k_lo, k_hi + 1)},
        "solves_per_s": args.batch / wall, "wall_s_excluding_host_data_generation": wall,
        "per_problem_ms_p50": float(np.percentile([r[5] * 1e3 for r in res], 50)),
        "per_problem_ms_p99": float(np.percentile([r[5] * 1e3 for r in res], 99)),
        "solve_ms_p50": float(np.percentile(ms, 50)), "solve_ms_p99": float(np.percentile(ms, 99)),
        "iterations_p50": float(np.percentile(its, 50)), "iterations_max": int(its.max()),
        "all_converged": ok, "max_true_rel_residual": max(r[4] for r in res), "roofline": roof, "cpu_baseline": cpu,
        "dtype": "f64" if extra.get("tuning", {}).get("cycle_dtype", args.mg_dtype) == "f64"
        else "f64 (Krylov) / f32 (V-cycle)",
        "data": "synthetic (seeded per problem), page-locked host arrays",
        "note": ("batched, in sub-batches whose uploads and read-backs overlap the other sub-batches' solves: "
                 "per-problem times are the whole job's" if args.batched else
                 f"{lanes} host thread(s), one context and stream each, through the public API")}),
        flush=True)
    return 0 if ok else 1


def run_convdiff(args):
    """Convection-dominated steady conv-diff on one grid: -nu Lap u + v.grad u = f, `--n` x `--n`
    interior (default 4095), nu from `--nu`, v from the stream-function law of the batched
    workload (8 modes, k, l <= 4, max|v| = 1), first-order upwind, Dirichlet 0, f ~ U[-1, 1],
    seeded.  Each solver to ||b - A x|| < 1e-10 ||f|| (FP64) from x = 0, preconditioned by the
    conv-diff V(2,2)-cycle (weighted Jacobi 0.8, full weighting / bilinear, coarsest 15^2 x 200
    sweeps): flexible GMRES(30), GMRES(30) (left-preconditioned: it stops on the preconditioned
    residual, so its true residual is reported beside it) and BiCGSTAB; FGMRES and BiCGSTAB
    again with the cycle in FP32 (the Krylov solver, its vectors and the residual stay FP64).  Device time with CUDA
    events around each solve; the true residual recomputed on the device.  These are the plain
    Jacobi-multigrid arms; the learned smoother's arms are --mode learned."""
    import torch
    from fluxion_b200 import (BiCgStabSolver, ConvDiffMultigrid, ConvDiffOperator, DType, Device, Field,
                              FgmresSolver, GmresSolver, Grid)
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity

    n = args.n
    dev = Device.Cuda(0)
    stream = torch.cuda.Stream()
    dev.backend().set_stream(stream.cuda_stream)
    vx, vy = stream_velocity(n, SEED + 40)
    f = poisson_uniform_rhs(n, SEED + 41)
    N, h = n + 2, 1.0 / (n + 1)
    g = Grid.square(N, h)
    VX, VY, b = Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev), Field.from_f64(g, f, dev)
    fnorm = float(np.linalg.norm(f))
    runs = []
    ok = True
    for nu in [float(v) for v in args.nu.split(",")]:
        op = ConvDiffOperator(g, VX, VY, -nu, sigma=0.0, coeff=1.0)
        def fg_cgs2():
            s_ = FgmresSolver(g, dev, 30, 1e-10 * fnorm, 2000)
            s_.set_orthogonalization("cgs2")
            return s_

        arms = [(mdt, name, make) for mdt in (DType.F64, DType.F32) for name, make in (
            ("fgmres30", lambda: FgmresSolver(g, dev, 30, 1e-10 * fnorm, 2000)),
            ("fgmres30_cgs2", fg_cgs2),
            ("gmres30", lambda: GmresSolver(g, dev, 30, 1e-10 * fnorm, 2000)),
            ("bicgstab", lambda: BiCgStabSolver(g, dev, 1e-10 * fnorm, 2000)))
            if mdt == DType.F64 or name != "gmres30"]
        for mdt, name, make in arms:
            mg = ConvDiffMultigrid(op, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS, mdt)
            solver = make()
            x = Field.zeros(g, DType.F64, dev)
            solver.solve_op(x, b, op, mg)  # warm-up solve (same problem)
            x.fill(0.0)
            stream.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = solver.solve_op(x, b, op, mg)
            e1.record(stream)
            stream.synchronize()
            ax = Field.zeros(g, DType.F64, dev)
            op.apply(x, ax)
            ax.axpy(-1.0, b)
            true_rel = ax.norm_l2() / fnorm
            ok = ok and st.converged() and (name == "gmres30" or true_rel < 1e-10)
            cell_peclet = h / (2.0 * nu)  # max|v| h / (2 nu)
            cyc = " + conv-diff V(2,2)-cycle" + (" in FP32" if mdt == DType.F32 else "")
            runs.append({"nu": nu, "solver": name + cyc, "iterations": st.iterations,
                         "converged": st.converged(), "ms": e0.elapsed_time(e1), "true_rel_residual": true_rel,
                         "ms_per_iteration": e0.elapsed_time(e1) / max(1, st.iterations),
                         "max_cell_peclet": cell_peclet})
            print(json.dumps(runs[-1]), flush=True, file=sys.stderr)
    print(json.dumps({"mode": "convdiff", "workload": f"convdiff_{n}sq_upwind_stream8", "n_interior": n,
                      "runs": runs, "dtype": "f64", "data": "synthetic (seeded)",
                      "note": "plain Jacobi-multigrid arms (the learned smoother's are --mode learned)"}),
          flush=True)
    return 0 if ok else 1


def run_learned(args):
    """The learned-smoother configuration: the network is trained on the GPU (the library's forward,
    backward and Adam kernels) on 20,480 samples cut from plain V-cycle iterates of seeded problems
    of 63^2 - 511^2 interior points with nu in {1e-2, 1e-3, 1e-4} (the stream-function velocity law,
    f ~ U[-1, 1]); then, on the --n^2 problem for each --nu, flexible GMRES(30) preconditioned by the
    conv-diff V(2,2)-cycle with the learned smoother (every level of at least 1024 points; per-cycle
    check with fallback to the plain cycle at 0.9) against the same solver with the plain
    weighted-Jacobi cycle, both to ||b - A x|| < 1e-10 ||f|| in FP64.  Reported per arm: iterations,
    device time (CUDA events), true relative residual, and the error against an FP64 solve of the
    same system to 1e-12 (FGMRES with the plain cycle)."""
    import torch
    from fluxion_b200 import (ConvDiffMultigrid, ConvDiffOperator, DType, Device, FgmresSolver, Field, GmresSolver,
                              Grid)
    from fluxion_b200.learned import LearnedSmoother, SmootherSamples
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity

    dev = Device.Cuda(0)
    stream = torch.cuda.Stream()
    dev.backend().set_stream(stream.cuda_stream)

    def problem(n, nu, seed):
        N, h = n + 2, 1.0 / (n + 1)
        g = Grid.square(N, h)
        vx, vy = stream_velocity(n, seed)
        f = poisson_uniform_rhs(n, seed + 1)
        keep = (Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev))
        return g, f, ConvDiffOperator(g, keep[0], keep[1], -nu, sigma=0.0, coeff=1.0), keep

    t0 = time.perf_counter()
    S = SmootherSamples(dev, 20480)
    per = {63: 96, 127: 256, 255: 512, 511: 842}
    k = 0
    for n in (63, 127, 255, 511):
        for nu in (1e-2, 1e-3, 1e-4):
            g, f, op, keep = problem(n, nu, SEED + 1000 + k)
            S.add_problem(op, Field.from_f64(g, f, dev), iterates=4, patches_per_iterate=per[n], seed=k)
            k += 1
    gen_s = time.perf_counter() - t0
    lsm = LearnedSmoother(dev, seed=SEED)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = lsm.train(S, epochs=30, batch=256, lr=2e-3, seed=SEED)
    train_s = time.perf_counter() - t0

    def solve(op, g, b, mg, tol, gmres=False):
        x = Field.zeros(g, DType.F64, dev)
        solver = GmresSolver(g, dev, 30, tol, 3000) if gmres else FgmresSolver(g, dev, 30, tol, 3000)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = solver.solve_op(x, b, op, mg)
        e1.record(stream)
        stream.synchronize()
        return x, st, e0.elapsed_time(e1)

    g, f, op, keep = problem(255, 1e-3, SEED + 7)  # warm-up of every kernel on a small problem
    for learned in (False, True):
        mg = ConvDiffMultigrid(op, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS)
        if learned:
            mg.set_learned(lsm, min_points=1024, fallback_ratio=0.9)
        solve(op, g, Field.from_f64(g, f, dev), mg, 1e-10 * np.linalg.norm(f))

    n = args.n
    runs = []
    ok = True
    for nu in [float(v) for v in args.nu.split(",")]:
        g, f, op, keep = problem(n, nu, SEED + 40)
        b = Field.from_f64(g, f, dev)
        fnorm = float(np.linalg.norm(f))
        xr, sr, _ = solve(op, g, b, ConvDiffMultigrid(op, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS), 1e-12 * fnorm)
        u_ref = xr.to_vec_f64()
        # arms: GMRES(30) with the plain (Jacobi) cycle, the configuration's comparison solver (left-
        # preconditioned: it stops on the preconditioned residual); FGMRES(30) with the plain cycle;
        # learned smoothing on every level of at least 1024 points; learned smoothing only on the
        # levels of the training problems' sizes (at most 513^2 points), without and with a patience
        # (8 fallbacks in a row switch the learned cycle off)
        for arm, lo, hi, pat in (("gmres30_plain", 0, 0, 0), ("plain", 0, 0, 0), ("learned", 1024, 0, 0),
                                 ("learned_levels_upto_513sq", 1024, 513 * 513, 0),
                                 ("learned_levels_upto_513sq_patience8", 1024, 513 * 513, 8)):
            learned = arm not in ("plain", "gmres30_plain")
            mg = ConvDiffMultigrid(op, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS)
            if learned:
                mg.set_learned(lsm, min_points=lo, fallback_ratio=0.9, max_points=hi)
                if pat:
                    mg.set_learned_patience(pat)
            x, st, ms = solve(op, g, b, mg, 1e-10 * fnorm, gmres=arm == "gmres30_plain")
            ax = Field.zeros(g, DType.F64, dev)
            op.apply(x, ax)
            ax.axpy(-1.0, b)
            rel = ax.norm_l2() / fnorm
            u = x.to_vec_f64()
            err = float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref))
            ok = ok and st.converged() and (rel < 1e-10 or arm == "gmres30_plain")
            r = {"nu": nu, "arm": arm, "iterations": st.iterations,
                 "converged": st.converged(), "ms": ms, "ms_per_iteration": ms / max(1, st.iterations),
                 "true_rel_residual": rel, "err_vs_fp64_reference_solve": err,
                 "reference_solve": {"iterations": sr.iterations, "tol": "1e-12 relative"}}
            if learned:
                apps, fb = mg.learned_stats()
                r["learned_cycles"] = {"applications": apps, "fallbacks": fb}
                if pat:
                    r["learned_cycles"]["switched_off"] = mg.learned_disabled()
            runs.append(r)
            print(json.dumps(r), file=sys.stderr, flush=True)
    print(json.dumps({"mode": "learned", "workload": f"convdiff_{n}sq_fgmres30_learned_smoother",
                      "samples": len(S), "sample_generation_s": gen_s, "training": {
                          "epochs": 30, "batch": 256, "lr": 2e-3, "loss": "high-frequency error after the step",
                          "seconds": train_s, "epoch_loss_first": hist[0], "epoch_loss_last": hist[-1]},
                      "runs": runs, "dtype": "f64 Krylov / f64 cycle; network bf16 weights and activations, "
                                             "f32 accumulation", "data": "synthetic (seeded)"}), flush=True)
    return 0 if ok else 1


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.mode == "vcycle":
        return run_vcycle(args)
    if args.mode == "batch":
        return run_batch(args)
    if args.mode == "convdiff":
        return run_convdiff(args)
    if args.mode == "learned":
        return run_learned(args)
    if args.mode == "lsm_step":
        return run_lsm_step(args)
    if args.mode == "micro":  # the microbenchmarks alone, on an --n^2 grid (a profiling target)
        import torch
        from fluxion_b200 import Device
        be = Device.Cuda(0).backend()
        stream = torch.cuda.Stream()
        be.set_stream(stream.cuda_stream)
        peak, _ = measured_peaks()
        print(json.dumps({"mode": "micro", "n": args.n, "microbench": microbench(be, peak, args, stream, args.n)}),
              flush=True)
        return 0

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from fluxion_b200 import (CgSolver, DType, Device, FcgSolver, Field, InnerPcgF32, MixedPrecisionRefinement,
                              Multigrid, PipelinedCgSolver)
    from fluxion_b200 import _lib as L
    from fluxion_b200.workloads import dst_poisson_solve, neg_laplacian_residual, poisson_modes_rhs, \
        poisson_problem

    peak, peak_kind = measured_peaks()
    dev = Device.Cuda(local)
    be = dev.backend()
    stream = torch.cuda.Stream(device=local)
    be.set_stream(stream.cuda_stream)

    n = args.n
    P = poisson_problem(n)
    N = n + 2
    f = poisson_modes_rhs(n, SEED + rank)
    fnorm = float(np.linalg.norm(f))
    tol = 1e-10 * fnorm
    b = Field.from_f64(P.grid, f, dev)
    x = Field.zeros(P.grid, DType.F64, dev)
    cg = CgSolver(P.grid, dev, tol, 100)
    pcg_pipe = PipelinedCgSolver(P.grid, dev, tol, 100)
    # FP64 iterative refinement around FP32 V-cycle PCG inner solves (inner tol 1e-4)
    ir = MixedPrecisionRefinement(P.grid, dev, tol, 20, 1e-4, 100)
    mg64 = Multigrid.vertex(P.grid, None, dev, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS, DType.F64)
    mg32 = Multigrid.vertex(P.grid, None, dev, 2, 2, OMEGA, COARSE_MAX, COARSE_SWEEPS, DType.F32)

    def solve(mg, solver=cg):
        x.fill(0.0)
        return solver.solve_preconditioned(x, b, P.coeff, P.stencil, None, mg)

    def timed(mg, k, w, kernel=None, solver=cg):
        for _ in range(w):
            solve(mg, solver)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        l0 = be.launch_count()
        if kernel:
            L.lib().fx_ctx_timing_begin(be.ctx, kernel.encode())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = None
        for _ in range(k):
            st = solve(mg, solver)
        e1.record(stream)
        torch.cuda.synchronize()
        ktime = None
        if kernel:
            import ctypes as C
            cap = 1 << 16
            ms, pts, byt = (C.c_double * cap)(), (C.c_double * cap)(), (C.c_double * cap)()
            cnt = C.c_size_t()
            L.lib().fx_ctx_timing_end_records(be.ctx, ms, pts, byt, cap, C.byref(cnt))
            ktime = [(ms[i], pts[i], byt[i]) for i in range(cnt.value)]
        launches = be.launch_count() - l0
        ms_total = e0.elapsed_time(e1)
        if dist:
            t = torch.tensor([ms_total], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms_total = float(t.item())
        return ms_total / k, st, launches, ktime

    # which kernel dominates the plain FP64 solve? (one untimed solve per candidate)
    import ctypes as C
    candidates = ["mg_down", "mg_up", "mg_tail", "mg_sweep", "pcg_update", "pcg_dir", "mg_residual", "mg_restrict_fw",
                  "mg_prolong_bilinear", "pcg_rz", "mg_convert", "mg_zero", "mg_coarse_solve"]
    solve(mg64)
    shares = {}
    for kname in candidates:
        L.lib().fx_ctx_timing_begin(be.ctx, kname.encode())
        solve(mg64)
        ms, cnt, pts = C.c_double(), C.c_ulonglong(), C.c_double()
        L.lib().fx_ctx_timing_end(be.ctx, C.byref(ms), C.byref(cnt), C.byref(pts))
        shares[kname] = ms.value
    dom = max(shares, key=shares.get)

    # the headline: the plain FP64 solve (clocks sampled over its timed region)
    with ClockSampler(local, uuid=str(torch.cuda.get_device_properties(local).uuid)) as clk:
        plain_ms, st64, launches, _ = timed(mg64, args.steps, args.warmup)
    u64 = x.to_vec_f64()
    # the dominant kernel's launches, bracketed by CUDA events on the launch stream, over a second
    # timed pass of the same K solves: the events split the programmatic-launch overlap, so they
    # stay out of the pass that gives `value`
    hooked_ms, _, _, ktime = timed(mg64, args.steps, 0, kernel=dom)
    # the mixed solve: FP64 CG, residual, update and inner products around the FP32 V-cycle
    mixed_ms, st32, mixed_launches, _ = timed(mg32, args.steps, args.warmup)
    u32 = x.to_vec_f64()
    # the configuration's second solver: pipelined CG preconditioned by the V-cycle (FP64 cycle:
    # the pipelined recurrences carry u = M r instead of recomputing it, and stall near 1e-6 with
    # the FP32 cycle's rounding)
    pipe_ms, stp, _, _ = timed(mg64, args.steps, args.warmup, solver=pcg_pipe)
    up = x.to_vec_f64()
    ir_ms, sti, _, _ = timed(mg32, args.steps, args.warmup, solver=ir)
    ui = x.to_vec_f64()
    # FP64 flexible CG around inner FP32 V-cycle PCG solves (inner tol 1e-4): the outer Krylov
    # space is kept where the refinement loop restarts
    fcg = FcgSolver(P.grid, dev, tol, 50)
    ipc = InnerPcgF32(P.grid, P.coeff, P.stencil, None, mg32, 1e-4, 100, dev)
    fcg_ms, stf, _, _ = timed(ipc, args.steps, args.warmup, solver=fcg)
    apps_f, inner_f = ipc.stats()
    uf = x.to_vec_f64()

    # verification in FP64 (plain operator) and against the exact DST-I solve
    u_ref = dst_poisson_solve(f, n)
    err32 = float(np.linalg.norm(u32 - u_ref) / np.linalg.norm(u_ref))
    err64 = float(np.linalg.norm(u64 - u_ref) / np.linalg.norm(u_ref))
    rr32 = neg_laplacian_residual(u32, f, n) / fnorm
    rr64 = neg_laplacian_residual(u64, f, n) / fnorm
    errp = float(np.linalg.norm(up - u_ref) / np.linalg.norm(u_ref))
    erri = float(np.linalg.norm(ui - u_ref) / np.linalg.norm(u_ref))
    rri = neg_laplacian_residual(ui, f, n) / fnorm
    errf = float(np.linalg.norm(uf - u_ref) / np.linalg.norm(u_ref))
    rrf = neg_laplacian_residual(uf, f, n) / fnorm
    rrp = neg_laplacian_residual(up, f, n) / fnorm

    # e2e: host f (pinned) -> solve -> host u (pinned), through the public API
    f_host = torch.empty(N * N, dtype=torch.float64, pin_memory=True).numpy()
    f_host[:] = f
    u_host = torch.empty(N * N, dtype=torch.float64, pin_memory=True).numpy()

    def e2e(mg, want):
        def step():
            b.write(f_host)
            x.fill(0.0)
            cg.solve_preconditioned(x, b, P.coeff, P.stencil, None, mg)
            x.storage.copy_to_host_f64(u_host)

        for _ in range(args.warmup):
            step()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        e_ms = max(e0.elapsed_time(e1), (time.perf_counter() - w0) * 1e3) / args.steps
        if dist:
            t = torch.tensor([e_ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        return {"value": e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": N * N * 8,
                "d2h_bytes_per_step": N * N * 8, "result_matches_device_run": bool(np.array_equal(u_host, want))}

    def e2e_pipelined(mg, want, nsteps):
        """The same stream of solves with the copies overlapped: step k's f is uploaded on one copy
        stream and step k-2's u read back on another while step k-1 solves (double-buffered b and
        x, ordered by events).  Every step still uploads its f and reads back its u."""
        up_s, down_s = torch.cuda.Stream(), torch.cuda.Stream()
        bs = [b, Field.zeros(P.grid, DType.F64, dev)]
        xs = [x, Field.zeros(P.grid, DType.F64, dev)]
        outs = [torch.empty(N * N, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
        ev_up = [torch.cuda.Event() for _ in range(2)]
        ev_down = [torch.cuda.Event() for _ in range(2)]
        for e_ in ev_down:
            e_.record(down_s)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        w0 = time.perf_counter()
        for k in range(nsteps + 2):
            if k < nsteps:  # upload of step k (its buffer's last reader, step k-2, has returned)
                bs[k % 2].write_async(f_host, up_s.cuda_stream)
                ev_up[k % 2].record(up_s)
            j = k - 2
            if 0 <= j < nsteps:  # read-back of step j (solved and returned)
                xs[j % 2].copy_to_host_async(outs[j % 2], down_s.cuda_stream)
                ev_down[j % 2].record(down_s)
            j = k - 1
            if 0 <= j < nsteps:  # solve of step j after its upload and the read-back that used its x
                stream.wait_event(ev_up[j % 2])
                stream.wait_event(ev_down[j % 2])
                xs[j % 2].fill(0.0)
                cg.solve_preconditioned(xs[j % 2], bs[j % 2], P.coeff, P.stencil, None, mg)
        torch.cuda.synchronize()
        e_ms = (time.perf_counter() - w0) * 1e3 / nsteps
        if dist:
            t = torch.tensor([e_ms], device=f"cuda:{local}")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e_ms = float(t.item())
        ok = all(bool(np.array_equal(o, want)) for o in outs)
        return {"value": e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": N * N * 8,
                "d2h_bytes_per_step": N * N * 8, "result_matches_device_run": ok,
                "how": "a stream of solves through the public API: step k's upload and step k-2's read-back "
                       "on two copy streams while step k-1 solves (pinned host memory, double-buffered)"}

    e2e_plain_serial = e2e(mg64, u64)
    e2e_mixed_serial = e2e(mg32, u32)
    e2e_pipelined(mg64, u64, max(2, args.warmup))  # warm-up of the copy streams and buffers
    e2e_plain = e2e_pipelined(mg64, u64, args.steps)
    e2e_plain["serial"] = e2e_plain_serial
    e2e_mixed = e2e_pipelined(mg32, u32, args.steps)
    e2e_mixed["serial"] = e2e_mixed_serial

    # roofline of the dominant kernel, live over the timed plain solves
    roof = None
    if ktime:
        # The roofline is taken over the dominant kernel's finest-grid launches (the multigrid
        # kernels also run on every coarser level, where they are latency-bound); the
        # all-launch average is reported beside it.  Kernels that do not state their bytes
        # get the table's F64 figure.
        bpp_table = BYTES_PER_POINT.get(dom, 3) * 8
        nbytes = [b if b > 0 else p * bpp_table for (_, p, b) in ktime]
        top = max(p for (_, p, _) in ktime)
        fine = [i for i, (_, p, _) in enumerate(ktime) if p == top]
        f_ms = sum(ktime[i][0] for i in fine) / len(fine)
        f_bytes = nbytes[fine[0]]
        achieved = f_bytes / (f_ms * 1e-3) / 1e9
        all_ms = sum(t for (t, _, _) in ktime)
        traffic = None
        tp = os.path.join(ROOT, "profiles", f"{dom}_f64_traffic.txt")
        if os.path.exists(tp):
            for ln in open(tp):
                if ln.startswith("dram_bytes_per_point:"):
                    traffic = float(ln.split(":")[1]) * top
        roof = {"kernel": dom + " (F64 cycle)", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                "nominal_peak": NOMINAL_HBM_GBS, "frac_of_nominal": achieved / NOMINAL_HBM_GBS,
                "algorithmic_bytes_per_launch": f_bytes, "bytes_per_point": f_bytes / top,
                "grid_points_per_launch": top, "launches": len(fine), "avg_launch_ms": f_ms,
                "all_levels": {"launches": len(ktime), "ms": all_ms,
                               "GBps": sum(nbytes) / (all_ms * 1e-3) / 1e9},
                "share_of_solve": (all_ms / args.steps) / hooked_ms,
                "timed_pass_ms_per_step": hooked_ms}

    micro = None
    if not args.no_micro:
        micro = microbench(be, peak, args, stream)

    cpu = None
    if rank == 0 and not args.no_cpu:
        try:
            runs = [oracle_solve(n, f) for _ in range(3)]  # best of 3
            t, iters, cores = min(runs)
            cpu = {"value": t, "unit": "s", "cores": cores, "kind": "port",
                   "sample": f"best of 3 full {n}^2 MG-PCG solves to 1e-10 ({iters} iterations), FP64"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "s", "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": plain_ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": plain_ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded 32-mode sin-sin source + 1e-3 uniform noise)",
            "config": headline_config(n, world),
            "iterations": int(st64.iterations), "rel_residual_fp64": rr64, "err_vs_fp64_direct": err64,
            "e2e": e2e_plain,
            "mixed_fp32_cycle": {"value": mixed_ms / 1e3, "unit": "s", "iterations": int(st32.iterations),
                                 "rel_residual_fp64": rr32, "err_vs_fp64_direct": err32, "e2e": e2e_mixed,
                                 "gpu_launches": int(mixed_launches),
                                 "solver": f"FP64 CG, residual, update and dots + F32 {SOLVER}"},
            "speedup_mixed_vs_plain": plain_ms / mixed_ms,
            "pipelined_pcg": {"value": pipe_ms / 1e3, "unit": "s", "iterations": int(stp.iterations),
                              "rel_residual_fp64": rrp, "err_vs_fp64_direct": errp,
                              "solver": f"pipelined CG (Ghysels-Vanroose, preconditioned) + F64 {SOLVER}"},
            "refinement_fp64_fp32_pcg": {"value": ir_ms / 1e3, "unit": "s", "outer_iterations": int(sti.iterations),
                                         "inner_iterations": ir.last_inner_iterations, "rel_residual_fp64": rri,
                                         "err_vs_fp64_direct": erri,
                                         "solver": f"FP64 refinement, FP32 CG + F32 {SOLVER} inner to 1e-4"},
            "fcg_fp64_outer_fp32_pcg_inner": {
                "value": fcg_ms / 1e3, "unit": "s", "outer_iterations": int(stf.iterations),
                "inner_iterations_per_solve": inner_f / max(1, args.steps + args.warmup),
                "rel_residual_fp64": rrf, "err_vs_fp64_direct": errf,
                "solver": f"FP64 flexible CG, inner FP32 CG + F32 {SOLVER} to 1e-4 per application"},
            "roofline": roof, "cpu_baseline": cpu, "clocks": clk.summary(),
            "gpu_launches": int(launches), "kernel_time_shares_ms": shares, "microbench": micro,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def microbench(be, peak, args, stream, n=16384):
    """Stencil / stencil-AXPY / AXPY / dual-dot on an n^2 grid (16384^2 by default: inputs far above L2)."""
    import torch
    from fluxion_b200 import Boundaries, DType, Grid, Stencil

    g = Grid.square(n, 1.0 / (n - 1))
    st = Stencil.laplacian_2d_5pt(g.dx, g.dy)
    bc = Boundaries.zero_dirichlet()
    out = {}
    reps = max(5, args.steps)
    for dt, es in ((DType.F64, 8), (DType.F32, 4)):
        a = be.allocate(n * n, dt)
        c = be.allocate(n * n, dt)
        be.fill(a, 1.0)
        cases = {
            "stencil": (lambda: be.apply_stencil(a, c, g, st, bc), 2 * es),
            "stencil_axpy": (lambda: be.stencil_axpy(0.5, a, c, g, st, bc), 3 * es),
            "axpy": (lambda: be.axpy(0.5, a, c), 3 * es),
            "dot2": (lambda: be.dot2(a, c, c, c), 2 * es),  # (a.c, c.c): 2 distinct vectors read
        }
        for name, (fn, bpp) in cases.items():
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)  # the stream every library kernel is launched on
            for _ in range(reps):
                fn()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            gbs = n * n * bpp / (ms * 1e-3) / 1e9
            out[f"{name}_{dt.name.lower()}"] = {"GBps": gbs, "frac_of_measured_peak": gbs / peak,
                                                "ms": ms, "bytes_per_point": bpp}
        a.free()
        c.free()
    return out


if __name__ == "__main__":
    sys.exit(main())
