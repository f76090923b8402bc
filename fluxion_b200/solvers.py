"""Solver structs of fluxion's runtime, executed by the native C++/CUDA solver loops.

``CgSolver`` (crates/runtime/src/cg.rs:52-256), ``PipelinedCgSolver``
(pipelined_cg.rs:25-237), ``BiCgStabSolver`` (bicgstab.rs:19-346),
``GmresSolver`` (gmres.rs:24-491), ``Multigrid`` (multigrid.rs:39-608),
``Identity`` / ``Preconditioner`` (preconditioner.rs:10-37), ``LinearSolver``
(linear_solver.rs:13-102), ``SolveStats`` / ``ConvergenceReason`` (cg.rs:9-41).
Same constructor arguments, public fields and solve signatures as the
reference; each ``solve`` is one call into ``libfluxion_cuda.so``.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass
from typing import Optional

from . import _lib as L
from .backend import StencilC, bcs_c, check, grid_c
from .core import Boundaries, DType, Grid, Stencil
from .field import Device, Field


class ConvergenceReason(enum.IntEnum):
    """cg.rs:9-18"""

    Converged = 0
    MaxIterations = 1
    Breakdown = 2


@dataclass
class SolveStats:
    """cg.rs:20-38"""

    iterations: int
    residual: float
    reason: ConvergenceReason

    def converged(self) -> bool:
        return self.reason == ConvergenceReason.Converged


CgStats = SolveStats


def _stats(st: L.FxStats) -> SolveStats:
    return SolveStats(int(st.iterations), float(st.residual), ConvergenceReason(st.reason))


# ------------------------------------------------------------------ preconditioners

class Preconditioner:
    """preconditioner.rs:10-29: ``apply(z, r)`` approximately solves M z = r."""

    def _handle(self, device: Device) -> int:
        raise NotImplementedError

    def apply(self, z: Field, r: Field) -> None:
        check(L.lib().fx_precond_apply(self._handle(z.device()), z.storage.handle, r.storage.handle))


class Identity(Preconditioner):
    """preconditioner.rs:31-37: z = r."""

    def __init__(self):
        self._h = {}

    def _handle(self, device: Device) -> int:
        h = self._h.get(device)
        if h is None:
            out = C.c_void_p()
            check(L.lib().fx_precond_identity(device.backend().ctx, C.byref(out)))
            h = out.value
            self._h[device] = h
        return h

    def __del__(self):
        try:
            for h in self._h.values():
                L.lib().fx_precond_destroy(h)
        except Exception:
            pass


class SmootherKind(enum.IntEnum):
    """multigrid.rs:11-20"""

    Jacobi = 0
    Chebyshev = 1


class Multigrid(Preconditioner):
    """Geometric multigrid V-cycle preconditioner.

    ``Multigrid(grid, boundaries, device, n_pre, n_post, omega)`` / ``Multigrid.build(...)`` give
    the reference hierarchy and operators (multigrid.rs:61-146).  ``Multigrid.vertex(...)`` gives
    the vertex-centred cycle for the operator actually solved (full weighting, bilinear
    prolongation, true weighted Jacobi, dense coarsest solve), which is the one the Poisson and
    convection-diffusion configurations use.
    """

    def __init__(self, grid: Grid, boundaries: Boundaries, device: Optional[Device] = None, n_pre: int = 2,
                 n_post: int = 2, omega: float = 2.0 / 3.0, smoother: SmootherKind = SmootherKind.Jacobi,
                 _handle: Optional[int] = None):
        self.device = device or Device.best()
        self.grid = grid
        if _handle is not None:
            self.h = _handle
            return
        out = C.c_void_p()
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_mg_create(self.device.backend().ctx, C.byref(g), C.byref(b), int(n_pre), int(n_post),
                                   float(omega), int(smoother), C.byref(out)))
        self.h = out.value

    @staticmethod
    def new(grid, boundaries, device=None, n_pre=2, n_post=2, omega=2.0 / 3.0) -> "Multigrid":
        return Multigrid(grid, boundaries, device, n_pre, n_post, omega)

    @staticmethod
    def build(grid, boundaries, device=None, n_pre=2, n_post=2, omega=2.0 / 3.0,
              smoother=SmootherKind.Jacobi) -> "Multigrid":
        return Multigrid(grid, boundaries, device, n_pre, n_post, omega, smoother)

    @staticmethod
    def vertex(grid: Grid, boundaries: Optional[Boundaries] = None, device: Optional[Device] = None,
               n_pre: int = 2, n_post: int = 2, omega: float = 0.8, coarse_max: int = 15,
               coarse_sweeps: int = 200, dtype: DType = DType.F64, op_coeff: float = 1.0,
               op_stencil: Optional[Stencil] = None) -> "Multigrid":
        device = device or Device.best()
        op_stencil = op_stencil or Stencil.poisson_neg_laplacian(grid.dx, grid.dy)
        sc = StencilC(op_stencil)
        opts = L.FxMgVertexOpts(int(n_pre), int(n_post), float(omega), int(coarse_max), int(coarse_sweeps),
                                int(dtype), float(op_coeff), sc.s)
        out = C.c_void_p()
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_mg_create_vertex(device.backend().ctx, C.byref(g), C.byref(b), C.byref(opts),
                                          C.byref(out)))
        return Multigrid(grid, boundaries, device, _handle=out.value)

    def depth(self) -> int:
        d = C.c_size_t()
        check(L.lib().fx_mg_depth(self.h, C.byref(d)))
        return d.value

    def level_dims(self, level: int):
        r, c = C.c_size_t(), C.c_size_t()
        check(L.lib().fx_mg_level_dims(self.h, int(level), C.byref(r), C.byref(c)))
        return r.value, c.value

    def v_cycle(self, x: Field, b: Field) -> None:
        check(L.lib().fx_mg_v_cycle(self.h, x.storage.handle, b.storage.handle))

    def set_tuning(self, chunk_pct: int = 100, tail_top_points: int = 0) -> None:
        """Layout of the fused cycle (no effect on its values): strip row chunks per launch in
        percent of one wave, and the largest level the one-block tail takes (0: default)."""
        t = L.FxMgTuning(int(chunk_pct), int(tail_top_points))
        check(L.lib().fx_mg_set_tuning(self.h, C.byref(t)))

    def get_tuning(self) -> dict:
        t = L.FxMgTuning()
        check(L.lib().fx_mg_get_tuning(self.h, C.byref(t)))
        return {"chunk_pct": t.chunk_pct, "tail_top_points": t.tail_top_points}

    def autotune(self, z: Field, r: Field, reps: int = 5) -> dict:
        """Time the candidate layouts of the fused cycle on (z, r) and keep the fastest
        (fx_mg_autotune); z is overwritten.  Returns the choice, its time per cycle and every
        candidate's time."""
        best = L.FxMgTuning()
        best_ms = C.c_double()
        cand = (C.c_double * 8)()
        ncand = C.c_size_t()
        check(L.lib().fx_mg_autotune(self.h, z.storage.handle, r.storage.handle, int(reps), C.byref(best),
                                     C.byref(best_ms), cand, 8, C.byref(ncand)))
        return {"chunk_pct": best.chunk_pct, "tail_top_points": best.tail_top_points, "ms": best_ms.value,
                "candidates_ms": [cand[i] for i in range(ncand.value)]}

    def precondition(self, z: Field, r: Field) -> None:
        """z = M^-1 r from a zero initial guess (z.fill(0); apply(z, r), cg.rs:196-197)."""
        check(L.lib().fx_mg_precondition(self.h, z.storage.handle, r.storage.handle))

    def _handle(self, device: Device) -> int:
        return L.lib().fx_mg_as_precond(self.h)

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_mg_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ------------------------------------------------------------------ solvers

class LinearSolver:
    """linear_solver.rs:13-36"""

    def solve(self, x: Field, b: Field, coeff: float, stencil: Stencil, boundaries: Boundaries) -> SolveStats:
        raise NotImplementedError

    def name(self) -> str:
        raise NotImplementedError


class _Native(LinearSolver):
    _prefix = ""

    def __init__(self, grid: Grid, device: Optional[Device], tol: float, max_iter: int, *extra):
        self.device = device or Device.best()
        self.grid = grid
        self._tol = float(tol)
        self._max_iter = int(max_iter)
        out = C.c_void_p()
        g = grid_c(grid)
        create = getattr(L.lib(), f"fx_{self._prefix}_create")
        check(create(self.device.backend().ctx, C.byref(g), *extra, self._tol, self._max_iter, C.byref(out)))
        self.h = out.value

    # public fields `tol` / `max_iter`, as in the reference structs
    @property
    def tol(self) -> float:
        return self._tol

    @tol.setter
    def tol(self, v: float) -> None:
        self._tol = float(v)
        self._push()

    @property
    def max_iter(self) -> int:
        return self._max_iter

    @max_iter.setter
    def max_iter(self, v: int) -> None:
        self._max_iter = int(v)
        self._push()

    def _push(self):
        check(getattr(L.lib(), f"fx_{self._prefix}_set_params")(self.h, self._tol, self._max_iter))

    def _run(self, fn, x: Field, b: Field, coeff, stencil, boundaries, *extra) -> SolveStats:
        sc = StencilC(stencil)
        bc = bcs_c(boundaries)
        st = L.FxStats()
        check(fn(self.h, x.storage.handle, b.storage.handle, float(coeff), sc.ptr, C.byref(bc), *extra,
                 C.byref(st)))
        return _stats(st)

    def solve(self, x, b, coeff, stencil, boundaries) -> SolveStats:
        return self._run(getattr(L.lib(), f"fx_{self._prefix}_solve"), x, b, coeff, stencil, boundaries)

    def solve_preconditioned(self, x, b, coeff, stencil, boundaries, pc: Preconditioner) -> SolveStats:
        fn = getattr(L.lib(), f"fx_{self._prefix}_solve_preconditioned")
        return self._run(fn, x, b, coeff, stencil, boundaries, pc._handle(self.device))

    def solve_op(self, x: Field, b: Field, op: "ConvDiffOperator", pc: Optional[Preconditioner] = None) -> SolveStats:
        """Solve A x = b for a `ConvDiffOperator` (BiCGSTAB, GMRES and FGMRES only), with an
        optional preconditioner."""
        fn = getattr(L.lib(), f"fx_{self._prefix}_solve_op", None)
        if fn is None:
            raise NotImplementedError(f"{self.name()} does not take a ConvDiffOperator")
        st = L.FxStats()
        check(fn(self.h, x.storage.handle, b.storage.handle, op.h, pc._handle(self.device) if pc else None,
                 C.byref(st)))
        return _stats(st)

    def __del__(self):
        try:
            if self.h:
                getattr(L.lib(), f"fx_{self._prefix}_destroy")(self.h)
                self.h = None
        except Exception:
            pass


class CgSolver(_Native):
    """cg.rs:52-256: matrix-free (P)CG on A v = v + coeff * S v."""

    _prefix = "cg"

    def __init__(self, grid: Grid, device: Optional[Device] = None, tol: float = 1e-8, max_iter: int = 500):
        super().__init__(grid, device, tol, max_iter)

    def name(self) -> str:
        return "CG"


class PipelinedCgSolver(_Native):
    """pipelined_cg.rs:25-237 (Ghysels-Vanroose).  `solve` is the reference's unpreconditioned
    method; `solve_preconditioned` is new: the preconditioned form of the same method (Ghysels &
    Vanroose 2014, Algorithm 4), one preconditioner application and one fused pass per iteration,
    stopping on ||r||_2 < tol as CgSolver does."""

    _prefix = "pipelined_cg"

    def __init__(self, grid: Grid, device: Optional[Device] = None, tol: float = 1e-8, max_iter: int = 500):
        super().__init__(grid, device, tol, max_iter)

    def name(self) -> str:
        return "PipelinedCG"


class MixedPrecisionRefinement:
    """FP64 iterative refinement around FP32 preconditioned CG (new: the reference has no
    refinement loop).  Each outer step computes r = b - A x and ||r||_2 in FP64, stops when
    ||r||_2 < tol or after `max_outer` corrections, and otherwise solves A d = r on FP32 vectors
    with the preconditioner (an FP32 vertex multigrid) until ||r_inner||_2 < inner_tol ||r||_2,
    then updates x += d in FP64.  Inner products and CG scalars stay compensated FP64.  x and b
    are FP64 fields; `last_inner_iterations` holds the inner CG iterations of the last solve."""

    def __init__(self, grid: Grid, device: Optional[Device] = None, tol: float = 1e-8, max_outer: int = 20,
                 inner_tol: float = 1e-4, inner_max_iter: int = 100):
        self.device = device or Device.best()
        self.grid = grid
        self.tol, self.max_outer = float(tol), int(max_outer)
        self.inner_tol, self.inner_max_iter = float(inner_tol), int(inner_max_iter)
        self.last_inner_iterations = 0
        out = C.c_void_p()
        g = grid_c(grid)
        check(L.lib().fx_ir_create(self.device.backend().ctx, C.byref(g), self.tol, self.max_outer,
                                   self.inner_tol, self.inner_max_iter, C.byref(out)))
        self.h = out.value

    def solve_preconditioned(self, x, b, coeff, stencil, boundaries, pc: Preconditioner) -> SolveStats:
        sc = StencilC(stencil)
        bc = bcs_c(boundaries)
        st = L.FxStats()
        inner = C.c_size_t()
        check(L.lib().fx_ir_solve_preconditioned(self.h, x.storage.handle, b.storage.handle, float(coeff), sc.ptr,
                                                 C.byref(bc), pc._handle(self.device), C.byref(st), C.byref(inner)))
        self.last_inner_iterations = int(inner.value)
        return _stats(st)

    def name(self) -> str:
        return "FP64 refinement / FP32 PCG"

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_ir_destroy(self.h)
                self.h = None
        except Exception:
            pass


class BiCgStabSolver(_Native):
    """bicgstab.rs:19-346."""

    _prefix = "bicgstab"

    def __init__(self, grid: Grid, device: Optional[Device] = None, tol: float = 1e-8, max_iter: int = 500):
        super().__init__(grid, device, tol, max_iter)

    def name(self) -> str:
        return "BiCGSTAB"


class ConvDiffOperator:
    """Convection-diffusion operator for `BiCgStabSolver`, `GmresSolver` and `FgmresSolver`
    (``solve_op``; new, the reference's solvers take only v + coeff S v):
    A v = sigma v + coeff (kappa Lap v + vx dv/dx + vy dv/dy) inside, first-order upwind on the
    sign of v as ``apply_conv_diff`` (backend.rs:375-384), A v = v on the ring.  sigma = 1 is
    the implicit-step operator, sigma = 0 the steady one.  ``kappa`` is an F64 `Field` or a
    float; ``vx``, ``vy`` are F64 fields, kept alive by the operator."""

    def __init__(self, grid: Grid, vx: Field, vy: Field, kappa, sigma: float = 1.0, coeff: float = 1.0):
        self.device = vx.device()
        self.grid = grid
        kf = kappa if isinstance(kappa, Field) else None
        ks = 0.0 if kf is not None else float(kappa)
        self._keep = (vx, vy, kf)
        g = grid_c(grid)
        out = C.c_void_p()
        check(L.lib().fx_op_conv_diff(self.device.backend().ctx, C.byref(g), float(sigma), float(coeff),
                                      kf.storage.handle if kf is not None else None, ks, vx.storage.handle,
                                      vy.storage.handle, C.byref(out)))
        self.h = out.value

    def apply(self, v: Field, out: Field) -> None:
        """out = A v."""
        check(L.lib().fx_op_apply(self.h, v.storage.handle, out.storage.handle))

    def jacobi(self) -> "OperatorJacobi":
        return OperatorJacobi(self)

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_op_destroy(self.h)
                self.h = None
        except Exception:
            pass


class ConvDiffMultigrid(Preconditioner):
    """Multigrid V-cycle preconditioner for a `ConvDiffOperator` (fx_cdmg_*; new): vertex
    hierarchy, each coarse level the operator rediscretised with h doubled and the fields
    injected from the coincident fine points, weighted Jacobi with the operator's diagonal,
    full weighting / bilinear transfers, `coarse_sweeps` sweeps on the coarsest level, one
    cycle from z = 0 per application."""

    def __init__(self, op: "ConvDiffOperator", n_pre: int = 2, n_post: int = 2, omega: float = 0.8,
                 coarse_max: int = 15, coarse_sweeps: int = 200, dtype: DType = DType.F64):
        """``dtype=DType.F32`` runs the cycle in single precision (fx_cdmg_create_typed); the
        vectors it is applied to stay F64."""
        self._op = op  # the cycle reads the operator's fields
        out = C.c_void_p()
        check(L.lib().fx_cdmg_create_typed(op.h, int(n_pre), int(n_post), float(omega), int(coarse_max),
                                           int(coarse_sweeps), int(dtype), C.byref(out)))
        self.h = out.value
        self.dtype = DType(dtype)

    def depth(self) -> int:
        d = C.c_size_t()
        check(L.lib().fx_cdmg_depth(self.h, C.byref(d)))
        return d.value

    def set_replay(self, enabled: bool) -> None:
        """Record each (z, r) pair's cycle into a CUDA graph once and replay it
        (fx_cdmg_set_replay; off by default)."""
        check(L.lib().fx_cdmg_set_replay(self.h, 1 if enabled else 0))

    def set_learned(self, smoother, min_points: int = 4096, fallback_ratio: float = 0.9, max_points: int = 0) -> None:
        """Smooth every level of `min_points` to `max_points` points (0: no bound; the coarsest
        excepted) with the learned smoother (`fluxion_b200.learned.LearnedSmoother`) in place of the
        Jacobi sweeps; each application whose ||r - A z|| exceeds fallback_ratio ||r|| is recomputed
        by the plain cycle on the device (fx_cdmg_set_learned).  None switches it off."""
        self._lsm = smoother
        check(L.lib().fx_cdmg_set_learned(self.h, smoother.h if smoother is not None else None, int(min_points),
                                          int(max_points), float(fallback_ratio)))

    def set_learned_patience(self, patience: int) -> None:
        """After `patience` fallbacks in a row the learned cycle is switched off for good (until
        set_learned or this call); 0 never switches it off (fx_cdmg_set_learned_patience)."""
        check(L.lib().fx_cdmg_set_learned_patience(self.h, int(patience)))

    def learned_disabled(self) -> bool:
        """Whether the patience has switched the learned cycle off."""
        d = C.c_int()
        check(L.lib().fx_cdmg_learned_disabled(self.h, C.byref(d)))
        return bool(d.value)

    def learned_stats(self):
        """(checked applications, fallbacks to the plain cycle) so far."""
        a, f = C.c_ulonglong(), C.c_ulonglong()
        check(L.lib().fx_cdmg_learned_stats(self.h, C.byref(a), C.byref(f)))
        return a.value, f.value

    def _handle(self, device: Device) -> int:
        return L.lib().fx_cdmg_as_precond(self.h)

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_cdmg_destroy(self.h)
                self.h = None
        except Exception:
            pass


class OperatorJacobi(Preconditioner):
    """z = r / diag(A) for a `ConvDiffOperator` (fx_precond_jacobi_op)."""

    def __init__(self, op: ConvDiffOperator):
        self._op = op  # the native preconditioner reads the operator
        out = C.c_void_p()
        check(L.lib().fx_precond_jacobi_op(op.h, C.byref(out)))
        self.h = out.value

    def _handle(self, device: Device) -> int:
        return self.h

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_precond_destroy(self.h)
                self.h = None
        except Exception:
            pass


class InnerCg(Preconditioner):
    """Inner-CG preconditioner (new): the k-th application runs ``steps[k % len(steps)]`` CG
    steps on (I + coeff S) z = r from z = 0 (preconditioned by ``inner`` when given), tolerance
    0.  With a schedule of different counts it changes from one application to the next, the
    case `FcgSolver` and `FgmresSolver` are for."""

    def __init__(self, grid: Grid, coeff: float, stencil: Stencil, boundaries: Boundaries, steps,
                 inner: Optional[Preconditioner] = None, device: Optional[Device] = None):
        self.device = device or Device.best()
        self._inner = inner  # kept alive: the native object holds its handle
        sched = (C.c_size_t * len(steps))(*[int(k) for k in steps])
        sc = StencilC(stencil)
        g, bc = grid_c(grid), bcs_c(boundaries)
        out = C.c_void_p()
        check(L.lib().fx_precond_inner_cg(self.device.backend().ctx, C.byref(g), float(coeff), sc.ptr, C.byref(bc),
                                          sched, len(steps), inner._handle(self.device) if inner else None,
                                          C.byref(out)))
        self.h = out.value

    def _handle(self, device: Device) -> int:
        return self.h

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_precond_destroy(self.h)
                self.h = None
        except Exception:
            pass


class InnerPcgF32(Preconditioner):
    """Inner FP32 PCG preconditioner (new): z = the FP32 solution of (I + coeff S) d = r by CG
    preconditioned by ``inner_f32`` (an FP32 `Multigrid.vertex`), from d = 0 to
    ||r - A d|| < rel_tol ||r|| or max_iter iterations (fx_precond_inner_pcg_f32).  For
    `FcgSolver` / `FgmresSolver`: FP64 outer Krylov, FP32 inner solves."""

    def __init__(self, grid: Grid, coeff: float, stencil: Stencil, boundaries: Optional[Boundaries],
                 inner_f32: Preconditioner, rel_tol: float = 1e-4, max_iter: int = 100,
                 device: Optional[Device] = None):
        self.device = device or Device.best()
        self._inner = inner_f32  # kept alive: the native object borrows its handle
        sc = StencilC(stencil)
        g, bc = grid_c(grid), bcs_c(boundaries if boundaries is not None else Boundaries.zero_dirichlet())
        out = C.c_void_p()
        check(L.lib().fx_precond_inner_pcg_f32(self.device.backend().ctx, C.byref(g), float(coeff), sc.ptr,
                                               C.byref(bc), inner_f32._handle(self.device), float(rel_tol),
                                               int(max_iter), C.byref(out)))
        self.h = out.value

    def stats(self):
        """(applications, inner FP32 CG iterations) so far."""
        a, i = C.c_size_t(), C.c_size_t()
        check(L.lib().fx_precond_inner_pcg_f32_stats(self.h, C.byref(a), C.byref(i)))
        return a.value, i.value

    def _handle(self, device: Device) -> int:
        return self.h

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_precond_destroy(self.h)
                self.h = None
        except Exception:
            pass


class FcgSolver(_Native):
    """Flexible CG (new; the reference has none): PCG with the Polak-Ribiere beta
    z_{k+1}.(r_{k+1} - r_k) / (z_k.r_k) (Golub & Ye 1999; Notay 2000), safe with a
    preconditioner that changes between applications.  Same fields, signatures and stop test as
    `CgSolver`; with a fixed SPD preconditioner it takes the same iterations."""

    _prefix = "fcg"

    def __init__(self, grid: Grid, device: Optional[Device] = None, tol: float = 1e-8, max_iter: int = 500):
        super().__init__(grid, device, tol, max_iter)

    def name(self) -> str:
        return "FCG"


class FgmresSolver(_Native):
    """Flexible GMRES(m) (new; Saad 1993): right preconditioning with the preconditioned
    directions kept, so the preconditioner may change between applications; it stops on the
    true ||b - A x||_2 < tol.  Without a preconditioner it is `GmresSolver` step for step."""

    _prefix = "fgmres"

    def __init__(self, grid: Grid, device: Optional[Device] = None, restart: int = 30, tol: float = 1e-8,
                 max_iter: int = 500):
        self.restart = int(restart)
        super().__init__(grid, device, tol, max_iter, C.c_size_t(self.restart))

    def name(self) -> str:
        return "FGMRES"

    def set_orthogonalization(self, method: str) -> None:
        """"mgs" (default, the reference's) or "cgs2" (classical Gram-Schmidt twice: three passes
        over the basis per Arnoldi step; restart <= 32)."""
        check(L.lib().fx_fgmres_set_orthogonalization(self.h, {"mgs": 0, "cgs2": 1}[method]))


class GmresSolver(_Native):
    """gmres.rs:24-491: restarted GMRES(m) with modified Gram-Schmidt."""

    _prefix = "gmres"

    def __init__(self, grid: Grid, device: Optional[Device] = None, restart: int = 30, tol: float = 1e-8,
                 max_iter: int = 500):
        self.restart = int(restart)
        super().__init__(grid, device, tol, max_iter, C.c_size_t(self.restart))

    def name(self) -> str:
        return "GMRES"
