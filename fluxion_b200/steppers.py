"""Time steppers of fluxion's runtime over the CUDA solve path.

``CrankNicolsonSolver`` (crates/runtime/src/implicit.rs:25-237), ``BdfSolver`` (bdf.rs:23-255),
``ImexSolver`` (imex.rs:26-273) and the explicit ``DiffusionSolver`` (solver.rs:30-642) restate
the reference's steppers.  The implicit ones: each step assembles its
right-hand side from the backend's field operations in the reference's order and solves the
implicit system with `CgSolver` (preconditioned by a reference-hierarchy `Multigrid` when one
is configured).  Same constructors, fields and step signatures as the reference.
"""
from __future__ import annotations

import enum
from typing import List, Optional

from .core import Boundaries, DType, Grid, Stencil
from .field import Device, Field
from .solvers import CgSolver, Multigrid, SmootherKind, SolveStats


class CrankNicolsonSolver:
    """implicit.rs:25-237: du/dt = alpha Lap u + source by
    (I - dt/2 alpha Lap) u^{n+1} = (I + dt/2 alpha Lap) u^n + dt source, solved by (P)CG."""

    def __init__(self, grid: Grid, alpha: float, dt: float, boundaries: Boundaries, device: Optional[Device] = None,
                 cg_tol: float = 1e-8, cg_max_iter: int = 100, mg: Optional[Multigrid] = None):
        self.device = device or Device.best()
        self.grid = grid
        self.stencil = Stencil.laplacian_2d_5pt(grid.dx, grid.dy)
        self.boundaries = boundaries
        self.cg = CgSolver(grid, self.device, cg_tol, cg_max_iter)
        self.mg = mg
        self.rhs = Field.zeros(grid, DType.F64, self.device)
        self.tmp = Field.zeros(grid, DType.F64, self.device)
        self._dt = float(dt)
        self.alpha = float(alpha)
        self._steps_done = 0

    @staticmethod
    def new(grid, alpha, dt, boundaries, device, cg_tol, cg_max_iter) -> "CrankNicolsonSolver":
        return CrankNicolsonSolver(grid, alpha, dt, boundaries, device, cg_tol, cg_max_iter)

    @staticmethod
    def with_multigrid(grid, alpha, dt, boundaries, device, cg_tol, cg_max_iter, mg_pre, mg_post,
                       mg_omega) -> "CrankNicolsonSolver":
        return CrankNicolsonSolver.with_multigrid_smoother(grid, alpha, dt, boundaries, device, cg_tol, cg_max_iter,
                                                           mg_pre, mg_post, mg_omega, SmootherKind.Jacobi)

    @staticmethod
    def with_multigrid_smoother(grid, alpha, dt, boundaries, device, cg_tol, cg_max_iter, mg_pre, mg_post, mg_omega,
                                smoother: SmootherKind) -> "CrankNicolsonSolver":
        device = device or Device.best()
        mg = Multigrid.build(grid, boundaries, device, mg_pre, mg_post, mg_omega, smoother)
        return CrankNicolsonSolver(grid, alpha, dt, boundaries, device, cg_tol, cg_max_iter, mg)

    def dt(self) -> float:
        return self._dt

    def steps_done(self) -> int:
        return self._steps_done

    def sim_time(self) -> float:
        return self._steps_done * self._dt

    def step(self, u: Field, source: Optional[Field] = None) -> SolveStats:
        """implicit.rs:178-226: rhs = u + dt/2 alpha Lap u (+ dt source), then solve with
        coeff = -dt/2 alpha from u^n as the initial guess."""
        half_dt_alpha = 0.5 * self._dt * self.alpha
        self.rhs.copy_from(u)
        self.tmp.copy_from(u)
        self.rhs.stencil_axpy(half_dt_alpha, self.tmp, self.stencil, self.boundaries)
        if source is not None:
            self.rhs.axpy(self._dt, source)
        if self.mg is not None:
            stats = self.cg.solve_preconditioned(u, self.rhs, -half_dt_alpha, self.stencil, self.boundaries, self.mg)
        else:
            stats = self.cg.solve(u, self.rhs, -half_dt_alpha, self.stencil, self.boundaries)
        self._steps_done += 1
        return stats

    def step_n(self, u: Field, n: int) -> None:
        for _ in range(n):
            self.step(u, None)


def bdf_coeffs(order: int):
    """bdf.rs:41-63: (history coefficients a_1.., lhs coefficient a_0) of BDF1-BDF4."""
    return {
        1: ([-1.0], 1.0),
        2: ([-2.0, 0.5], 1.5),
        3: ([-3.0, 1.5, -1.0 / 3.0], 11.0 / 6.0),
        4: ([-4.0, 3.0, -4.0 / 3.0, 0.25], 25.0 / 12.0),
    }[order]


class BdfSolver:
    """bdf.rs:23-255: BDF1-BDF4 for du/dt = alpha Lap u, the order ramping up from 1 while the
    history fills; each step solves (I + coeff Lap) u^{n+1} = rhs / a_0 with
    coeff = -dt alpha / a_0 by (P)CG."""

    def __init__(self, grid: Grid, alpha: float, dt: float, order: int, boundaries: Boundaries,
                 device: Optional[Device] = None, cg_tol: float = 1e-8, cg_max_iter: int = 100,
                 mg: Optional[Multigrid] = None):
        if not 1 <= int(order) <= 4:
            raise ValueError(f"BDF order must be 1-4, got {order}")
        self.device = device or Device.best()
        self.grid = grid
        self.stencil = Stencil.laplacian_2d_5pt(grid.dx, grid.dy)
        self.boundaries = boundaries
        self.cg = CgSolver(grid, self.device, cg_tol, cg_max_iter)
        self.mg = mg
        self.history: List[Field] = [Field.zeros(grid, DType.F64, self.device) for _ in range(int(order))]
        self.rhs = Field.zeros(grid, DType.F64, self.device)
        self._dt = float(dt)
        self.alpha = float(alpha)
        self._order = int(order)
        self._steps_done = 0

    @staticmethod
    def new(grid, alpha, dt, order, boundaries, device, cg_tol, cg_max_iter) -> "BdfSolver":
        return BdfSolver(grid, alpha, dt, order, boundaries, device, cg_tol, cg_max_iter)

    @staticmethod
    def with_multigrid(grid, alpha, dt, order, boundaries, device, cg_tol, cg_max_iter, mg_pre, mg_post,
                       mg_omega) -> "BdfSolver":
        device = device or Device.best()
        mg = Multigrid.new(grid, boundaries, device, mg_pre, mg_post, mg_omega)
        return BdfSolver(grid, alpha, dt, order, boundaries, device, cg_tol, cg_max_iter, mg)

    def dt(self) -> float:
        return self._dt

    def order(self) -> int:
        return self._order

    def steps_done(self) -> int:
        return self._steps_done

    def sim_time(self) -> float:
        return self._steps_done * self._dt

    def step(self, u: Field) -> SolveStats:
        """bdf.rs:171-244."""
        eff_order = min(self._order, self._steps_done + 1)
        hist, lhs = bdf_coeffs(eff_order)
        self.rhs.copy_from(u)
        self.rhs.scale(-hist[0])
        for i, c in enumerate(hist[1:], start=1):
            self.rhs.axpy(-c, self.history[i - 1])
        coeff = -self._dt * self.alpha / lhs
        self.rhs.scale(1.0 / lhs)
        for i in range(len(self.history) - 1, 0, -1):
            self.history[i].copy_from(self.history[i - 1])
        if self.history:
            self.history[0].copy_from(u)
        if self.mg is not None:
            stats = self.cg.solve_preconditioned(u, self.rhs, coeff, self.stencil, self.boundaries, self.mg)
        else:
            stats = self.cg.solve(u, self.rhs, coeff, self.stencil, self.boundaries)
        self._steps_done += 1
        return stats

    def step_n(self, u: Field, n: int) -> None:
        for _ in range(n):
            self.step(u)


class ImexSolver:
    """imex.rs:26-273: convection explicit, diffusion implicit.  conv = v . grad u by the upwind
    convection-diffusion operator with a zero kappa field; rhs = u + dt/2 kappa Lap u + dt conv;
    solve (I - dt/2 kappa Lap) u^{n+1} = rhs by (P)CG.  Constant velocity (vx, vy)."""

    def __init__(self, grid: Grid, kappa: float, vx_val: float, vy_val: float, dt: float, boundaries: Boundaries,
                 device: Optional[Device] = None, cg_tol: float = 1e-8, cg_max_iter: int = 100,
                 mg: Optional[Multigrid] = None):
        self.device = device or Device.best()
        self.grid = grid
        self.stencil = Stencil.laplacian_2d_5pt(grid.dx, grid.dy)
        self.boundaries = boundaries
        self.cg = CgSolver(grid, self.device, cg_tol, cg_max_iter)
        self.mg = mg
        self.rhs = Field.zeros(grid, DType.F64, self.device)
        self.conv = Field.zeros(grid, DType.F64, self.device)
        self.kappa_zero = Field.zeros(grid, DType.F64, self.device)
        self.vx = Field.zeros(grid, DType.F64, self.device)
        self.vx.fill(vx_val)
        self.vy = Field.zeros(grid, DType.F64, self.device)
        self.vy.fill(vy_val)
        self._dt = float(dt)
        self.kappa = float(kappa)
        self._steps_done = 0

    @staticmethod
    def new(grid, kappa, vx_val, vy_val, dt, boundaries, device, cg_tol, cg_max_iter) -> "ImexSolver":
        return ImexSolver(grid, kappa, vx_val, vy_val, dt, boundaries, device, cg_tol, cg_max_iter)

    @staticmethod
    def with_multigrid(grid, kappa, vx_val, vy_val, dt, boundaries, device, cg_tol, cg_max_iter, mg_pre, mg_post,
                       mg_omega) -> "ImexSolver":
        device = device or Device.best()
        mg = Multigrid.new(grid, boundaries, device, mg_pre, mg_post, mg_omega)
        return ImexSolver(grid, kappa, vx_val, vy_val, dt, boundaries, device, cg_tol, cg_max_iter, mg)

    def dt(self) -> float:
        return self._dt

    def steps_done(self) -> int:
        return self._steps_done

    def sim_time(self) -> float:
        return self._steps_done * self._dt

    def step(self, u: Field) -> SolveStats:
        """imex.rs:152-202."""
        half_dt_kappa = 0.5 * self._dt * self.kappa
        u.apply_conv_diff_into(self.kappa_zero, self.vx, self.vy, self.boundaries, self.conv)  # :219-273
        self.rhs.copy_from(u)
        self.rhs.stencil_axpy(half_dt_kappa, u, self.stencil, self.boundaries)
        self.rhs.axpy(self._dt, self.conv)
        coeff = -half_dt_kappa
        if self.mg is not None:
            stats = self.cg.solve_preconditioned(u, self.rhs, coeff, self.stencil, self.boundaries, self.mg)
        else:
            stats = self.cg.solve(u, self.rhs, coeff, self.stencil, self.boundaries)
        self._steps_done += 1
        return stats

    def step_n(self, u: Field, n: int) -> None:
        for _ in range(n):
            self.step(u)


class TimeScheme(enum.Enum):
    """solver.rs:16-24"""

    Euler = 0
    Rk2 = 1
    Rk4 = 2


class DiffusionSolver:
    """solver.rs:30-642: explicit du/dt = alpha Lap u (+ source) by forward Euler, Heun (RK2) or
    classical RK4, each stage the reference's sequence of field operations.  The default dt is
    the reference's stability bound safety * h_min^2 / (4 alpha) (safety 0.4 / 0.8 / 1.4).
    ``enable_graph()`` is the HipGraph path (solver.rs:182-325) on CUDA graphs: the first
    ``step_n`` records one step on the backend's stream and later steps replay it."""

    def __init__(self, grid: Grid, alpha: float, dt: Optional[float], boundaries: Boundaries,
                 scheme: "TimeScheme", device: Optional[Device] = None):
        self.device = device or Device.best()
        self.grid = grid
        h_min = min(grid.dx, grid.dy)
        safety = {TimeScheme.Euler: 0.4, TimeScheme.Rk2: 0.8, TimeScheme.Rk4: 1.4}[scheme]
        self._dt = float(dt) if dt is not None else safety * h_min * h_min / (4.0 * alpha)
        self.alpha = float(alpha)
        self.stencil = Stencil.laplacian_2d_5pt(grid.dx, grid.dy)
        self.boundaries = boundaries
        self._scheme = scheme
        n_scratch = {TimeScheme.Euler: 1, TimeScheme.Rk2: 2, TimeScheme.Rk4: 5}[scheme]
        self.scratch = [Field.zeros(grid, DType.F64, self.device) for _ in range(n_scratch)]
        self._steps_done = 0
        self._use_graph = False
        self._graph = None
        self._graph_u = None

    @staticmethod
    def new(grid: Grid, alpha: float, dt: Optional[float], device: Optional[Device] = None) -> "DiffusionSolver":
        return DiffusionSolver(grid, alpha, dt, Boundaries.zero_dirichlet(), TimeScheme.Euler, device)

    @staticmethod
    def with_boundaries(grid, alpha, dt, boundaries, device=None) -> "DiffusionSolver":
        return DiffusionSolver(grid, alpha, dt, boundaries, TimeScheme.Euler, device)

    @staticmethod
    def build(grid, alpha, dt, boundaries, scheme, device=None) -> "DiffusionSolver":
        return DiffusionSolver(grid, alpha, dt, boundaries, scheme, device)

    def dt(self) -> float:
        return self._dt

    def steps_done(self) -> int:
        return self._steps_done

    def sim_time(self) -> float:
        return self._steps_done * self._dt

    def scheme(self) -> "TimeScheme":
        return self._scheme

    def enable_graph(self) -> None:
        """solver.rs:182-186 (enable_hip_graph)."""
        self._use_graph = True

    def step(self, u: Field, source: Optional[Field] = None) -> None:
        self._record(u, source)
        self._steps_done += 1

    def step_n(self, u: Field, n: int) -> None:
        """solver.rs:231-257; with the graph enabled, the recorded step is replayed n times
        (one graph per solver, recorded on the first field passed)."""
        if n == 0:
            return
        if self._use_graph:
            if self._graph is None:
                be = self.device.backend()
                be.graph_begin()
                try:
                    self._record(u, None)
                finally:
                    self._graph = be.graph_end()
                self._graph_u = u
            if u is not self._graph_u:
                raise ValueError("the recorded step belongs to another field")
            for _ in range(n):
                self._graph.launch()
                self._steps_done += 1
            return
        for _ in range(n):
            self.step(u, None)

    def step_n_with_source(self, u: Field, n: int, source: Field) -> None:
        for _ in range(n):
            self.step(u, source)

    def _record(self, u: Field, source: Optional[Field]) -> None:
        {TimeScheme.Euler: self._euler, TimeScheme.Rk2: self._rk2, TimeScheme.Rk4: self._rk4}[self._scheme](u, source)

    def _euler(self, u: Field, source: Optional[Field]) -> None:  # solver.rs:344-369
        coeff = self.alpha * self._dt
        self.scratch[0].copy_from(u)
        u.stencil_axpy(coeff, self.scratch[0], self.stencil, self.boundaries)
        if source is not None:
            u.axpy(self._dt, source)

    def _rk2(self, u: Field, source: Optional[Field]) -> None:  # solver.rs:371-419
        dt = self._dt
        coeff = dt * self.alpha
        self.scratch[1].copy_from(u)
        for _ in range(2):
            self.scratch[0].copy_from(u)
            u.stencil_axpy(coeff, self.scratch[0], self.stencil, self.boundaries)
            if source is not None:
                u.axpy(dt, source)
        u.axpy(1.0, self.scratch[1])
        u.scale(0.5)

    def _rk4(self, u: Field, source: Optional[Field]) -> None:  # solver.rs:421-495
        dt, alpha = self._dt, self.alpha
        k, u_old = self.scratch, self.scratch[4]
        u_old.copy_from(u)
        u.apply_stencil_into(self.stencil, self.boundaries, k[0])
        u.copy_from(u_old)
        u.stencil_axpy(0.5 * dt * alpha, u_old, self.stencil, self.boundaries)
        u.apply_stencil_into(self.stencil, self.boundaries, k[1])
        u.copy_from(u_old)
        u.axpy(0.5 * dt * alpha, k[1])
        u.zero_boundaries()
        u.apply_stencil_into(self.stencil, self.boundaries, k[2])
        u.copy_from(u_old)
        u.axpy(dt * alpha, k[2])
        u.zero_boundaries()
        u.apply_stencil_into(self.stencil, self.boundaries, k[3])
        u.copy_from(u_old)
        c = dt * alpha / 6.0
        u.axpy(c, k[0])
        u.axpy(2.0 * c, k[1])
        u.axpy(2.0 * c, k[2])
        u.axpy(c, k[3])
        if source is not None:
            u.axpy(dt, source)
