"""Core data types of the solve path, mirroring ``crates/core`` of fluxion.

``Grid`` (crates/core/src/grid.rs:3-62), ``StencilEntry`` / ``Stencil``
(crates/core/src/stencil.rs:1-239), ``BoundaryCondition`` / ``Boundaries``
(crates/core/src/boundary.rs:1-44), ``DType`` (crates/core/src/dtype.rs:1-15)
and the ``CoreError`` family (crates/core/src/error.rs:1-20).  Same names,
argument meaning and error behaviour as the reference, so that callers of
the reference API find the same surface here.
"""
from __future__ import annotations

import enum
import math
from dataclasses import dataclass
from typing import List, Sequence, Tuple


# ----------------------------------------------------------------- errors

class CoreError(Exception):
    """crates/core/src/error.rs:4-20."""


class DimensionMismatch(CoreError):
    def __init__(self, expected: int, got: int):
        super().__init__(f"dimension mismatch: expected {expected}, got {got}")
        self.expected = expected
        self.got = got


class InvalidGrid(CoreError):
    def __init__(self, msg: str):
        super().__init__(f"invalid grid: {msg}")


class InvalidStencil(CoreError):
    def __init__(self, msg: str):
        super().__init__(f"invalid stencil: {msg}")


class BackendError(CoreError):
    def __init__(self, msg: str):
        super().__init__(f"backend error: {msg}")


# ----------------------------------------------------------------- dtype

class DType(enum.IntEnum):
    """crates/core/src/dtype.rs:2-15.  Values match the C ABI (FX_F32=0, FX_F64=1)."""

    F32 = 0
    F64 = 1

    def size_bytes(self) -> int:
        return 4 if self is DType.F32 else 8


# ----------------------------------------------------------------- grid

@dataclass(frozen=True)
class Grid:
    """Structured 2D grid; ``rows x cols`` includes the boundary ring (grid.rs:4-9)."""

    rows: int
    cols: int
    dx: float
    dy: float

    def __post_init__(self):
        # grid.rs:15-36
        if self.rows < 3 or self.cols < 3:
            raise InvalidGrid(f"minimum 3x3, got {self.rows}x{self.cols}")
        if (not math.isfinite(self.dx) or not math.isfinite(self.dy)
                or self.dx <= 0.0 or self.dy <= 0.0):
            raise InvalidGrid(
                f"spacing must be finite and positive, got dx={self.dx}, dy={self.dy}")

    @staticmethod
    def new(rows: int, cols: int, dx: float, dy: float) -> "Grid":
        return Grid(int(rows), int(cols), float(dx), float(dy))

    @staticmethod
    def square(n: int, h: float) -> "Grid":
        return Grid(int(n), int(n), float(h), float(h))

    def len(self) -> int:
        return self.rows * self.cols

    def __len__(self) -> int:
        return self.rows * self.cols

    def is_empty(self) -> bool:
        return self.rows == 0 or self.cols == 0

    def idx(self, row: int, col: int) -> int:
        return row * self.cols + col


# ----------------------------------------------------------------- stencil

@dataclass(frozen=True)
class StencilEntry:
    dr: int
    dc: int
    weight: float


class Stencil:
    """Finite-difference stencil as (dr, dc, weight) entries (stencil.rs:5-141)."""

    def __init__(self, entries: Sequence[StencilEntry]):
        entries = list(entries)
        if not entries:
            raise InvalidStencil("stencil must have at least one entry")
        self._entries: List[StencilEntry] = [
            e if isinstance(e, StencilEntry) else StencilEntry(int(e[0]), int(e[1]), float(e[2]))
            for e in entries
        ]

    @staticmethod
    def new(entries: Sequence[StencilEntry]) -> "Stencil":
        return Stencil(entries)

    def entries(self) -> List[StencilEntry]:
        return list(self._entries)

    def len(self) -> int:
        return len(self._entries)

    def __len__(self) -> int:
        return len(self._entries)

    def is_empty(self) -> bool:
        return not self._entries

    def as_triples(self) -> List[Tuple[int, int, float]]:
        return [(e.dr, e.dc, e.weight) for e in self._entries]

    def __eq__(self, other):
        return isinstance(other, Stencil) and self._entries == other._entries

    def __repr__(self):
        return f"Stencil({self.as_triples()})"

    @staticmethod
    def laplacian_2d_5pt(dx: float, dy: float) -> "Stencil":
        """stencil.rs:143-168."""
        inv_dx2 = 1.0 / (dx * dx)
        inv_dy2 = 1.0 / (dy * dy)
        return Stencil([
            StencilEntry(0, 0, -2.0 * (inv_dx2 + inv_dy2)),
            StencilEntry(-1, 0, inv_dy2),
            StencilEntry(1, 0, inv_dy2),
            StencilEntry(0, -1, inv_dx2),
            StencilEntry(0, 1, inv_dx2),
        ])

    @staticmethod
    def laplacian_2d_9pt(dx: float, dy: float) -> "Stencil":
        """Mehrstellen (Collatz) compact 9-point Laplacian, stencil.rs:170-238."""
        inv_dx2 = 1.0 / (dx * dx)
        inv_dy2 = 1.0 / (dy * dy)
        dx2 = dx * dx
        dy2 = dy * dy
        k = (dx2 + dy2) / 12.0
        inv_dx2dy2 = inv_dx2 * inv_dy2
        w_c = -2.0 * (inv_dx2 + inv_dy2) + 4.0 * k * inv_dx2dy2
        w_n = inv_dy2 - 2.0 * k * inv_dx2dy2
        w_w = inv_dx2 - 2.0 * k * inv_dx2dy2
        w_diag = k * inv_dx2dy2
        return Stencil([
            StencilEntry(0, 0, w_c),
            StencilEntry(-1, 0, w_n), StencilEntry(1, 0, w_n),
            StencilEntry(0, -1, w_w), StencilEntry(0, 1, w_w),
            StencilEntry(-1, -1, w_diag), StencilEntry(-1, 1, w_diag),
            StencilEntry(1, -1, w_diag), StencilEntry(1, 1, w_diag),
        ])

    @staticmethod
    def poisson_neg_laplacian(dx: float, dy: float) -> "Stencil":
        """The stencil ``S`` for which the solver operator ``v + 1*S v`` is ``-Laplacian(v)``.

        The reference solvers always solve ``A v = v + coeff*S v`` (linear_solver.rs:7-22); with
        coeff = 1, centre weight ``2/dx^2 + 2/dy^2 - 1`` and neighbour weights ``-1/dx^2``,
        ``-1/dy^2`` that operator is the 5-point ``-Laplacian``.
        """
        inv_dx2 = 1.0 / (dx * dx)
        inv_dy2 = 1.0 / (dy * dy)
        return Stencil([
            StencilEntry(0, 0, 2.0 * (inv_dx2 + inv_dy2) - 1.0),
            StencilEntry(-1, 0, -inv_dy2),
            StencilEntry(1, 0, -inv_dy2),
            StencilEntry(0, -1, -inv_dx2),
            StencilEntry(0, 1, -inv_dx2),
        ])


# ----------------------------------------------------------------- boundaries

class BcKind(enum.IntEnum):
    DIRICHLET = 0
    NEUMANN = 1
    ROBIN = 2
    PERIODIC = 3


@dataclass(frozen=True)
class BoundaryCondition:
    """boundary.rs:2-15.  Build with the constructors below."""

    kind: BcKind
    a: float = 0.0  # Dirichlet value / Neumann flux / Robin alpha
    b: float = 0.0  # Robin beta
    g: float = 0.0  # Robin g

    @staticmethod
    def Dirichlet(val: float) -> "BoundaryCondition":  # noqa: N802 - reference variant name
        return BoundaryCondition(BcKind.DIRICHLET, float(val))

    @staticmethod
    def Neumann(flux: float) -> "BoundaryCondition":  # noqa: N802
        return BoundaryCondition(BcKind.NEUMANN, float(flux))

    @staticmethod
    def Robin(alpha: float, beta: float, g: float) -> "BoundaryCondition":  # noqa: N802
        return BoundaryCondition(BcKind.ROBIN, float(alpha), float(beta), float(g))

    @staticmethod
    def Periodic() -> "BoundaryCondition":  # noqa: N802
        return BoundaryCondition(BcKind.PERIODIC)

    def as_tuple(self) -> Tuple[int, float, float, float]:
        return (int(self.kind), self.a, self.b, self.g)


@dataclass(frozen=True)
class Boundaries:
    """boundary.rs:17-44: one condition per side."""

    top: BoundaryCondition
    bottom: BoundaryCondition
    left: BoundaryCondition
    right: BoundaryCondition

    @staticmethod
    def uniform(bc: BoundaryCondition) -> "Boundaries":
        return Boundaries(bc, bc, bc, bc)

    @staticmethod
    def zero_dirichlet() -> "Boundaries":
        return Boundaries.uniform(BoundaryCondition.Dirichlet(0.0))

    @staticmethod
    def periodic() -> "Boundaries":
        return Boundaries.uniform(BoundaryCondition.Periodic())

    def sides(self) -> Tuple[BoundaryCondition, ...]:
        return (self.top, self.bottom, self.left, self.right)

    def as_tuples(self):
        return [s.as_tuple() for s in self.sides()]

    def clone(self) -> "Boundaries":
        return self

    def is_zero_dirichlet(self) -> bool:
        return all(s.kind == BcKind.DIRICHLET and s.a == 0.0 for s in self.sides())
