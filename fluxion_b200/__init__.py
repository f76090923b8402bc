"""fluxion_b200 -- B200 (sm_100a) backend for fluxion's matrix-free solve path.

Hand-written CUDA kernels behind a C ABI (``include/fluxion_cuda.h``,
``libfluxion_cuda.so``) that mirrors the reference's ``Backend`` trait and
solver structs; this package is the Python view of that ABI with the
reference's type and method names.
"""
from .core import (BackendError, BcKind, Boundaries, BoundaryCondition, CoreError, DimensionMismatch, DType,
                   Grid, InvalidGrid, InvalidStencil, Stencil, StencilEntry)

__all__ = [
    "BackendError", "BcKind", "Boundaries", "BoundaryCondition", "CoreError", "DimensionMismatch", "DType",
    "Grid", "InvalidGrid", "InvalidStencil", "Stencil", "StencilEntry",
    "CudaBackend", "CudaBuffer", "BackendUnavailable", "InvalidArgument", "Device", "Field", "DeviceMismatch",
    "CgSolver", "CgStats", "PipelinedCgSolver", "BiCgStabSolver", "GmresSolver", "Multigrid", "SmootherKind",
    "Identity", "Preconditioner", "LinearSolver", "SolveStats", "ConvergenceReason",
    "MixedPrecisionRefinement", "CudaGraph", "FcgSolver", "FgmresSolver", "InnerCg", "InnerPcgF32",
    "ConvDiffOperator", "OperatorJacobi", "ConvDiffMultigrid",
    "CrankNicolsonSolver", "BdfSolver", "ImexSolver", "DiffusionSolver", "TimeScheme",
]


def __getattr__(name):
    # The backend-facing classes load libfluxion_cuda.so; import them lazily so that the
    # core data types stay importable where the library has not been built.
    if name in ("CudaBackend", "CudaBuffer", "BackendUnavailable", "InvalidArgument", "CudaGraph"):
        from . import backend
        return getattr(backend, name)
    if name in ("Device", "Field", "DeviceMismatch"):
        from . import field
        return getattr(field, name)
    if name in ("CgSolver", "CgStats", "PipelinedCgSolver", "BiCgStabSolver", "GmresSolver", "Multigrid",
                "MixedPrecisionRefinement", "FcgSolver", "FgmresSolver", "InnerCg", "InnerPcgF32",
                "ConvDiffOperator", "OperatorJacobi", "ConvDiffMultigrid", "SmootherKind", "Identity", "Preconditioner", "LinearSolver", "SolveStats",
                "ConvergenceReason"):
        from . import solvers
        return getattr(solvers, name)
    if name in ("CrankNicolsonSolver", "BdfSolver", "ImexSolver", "DiffusionSolver", "TimeScheme"):
        from . import steppers
        return getattr(steppers, name)
    raise AttributeError(name)
