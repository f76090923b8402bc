"""Failure handling made on the host (no GPU fault): a right-hand side holding a NaN or an Inf
stops every solver with Breakdown (the reference's error surface, crates/core/src/error.rs:4-20
and ConvergenceReason, crates/runtime/src/cg.rs:11-18, has no separate case for it; its stop test
would never pass and the solve would run to max_iter), a forced allocation failure returns
FX_ERR_BACKEND from every entry point that allocates and leaves the context usable, and in a batch
a poisoned problem stops alone while the others converge."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


def _poisson(n, dev):
    from fluxion_b200.workloads import poisson_problem, poisson_uniform_rhs
    P = poisson_problem(n)
    return P, poisson_uniform_rhs(n, seed=3)


@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_nonfinite_rhs_stops_every_solver_with_breakdown(dev, bad):
    from fluxion_b200 import (BiCgStabSolver, CgSolver, ConvergenceReason, DType, FcgSolver, FgmresSolver, Field,
                              GmresSolver, MixedPrecisionRefinement, Multigrid, PipelinedCgSolver)
    n = 63
    P, f = _poisson(n, dev)
    f = f.copy()
    f[(n + 2) * 20 + 17] = bad
    tol = 1e-10
    mk = {
        "cg": lambda: (CgSolver(P.grid, dev, tol, 200), None),
        "pcg": lambda: (CgSolver(P.grid, dev, tol, 200), Multigrid.vertex(P.grid, None, dev)),
        "pipelined": lambda: (PipelinedCgSolver(P.grid, dev, tol, 200), None),
        "bicgstab": lambda: (BiCgStabSolver(P.grid, dev, tol, 200), None),
        "gmres": lambda: (GmresSolver(P.grid, dev, 30, tol, 200), None),
        "fgmres": lambda: (FgmresSolver(P.grid, dev, 30, tol, 200), Multigrid.vertex(P.grid, None, dev)),
        "fcg": lambda: (FcgSolver(P.grid, dev, tol, 200), Multigrid.vertex(P.grid, None, dev)),
        "ir": lambda: (MixedPrecisionRefinement(P.grid, dev, tol, 20, 1e-4, 100),
                       Multigrid.vertex(P.grid, None, dev, dtype=DType.F32)),
    }
    for name, make in mk.items():
        solver, pc = make()
        x = Field.zeros(P.grid, DType.F64, dev)
        b = Field.from_f64(P.grid, f, dev)
        if pc is None:
            st = solver.solve(x, b, P.coeff, P.stencil, None)
        else:
            st = solver.solve_preconditioned(x, b, P.coeff, P.stencil, None, pc)
        assert st.reason == ConvergenceReason.Breakdown, (name, st)
        assert st.iterations < 200, (name, st)
    # the context keeps working
    _, good = _poisson(n, dev)
    x = Field.zeros(P.grid, DType.F64, dev)
    st = CgSolver(P.grid, dev, 1e-10 * np.linalg.norm(good), 500).solve(x, Field.from_f64(P.grid, good, dev),
                                                                        P.coeff, P.stencil, None)
    assert st.converged()


def test_forced_allocation_failure_is_an_error_and_the_context_survives(dev):
    from fluxion_b200 import BackendError, CgSolver, DType, Field, Multigrid
    from fluxion_b200 import _lib as L
    n = 63
    P, f = _poisson(n, dev)
    try:
        L.lib().fx_test_fail_allocations(1)
        with pytest.raises(BackendError):
            Field.zeros(P.grid, DType.F64, dev)
        Field.zeros(P.grid, DType.F64, dev)  # the next one works
        for k in (1, 2, 3):  # solver and multigrid creation fail at their k-th allocation
            L.lib().fx_test_fail_allocations(k)
            with pytest.raises(BackendError):
                CgSolver(P.grid, dev, 1e-10, 100)
            L.lib().fx_test_fail_allocations(k)
            with pytest.raises(BackendError):
                Multigrid.vertex(P.grid, None, dev)
    finally:
        L.lib().fx_test_fail_allocations(0)
    x = Field.zeros(P.grid, DType.F64, dev)
    st = CgSolver(P.grid, dev, 1e-10 * np.linalg.norm(f), 100).solve_preconditioned(
        x, Field.from_f64(P.grid, f, dev), P.coeff, P.stencil, None, Multigrid.vertex(P.grid, None, dev))
    assert st.converged()


def test_batch_problem_with_nan_stops_alone(dev):
    from fluxion_b200 import ConvergenceReason, DType
    from fluxion_b200.batch import BatchSolver
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    be = dev.backend()
    sides = [65, 129, 65, 33]
    vx, vy, f = [], [], []
    for k, s in enumerate(sides):
        a, b = stream_velocity(s - 2, 50 + k)
        vx.append(a)
        vy.append(b)
        f.append(poisson_uniform_rhs(s - 2, 60 + k))
    f[1][129 * 40 + 40] = np.nan
    B = BatchSolver(dev, sides, 1e-2, be.upload_f64(np.concatenate(vx)), be.upload_f64(np.concatenate(vy)))
    x = be.allocate(B.offsets[-1], DType.F64)
    stats, _ = B.bicgstab(x, be.upload_f64(np.concatenate(f)), 1e-10, 100)
    assert stats[1].reason == ConvergenceReason.Breakdown
    assert all(stats[p].converged() for p in (0, 2, 3))
