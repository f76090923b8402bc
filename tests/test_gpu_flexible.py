"""Flexible CG and flexible GMRES on the GPU against the oracle: with a fixed preconditioner they
are PCG and GMRES, and with the inner-CG preconditioner on a varying step schedule they follow
the oracle's iteration counts and reach the tolerance on the FP64 residual recomputed here."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

SCHEDULE = [1, 2, 3, 4, 5, 6]


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


def _setup(n, dev, seed=3):
    from fluxion_b200 import Boundaries, Field
    from fluxion_b200.workloads import poisson_modes_rhs, poisson_problem
    P = poisson_problem(n)
    f = poisson_modes_rhs(n, seed)
    b = Field.from_f64(P.grid, f, dev)
    return P, n + 2, f, b, 1e-10 * np.linalg.norm(f), Boundaries.zero_dirichlet()


def _true_rel(x, f, n):
    from fluxion_b200.workloads import neg_laplacian_residual
    return neg_laplacian_residual(x, f, n) / np.linalg.norm(f)


def test_fcg_with_multigrid_is_pcg(dev):
    from fluxion_b200 import CgSolver, DType, FcgSolver, Field, Multigrid
    P, N, f, b, tol, bc = _setup(255, dev)
    mg = Multigrid.vertex(P.grid, None, dev)
    xp, xf = Field.zeros(P.grid, DType.F64, dev), Field.zeros(P.grid, DType.F64, dev)
    sp = CgSolver(P.grid, dev, tol, 100).solve_preconditioned(xp, b, P.coeff, P.stencil, bc, mg)
    sf = FcgSolver(P.grid, dev, tol, 100).solve_preconditioned(xf, b, P.coeff, P.stencil, bc, mg)
    assert sp.converged() and sf.converged() and sp.iterations == sf.iterations
    assert rel_err(xf.to_vec_f64(), xp.to_vec_f64()) < 1e-9
    assert _true_rel(xf.to_vec_f64(), f, 255) < 1.01e-10


def test_fgmres_without_preconditioner_is_gmres(dev):
    from fluxion_b200 import DType, FgmresSolver, Field, GmresSolver
    P, N, f, b, tol, bc = _setup(31, dev)
    xg, xf = Field.zeros(P.grid, DType.F64, dev), Field.zeros(P.grid, DType.F64, dev)
    sg = GmresSolver(P.grid, dev, 20, tol, 2000).solve(xg, b, P.coeff, P.stencil, bc)
    sf = FgmresSolver(P.grid, dev, 20, tol, 2000).solve(xf, b, P.coeff, P.stencil, bc)
    assert sg == sf and sg.converged()
    assert np.array_equal(xg.to_vec_f64(), xf.to_vec_f64())
    xo = np.zeros(N * N)
    it, _, reason = O.fgmres_solve(xo, f, N, N, P.coeff, P.stencil.as_triples(), 20, tol, 2000)
    assert reason == 0 and abs(it - sf.iterations) <= 1


def test_fgmres_with_multigrid_matches_oracle(dev):
    from fluxion_b200 import DType, FgmresSolver, Field, Multigrid
    P, N, f, b, tol, bc = _setup(127, dev)
    mg = Multigrid.vertex(P.grid, None, dev)
    x = Field.zeros(P.grid, DType.F64, dev)
    s = FgmresSolver(P.grid, dev, 30, tol, 200).solve_preconditioned(x, b, P.coeff, P.stencil, bc, mg)
    ent = P.stencil.as_triples()
    omg = O.Multigrid(N, N, P.h, P.h, 2, 2, 0.8, mode=1, op_coeff=1.0, entries=ent)
    xo = np.zeros(N * N)
    it, _, reason = O.fgmres_solve(xo, f, N, N, P.coeff, ent, 30, tol, 200, pc=omg)
    assert s.converged() and reason == 0 and s.iterations == it
    assert rel_err(x.to_vec_f64(), xo) < 1e-9
    assert _true_rel(x.to_vec_f64(), f, 127) < 1.01e-10


@pytest.mark.parametrize("solver", ["fcg", "fgmres"])
def test_flexible_solvers_with_varying_preconditioner_match_oracle(dev, solver):
    from fluxion_b200 import CgSolver, DType, FcgSolver, FgmresSolver, Field, InnerCg
    P, N, f, b, tol, bc = _setup(63, dev)
    ent = P.stencil.as_triples()
    pc = InnerCg(P.grid, P.coeff, P.stencil, bc, SCHEDULE, device=dev)
    opc = O.InnerCgPC(N, N, P.coeff, ent, SCHEDULE)
    x = Field.zeros(P.grid, DType.F64, dev)
    xo = np.zeros(N * N)
    if solver == "fcg":
        s = FcgSolver(P.grid, dev, tol, 3000).solve_preconditioned(x, b, P.coeff, P.stencil, bc, pc)
        it, _, reason = O.fcg_solve(xo, f, N, N, P.coeff, ent, tol, 3000, opc)
    else:
        s = FgmresSolver(P.grid, dev, 30, tol, 3000).solve_preconditioned(x, b, P.coeff, P.stencil, bc, pc)
        it, _, reason = O.fgmres_solve(xo, f, N, N, P.coeff, ent, 30, tol, 3000, pc=opc)
    assert s.converged() and reason == 0
    # a nonlinear preconditioner amplifies roundoff differences in the inner products
    assert abs(s.iterations - it) <= max(3, it // 20), (s.iterations, it)
    assert _true_rel(x.to_vec_f64(), f, 63) < 1.01e-10
    if solver == "fcg":
        # the same preconditioner in plain PCG: at least twice the iterations
        xp = Field.zeros(P.grid, DType.F64, dev)
        pc2 = InnerCg(P.grid, P.coeff, P.stencil, bc, SCHEDULE, device=dev)
        sp = CgSolver(P.grid, dev, tol, 3000).solve_preconditioned(xp, b, P.coeff, P.stencil, bc, pc2)
        assert sp.iterations >= 2 * s.iterations


def test_inner_cg_preconditioner_matches_oracle_steps(dev):
    """One application = the scheduled number of CG steps, as the oracle's."""
    from fluxion_b200 import DType, Field, InnerCg
    P, N, f, b, tol, bc = _setup(63, dev)
    ent = P.stencil.as_triples()
    pc = InnerCg(P.grid, P.coeff, P.stencil, bc, [4, 2], device=dev)
    opc = O.InnerCgPC(N, N, P.coeff, ent, [4, 2])
    for _ in range(3):
        z = Field.zeros(P.grid, DType.F64, dev)
        pc.apply(z, b)
        zo = np.zeros(N * N)
        O.lib().fxo_inner_cg_pc_apply(opc._ctx, O._p(zo), O._p(f))
        assert rel_err(z.to_vec_f64(), zo) < 1e-12
