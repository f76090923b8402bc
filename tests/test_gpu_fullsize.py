"""Parity at the benchmark's own sizes, not only below them.

- 4095^2 Poisson (4097^2 grid, the 32-mode source), CG preconditioned by the V(2,2)-cycle
  (full weighting, bilinear, weighted Jacobi 0.8, coarsest 15^2 x 200 sweeps) to 1e-10, with the
  cycle in FP64 and in FP32: the GPU solve against the oracle's solve of the same system (same
  stop reason, iterations within one, solutions within 1e-8) and against the exact DST-I solve;
  one fused cycle of each precision bit for bit against the oracle's cycle of that precision.
- 8191^2 (8193^2 grid): the mixed PCG and the FP64 refinement around FP32 PCG against DST-I,
  with the FP64 residual recomputed by numpy.
- 1023^2 convection-diffusion (nu = 1e-3, the stream-function velocity law): flexible GMRES(30)
  preconditioned by the conv-diff V-cycle against the oracle's solve of the same system.

The oracle solves take a few seconds on the host's cores.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

OMEGA, CMAX, CSW = 0.8, 15, 200


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    O.set_threads(os.cpu_count() or 1)
    return Device.best()


@pytest.fixture(scope="module")
def p4095():
    from fluxion_b200.workloads import dst_poisson_solve, poisson_modes_rhs, poisson_problem
    n = 4095
    f = poisson_modes_rhs(n, seed=2024)
    return n, poisson_problem(n), f, dst_poisson_solve(f, n)


def _omg(P, N, f32=False):
    return O.Multigrid(N, N, P.h, P.h, 2, 2, OMEGA, mode=1, op_coeff=1.0, entries=P.stencil.as_triples(),
                       coarse_max=CMAX, coarse_sweeps=CSW, f32=f32)


def test_cycles_4095_bitwise_vs_oracle(dev, p4095):
    """One fused cycle z = M^-1 r from zero at 4097^2, F64 and F32, equals the oracle's cycle of the
    same precision bit for bit."""
    from fluxion_b200 import DType, Field, Multigrid
    n, P, f, _ = p4095
    N = n + 2
    b = Field.from_f64(P.grid, f, dev)
    for dt, f32 in ((DType.F64, False), (DType.F32, True)):
        mg = Multigrid.vertex(P.grid, None, dev, 2, 2, OMEGA, CMAX, CSW, dt)
        z = Field.zeros(P.grid, DType.F64, dev)
        mg.precondition(z, b)
        zo = np.zeros(N * N)
        omg = _omg(P, N, f32)
        assert omg.depth() == mg.depth()
        if f32:
            omg.v_cycle_f32(zo, f)
        else:
            omg.v_cycle(zo, f)
        assert np.array_equal(z.to_vec_f64(), zo), dt


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_mg_pcg_4095_matches_oracle_and_direct(dev, p4095, dtype):
    from fluxion_b200 import CgSolver, DType, Field, Multigrid
    from fluxion_b200.workloads import neg_laplacian_residual
    n, P, f, u_ref = p4095
    N = n + 2
    tol = 1e-10 * float(np.linalg.norm(f))
    dt = DType.F32 if dtype == "f32" else DType.F64
    b = Field.from_f64(P.grid, f, dev)
    x = Field.zeros(P.grid, DType.F64, dev)
    mg = Multigrid.vertex(P.grid, None, dev, 2, 2, OMEGA, CMAX, CSW, dt)
    s = CgSolver(P.grid, dev, tol, 100).solve_preconditioned(x, b, P.coeff, P.stencil, None, mg)
    xo = np.zeros(N * N)
    it, res, reason = O.cg_solve(xo, f, N, N, 1.0, P.stencil.as_triples(), tol, 100, pc=_omg(P, N, dtype == "f32"))
    u = x.to_vec_f64()
    assert s.converged() and reason == 0, (s, it, reason)
    assert abs(s.iterations - it) <= 1, (s.iterations, it)
    assert rel_err(u, xo) <= 1e-8
    assert neg_laplacian_residual(u, f, n) < 1.01e-10 * np.linalg.norm(f)
    assert rel_err(u, u_ref) <= 1e-8


def test_8191_mixed_pcg_and_refinement_vs_direct(dev):
    """The larger mixed-precision size: FP32 V-cycle inside FP64 CG, and FP64 iterative refinement
    around FP32 V-cycle PCG (inner tolerance 1e-4), each to 1e-10 on the FP64 residual, within
    1e-8 of the exact solve."""
    from fluxion_b200 import CgSolver, DType, Field, MixedPrecisionRefinement, Multigrid
    from fluxion_b200.workloads import dst_poisson_solve, neg_laplacian_residual, poisson_modes_rhs, \
        poisson_problem
    n = 8191
    P = poisson_problem(n)
    f = poisson_modes_rhs(n, seed=2024)
    fnorm = float(np.linalg.norm(f))
    tol = 1e-10 * fnorm
    u_ref = dst_poisson_solve(f, n)
    b = Field.from_f64(P.grid, f, dev)
    x = Field.zeros(P.grid, DType.F64, dev)
    mg32 = Multigrid.vertex(P.grid, None, dev, 2, 2, OMEGA, CMAX, CSW, DType.F32)
    s = CgSolver(P.grid, dev, tol, 100).solve_preconditioned(x, b, P.coeff, P.stencil, None, mg32)
    u = x.to_vec_f64()
    assert s.converged() and s.iterations <= 15, s
    assert neg_laplacian_residual(u, f, n) < 1.01e-10 * fnorm
    assert rel_err(u, u_ref) <= 1e-8
    x.fill(0.0)
    ir = MixedPrecisionRefinement(P.grid, dev, tol, 20, 1e-4, 100)
    si = ir.solve_preconditioned(x, b, P.coeff, P.stencil, None, mg32)
    u = x.to_vec_f64()
    assert si.converged(), si
    assert neg_laplacian_residual(u, f, n) < 1.01e-10 * fnorm
    assert rel_err(u, u_ref) <= 1e-8


def test_convdiff_1023_fgmres_multigrid_matches_oracle(dev):
    from fluxion_b200 import ConvDiffMultigrid, ConvDiffOperator, DType, FgmresSolver, Field, Grid
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    n, nu = 1023, 1e-3
    N, h = n + 2, 1.0 / (n + 1)
    g = Grid.square(N, h)
    vx, vy = stream_velocity(n, 77)
    f = poisson_uniform_rhs(n, 78)
    tol = 1e-10 * float(np.linalg.norm(f))
    op = ConvDiffOperator(g, Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev), -nu, sigma=0.0, coeff=1.0)
    oop = O.cd_op(N, N, h, h, vx, vy, kappa=None, kappa_s=-nu, sigma=0.0, coeff=1.0)
    x = Field.zeros(g, DType.F64, dev)
    s = FgmresSolver(g, dev, 30, tol, 300).solve_op(x, Field.from_f64(g, f, dev), op, ConvDiffMultigrid(op))
    xo = np.zeros(N * N)
    it, _, reason = O.fgmres_solve_op(xo, f, oop, 30, tol, 300, O.CdMultigrid(oop))
    assert s.converged() and reason == 0 and abs(s.iterations - it) <= 1, (s, it, reason)
    assert np.linalg.norm(O.op_apply(oop, x.to_vec_f64()) - f) < 1.01 * tol
    assert rel_err(x.to_vec_f64(), xo) <= 1e-8
