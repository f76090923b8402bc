"""The convection-diffusion operator in the GPU solvers against the oracle: the operator and its
Jacobi preconditioner bit for bit, and BiCGSTAB, GMRES and flexible GMRES on the steady
problem (-nu Lap u + v.grad u = f) and on an implicit step ((I + dt CD) u = b) with the oracle's
stop reasons, close iteration counts, and the tolerance met on the FP64 residual recomputed by
the oracle's operator."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


def _problem(n, dev, nu=1e-2, sigma=0.0, coeff=1.0, kappa_field=False, seed=5):
    from fluxion_b200 import ConvDiffOperator, Field, Grid
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    N, h = n + 2, 1.0 / (n + 1)
    g = Grid.square(N, h)
    vx, vy = stream_velocity(n, seed)
    kappa = np.full(N * N, -nu) if kappa_field else None
    f = poisson_uniform_rhs(n, seed + 1)
    VX, VY = Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev)
    K = Field.from_f64(g, kappa, dev) if kappa_field else -nu
    op = ConvDiffOperator(g, VX, VY, K, sigma=sigma, coeff=coeff)
    oop = O.cd_op(N, N, h, h, vx, vy, kappa=kappa, kappa_s=-nu, sigma=sigma, coeff=coeff)
    return g, N, f, op, oop


@pytest.mark.parametrize("kappa_field,sigma,coeff", [(False, 0.0, 1.0), (True, 1.0, -2e-3), (True, 0.3, 0.8)])
def test_operator_and_jacobi_match_oracle_bitwise(dev, kappa_field, sigma, coeff):
    from fluxion_b200 import DType, Field
    g, N, f, op, oop = _problem(61, dev, sigma=sigma, coeff=coeff, kappa_field=kappa_field)
    u = np.random.default_rng(2).uniform(-1, 1, N * N)
    U, out = Field.from_f64(g, u, dev), Field.zeros(g, DType.F64, dev)
    op.apply(U, out)
    assert np.array_equal(out.to_vec_f64(), O.op_apply(oop, u))
    z = Field.zeros(g, DType.F64, dev)
    op.jacobi().apply(z, U)
    zo = np.zeros(N * N)
    O.lib().fxo_cd_jacobi_apply(O.CdJacobiPC(oop)._ctx, O._p(zo), O._p(u))
    assert np.array_equal(z.to_vec_f64(), zo)


@pytest.mark.parametrize("solver,jacobi", [("bicgstab", False), ("bicgstab", True), ("gmres", True),
                                           ("fgmres", True), ("fgmres", False)])
def test_steady_conv_diff_solve_matches_oracle(dev, solver, jacobi):
    from fluxion_b200 import BiCgStabSolver, DType, FgmresSolver, Field, GmresSolver
    g, N, f, op, oop = _problem(63, dev)
    tol = 1e-10 * np.linalg.norm(f)
    b = Field.from_f64(g, f, dev)
    x = Field.zeros(g, DType.F64, dev)
    pc = op.jacobi() if jacobi else None
    opc = O.CdJacobiPC(oop) if jacobi else None
    xo = np.zeros(N * N)
    if solver == "bicgstab":
        s = BiCgStabSolver(g, dev, tol, 5000).solve_op(x, b, op, pc)
        it, _, reason = O.bicgstab_solve_op(xo, f, oop, tol, 5000, opc)
    elif solver == "gmres":
        s = GmresSolver(g, dev, 30, tol, 5000).solve_op(x, b, op, pc)
        it, _, reason = O.gmres_solve_op(xo, f, oop, 30, tol, 5000, opc)
    else:
        s = FgmresSolver(g, dev, 30, tol, 5000).solve_op(x, b, op, pc)
        it, _, reason = O.fgmres_solve_op(xo, f, oop, 30, tol, 5000, opc)
    assert int(s.reason) == reason == 0
    # hundreds of non-symmetric Krylov steps: roundoff in the inner products (compensated on the
    # GPU, Kahan in the oracle) moves the stopping step by a few
    assert abs(s.iterations - it) <= max(3, it // 20), (s.iterations, it)
    xv = x.to_vec_f64()
    true = np.linalg.norm(O.op_apply(oop, xv) - f)
    if solver != "gmres":
        assert true < 1.01 * tol
        assert rel_err(xv, xo) < 1e-7  # two solutions within the tolerance differ by ~1e-9
    else:  # left-preconditioned GMRES stops on ||M^-1 r||, as the reference's
        assert rel_err(xv, xo) < 1e-5


def test_implicit_step_matches_oracle(dev):
    """(I + dt CD) u = b with kappa = -nu: a backward-Euler step of u_t = nu Lap u - v.grad u,
    the operator conv_diff_axpy(dt, u, u) of the reference's implicit use."""
    from fluxion_b200 import BiCgStabSolver, DType, Field
    g, N, f, op, oop = _problem(127, dev, nu=1e-3, sigma=1.0, coeff=5e-3, kappa_field=True)
    tol = 1e-10 * np.linalg.norm(f)
    b = Field.from_f64(g, f, dev)
    x = Field.zeros(g, DType.F64, dev)
    s = BiCgStabSolver(g, dev, tol, 500).solve_op(x, b, op, op.jacobi())
    xo = np.zeros(N * N)
    it, _, reason = O.bicgstab_solve_op(xo, f, oop, tol, 500, O.CdJacobiPC(oop))
    assert s.converged() and reason == 0 and abs(s.iterations - it) <= 1
    assert np.linalg.norm(O.op_apply(oop, x.to_vec_f64()) - f) < 1.01 * tol
    assert rel_err(x.to_vec_f64(), xo) < 1e-9


@pytest.mark.parametrize("n,nu,sigma,coeff,kappa_field", [(63, 1e-2, 0.0, 1.0, False), (127, 1e-3, 1.0, 5e-3, True)])
def test_multigrid_cycle_matches_oracle_bitwise(dev, n, nu, sigma, coeff, kappa_field):
    from fluxion_b200 import ConvDiffMultigrid, DType, Field
    g, N, f, op, oop = _problem(n, dev, nu=nu, sigma=sigma, coeff=coeff, kappa_field=kappa_field)
    mg = ConvDiffMultigrid(op)
    omg = O.CdMultigrid(oop)
    assert mg.depth() == omg.depth() >= 3
    r = np.random.default_rng(9).uniform(-1, 1, N * N)
    for _ in range(2):  # the second application starts from the buffers the first left
        z = Field.zeros(g, DType.F64, dev)
        mg.apply(z, Field.from_f64(g, r, dev))
        assert np.array_equal(z.to_vec_f64(), omg.apply(r))


@pytest.mark.parametrize("solver", ["bicgstab", "fgmres"])
def test_multigrid_preconditioned_solve_matches_oracle(dev, solver):
    from fluxion_b200 import BiCgStabSolver, ConvDiffMultigrid, DType, FgmresSolver, Field
    g, N, f, op, oop = _problem(127, dev)
    tol = 1e-10 * np.linalg.norm(f)
    b = Field.from_f64(g, f, dev)
    x = Field.zeros(g, DType.F64, dev)
    mg, omg = ConvDiffMultigrid(op), O.CdMultigrid(oop)
    xo = np.zeros(N * N)
    if solver == "bicgstab":
        s = BiCgStabSolver(g, dev, tol, 200).solve_op(x, b, op, mg)
        it, _, reason = O.bicgstab_solve_op(xo, f, oop, tol, 200, omg)
    else:
        s = FgmresSolver(g, dev, 30, tol, 200).solve_op(x, b, op, mg)
        it, _, reason = O.fgmres_solve_op(xo, f, oop, 30, tol, 200, omg)
    assert s.converged() and reason == 0 and abs(s.iterations - it) <= 1 and s.iterations <= 20
    assert np.linalg.norm(O.op_apply(oop, x.to_vec_f64()) - f) < 1.01 * tol
    assert rel_err(x.to_vec_f64(), xo) < 1e-8


@pytest.mark.parametrize("n,nu,sigma,coeff,kappa_field", [(63, 1e-2, 0.0, 1.0, False), (127, 1e-3, 1.0, 5e-3, True)])
def test_f32_multigrid_cycle_close_to_oracle(dev, n, nu, sigma, coeff, kappa_field):
    """The cycle in single precision (fx_cdmg_create_typed, FX_F32): the same hierarchy and the
    same cycle as the F64 one, rounded to F32 -- within 1e-4 of the oracle's F64 cycle, and not
    equal to it (it does compute in F32)."""
    from fluxion_b200 import ConvDiffMultigrid, DType, Field
    g, N, f, op, oop = _problem(n, dev, nu=nu, sigma=sigma, coeff=coeff, kappa_field=kappa_field)
    mg = ConvDiffMultigrid(op, dtype=DType.F32)
    omg = O.CdMultigrid(oop)
    assert mg.depth() == omg.depth() >= 3 and mg.dtype == DType.F32
    r = np.random.default_rng(9).uniform(-1, 1, N * N)
    zo = omg.apply(r)
    for _ in range(2):
        z = Field.zeros(g, DType.F64, dev)
        z.fill(7.0)  # every point is written
        mg.apply(z, Field.from_f64(g, r, dev))
        e = rel_err(z.to_vec_f64(), zo)
        assert 0.0 < e < 1e-4, e


@pytest.mark.parametrize("solver,nu", [("bicgstab", 1e-2), ("fgmres", 1e-2), ("bicgstab", 1e-3), ("fgmres", 1e-3)])
def test_f32_multigrid_inside_fp64_solvers(dev, solver, nu):
    """BiCGSTAB and FGMRES in FP64 with the F32 cycle as preconditioner reach the FP64 tolerance
    on the true residual (recomputed by the oracle's operator) in at most two iterations more
    than with the F64 cycle."""
    from fluxion_b200 import BiCgStabSolver, ConvDiffMultigrid, DType, FgmresSolver, Field
    g, N, f, op, oop = _problem(127, dev, nu=nu)
    tol = 1e-10 * np.linalg.norm(f)
    b = Field.from_f64(g, f, dev)
    its = {}
    for dt in (DType.F64, DType.F32):
        mg = ConvDiffMultigrid(op, dtype=dt)
        x = Field.zeros(g, DType.F64, dev)
        if solver == "bicgstab":
            s = BiCgStabSolver(g, dev, tol, 200).solve_op(x, b, op, mg)
        else:
            s = FgmresSolver(g, dev, 30, tol, 200).solve_op(x, b, op, mg)
        assert s.converged(), (dt, s)
        assert np.linalg.norm(O.op_apply(oop, x.to_vec_f64()) - f) < 1.01 * tol
        its[dt] = s.iterations
    assert its[DType.F32] <= its[DType.F64] + 2, its


def test_multigrid_replays_its_recorded_cycle(dev):
    """With replay on, the first application to a (z, r) pair records the cycle into a CUDA graph
    (its kernels counted once as launched), later ones replay it as one launch; every
    application gives the same z, equal to the oracle's cycle in F64."""
    from fluxion_b200 import ConvDiffMultigrid, DimensionMismatch, DType, Field, Grid
    g, N, f, op, oop = _problem(127, dev)
    be = dev.backend()
    rv = np.random.default_rng(3).uniform(-1, 1, N * N)
    zo = O.CdMultigrid(oop).apply(rv)
    for dt in (DType.F64, DType.F32):
        mg = ConvDiffMultigrid(op, dtype=dt)
        mg.set_replay(True)
        r, z = Field.from_f64(g, rv, dev), Field.zeros(g, DType.F64, dev)
        outs, counts = [], []
        for _ in range(3):
            c0 = be.launch_count()
            mg.apply(z, r)
            counts.append(be.launch_count() - c0)
            outs.append(z.to_vec_f64())
        assert counts[0] > 10 and counts[1] == counts[2] == 1, counts
        assert all(np.array_equal(o, outs[0]) for o in outs)
        if dt == DType.F64:
            assert np.array_equal(outs[0], zo)
        small = Grid.square(N - 2, 1.0)  # vectors of another extent are refused before any replay
        with pytest.raises(DimensionMismatch):
            mg.apply(Field.zeros(small, DType.F64, dev), Field.zeros(small, DType.F64, dev))


@pytest.mark.parametrize("nu", [1e-2, 1e-3])
def test_fgmres_cgs2_matches_oracle_mgs_solve(dev, nu):
    """Flexible GMRES(30) with classical Gram-Schmidt twice (three passes over the basis per Arnoldi
    step) reaches the oracle's MGS solve: same stop reason, iterations within one, solutions within
    1e-8, the tolerance met on the residual the oracle recomputes."""
    from fluxion_b200 import ConvDiffMultigrid, DType, FgmresSolver, Field
    g, N, f, op, oop = _problem(127, dev, nu=nu)
    tol = 1e-10 * np.linalg.norm(f)
    b = Field.from_f64(g, f, dev)
    x = Field.zeros(g, DType.F64, dev)
    solver = FgmresSolver(g, dev, 30, tol, 300)
    solver.set_orthogonalization("cgs2")
    s = solver.solve_op(x, b, op, ConvDiffMultigrid(op))
    xo = np.zeros(N * N)
    it, _, reason = O.fgmres_solve_op(xo, f, oop, 30, tol, 300, O.CdMultigrid(oop))
    assert s.converged() and reason == 0 and abs(s.iterations - it) <= 1, (s, it)
    assert np.linalg.norm(O.op_apply(oop, x.to_vec_f64()) - f) < 1.01 * tol
    assert rel_err(x.to_vec_f64(), xo) < 1e-8
