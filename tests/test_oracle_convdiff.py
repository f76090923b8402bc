"""The oracle's convection-diffusion operator for the solvers (CPU): it is the reference's
conv_diff_axpy on a copy when sigma = 1, an independent numpy restatement of the upwind
-nu Lap u + v.grad u when sigma = 0, its Jacobi diagonal is the operator's, and BiCGSTAB and
flexible GMRES reach the tolerance on the steady problem."""
import numpy as np

from oracle import oracle as O
from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity


def _fields(n, seed=5):
    vx, vy = stream_velocity(n, seed)
    N = n + 2
    kappa = np.random.default_rng(seed + 1).uniform(-0.02, -0.005, N * N)
    return N, 1.0 / (n + 1), vx, vy, kappa


def _cd_numpy(u, kap, vx, vy, h, N):
    """kappa Lap u + vx du/dx + vy du/dy on the interior, first-order upwind on sign(v)."""
    U = u.reshape(N, N)
    K = np.broadcast_to(kap, (N * N,)).reshape(N, N)
    VX, VY = vx.reshape(N, N), vy.reshape(N, N)
    c = U[1:-1, 1:-1]
    w, e, no, so = U[1:-1, :-2], U[1:-1, 2:], U[:-2, 1:-1], U[2:, 1:-1]
    lap = (w + e - 2 * c) / h ** 2 + (no + so - 2 * c) / h ** 2
    vxi, vyi = VX[1:-1, 1:-1], VY[1:-1, 1:-1]
    dudx = np.where(vxi >= 0, (c - w) / h, (e - c) / h)
    dudy = np.where(vyi >= 0, (c - no) / h, (so - c) / h)
    return K[1:-1, 1:-1] * lap + vxi * dudx + vyi * dudy


def test_sigma_one_is_conv_diff_axpy_on_a_copy():
    N, h, vx, vy, kappa = _fields(29)
    u = np.random.default_rng(3).uniform(-1, 1, N * N)
    op = O.cd_op(N, N, h, h, vx, vy, kappa=kappa, sigma=1.0, coeff=-0.37)
    out = u.copy()
    O.conv_diff_axpy(-0.37, u, out, kappa, vx, vy, N, N, h, h)
    assert np.array_equal(O.op_apply(op, u), out)


def test_steady_operator_matches_numpy():
    N, h, vx, vy, _ = _fields(31)
    u = np.random.default_rng(4).uniform(-1, 1, N * N)
    nu = 1e-2
    op = O.cd_op(N, N, h, h, vx, vy, kappa_s=-nu, sigma=0.0, coeff=1.0)
    got = O.op_apply(op, u).reshape(N, N)
    ref = _cd_numpy(u, -nu, vx, vy, h, N)
    assert np.max(np.abs(got[1:-1, 1:-1] - ref)) <= 1e-12 * np.max(np.abs(ref))
    ring = np.ones((N, N), bool)
    ring[1:-1, 1:-1] = False
    assert np.array_equal(got[ring], u.reshape(N, N)[ring])


def test_jacobi_divides_by_the_operator_diagonal():
    n = 5
    N, h, vx, vy, kappa = _fields(n)
    op = O.cd_op(N, N, h, h, vx, vy, kappa=kappa, sigma=0.4, coeff=0.7)
    diag = np.array([O.op_apply(op, np.eye(N * N)[i])[i] for i in range(N * N)])
    r = np.random.default_rng(8).uniform(-1, 1, N * N)
    z = np.zeros(N * N)
    pc = O.CdJacobiPC(op)
    O.lib().fxo_cd_jacobi_apply(pc._ctx, O._p(z), O._p(r))
    assert np.allclose(z, r / diag, rtol=1e-13, atol=0)


def test_solvers_reach_the_tolerance_on_the_steady_problem():
    n, nu = 63, 1e-2
    N, h, vx, vy, _ = _fields(n)
    f = poisson_uniform_rhs(n, 6)
    op = O.cd_op(N, N, h, h, vx, vy, kappa_s=-nu, sigma=0.0, coeff=1.0)
    tol = 1e-10 * np.linalg.norm(f)
    for name in ("bicgstab", "bicgstab_jacobi", "fgmres_jacobi"):
        x = np.zeros(N * N)
        pc = O.CdJacobiPC(op) if name.endswith("jacobi") else None
        if name.startswith("bicgstab"):
            it, _, reason = O.bicgstab_solve_op(x, f, op, tol, 5000, pc)
        else:
            it, _, reason = O.fgmres_solve_op(x, f, op, 30, tol, 5000, pc)
        assert reason == 0, name
        true = np.linalg.norm(O.op_apply(op, x) - f)
        assert true < 1.01 * tol, (name, it, true / np.linalg.norm(f))


def test_multigrid_preconditions_the_steady_problem():
    """The rediscretised V-cycle makes BiCGSTAB and FGMRES converge in a few iterations, where
    Jacobi needs hundreds, and the count does not grow with the grid."""
    nu = 1e-2
    for n, depth in ((63, 3), (127, 4)):
        N, h, vx, vy, _ = _fields(n)
        f = poisson_uniform_rhs(n, 6)
        op = O.cd_op(N, N, h, h, vx, vy, kappa_s=-nu, sigma=0.0, coeff=1.0)
        tol = 1e-10 * np.linalg.norm(f)
        mg = O.CdMultigrid(op)
        assert mg.depth() == depth
        x = np.zeros(N * N)
        it_j, _, _ = O.bicgstab_solve_op(x, f, op, tol, 5000, O.CdJacobiPC(op))
        for solver, limit in (("bicgstab", 12), ("fgmres", 20)):
            x = np.zeros(N * N)
            if solver == "bicgstab":
                it, _, reason = O.bicgstab_solve_op(x, f, op, tol, 200, mg)
            else:
                it, _, reason = O.fgmres_solve_op(x, f, op, 30, tol, 200, mg)
            assert reason == 0 and it <= limit and it * 10 < it_j, (n, solver, it, it_j)
            assert np.linalg.norm(O.op_apply(op, x) - f) < 1.01 * tol


def test_chebyshev_smoother_reduces_residual_faster_than_jacobi():
    """analytical.rs:447-521 in the oracle with both smoothers of the reference hierarchy
    (multigrid.rs:233-473): the residual falls every cycle, and further with Chebyshev."""
    n = 64
    h = 1.0 / (n - 1)
    t = np.arange(n) * h
    X, Y = np.meshgrid(t, t)
    b = (np.sin(np.pi * X) * np.sin(np.pi * Y)).ravel()
    st = O.laplacian_5pt(h, h)
    final = []
    for smoother in (0, 1):
        mg = O.Multigrid(n, n, h, h, 3, 3, 2.0 / 3.0, mode=0, smoother=smoother)
        x = np.zeros(n * n)
        prev = np.inf
        for _ in range(10):
            mg.v_cycle(x, b)
            ax = np.zeros(n * n)
            O.apply_stencil(x, ax, n, n, h, h, st)
            res = np.linalg.norm(b - ax)
            assert res < prev
            prev = res
        final.append(prev)
    assert final[1] < final[0] < 10.0
