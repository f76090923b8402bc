"""Flexible CG and flexible GMRES in the oracle (CPU): with a fixed preconditioner they reduce to
PCG and GMRES, and with one that changes between applications (an inner CG whose step count
follows a schedule) they still reach the tolerance on the true residual, where PCG needs far
more iterations and left-preconditioned GMRES stops on a residual that is not the true one."""
import numpy as np

from oracle import oracle as O
from fluxion_b200.workloads import neg_laplacian_residual, poisson_modes_rhs, poisson_problem

N_INT = 63
SCHEDULE = [1, 2, 3, 4, 5, 6]


def _problem(n=N_INT):
    P = poisson_problem(n)
    f = poisson_modes_rhs(n, 3)
    return P, n + 2, f, 1e-10 * np.linalg.norm(f), P.stencil.as_triples()


def _true_rel(x, f, n):
    return neg_laplacian_residual(x, f, n) / np.linalg.norm(f)


def test_fcg_with_fixed_multigrid_is_pcg():
    P, N, f, tol, ent = _problem()
    mg = O.Multigrid(N, N, P.h, P.h, 2, 2, 0.8, mode=1, op_coeff=1.0, entries=ent, coarse_max=15,
                     coarse_sweeps=200)
    xp, xf = np.zeros(N * N), np.zeros(N * N)
    itp, _, rp = O.cg_solve(xp, f, N, N, P.coeff, ent, tol, 200, pc=mg)
    itf, _, rf = O.fcg_solve(xf, f, N, N, P.coeff, ent, tol, 200, mg)
    assert rp == rf == 0 and itp == itf
    assert np.max(np.abs(xp - xf)) <= 1e-10 * np.max(np.abs(xp))


def test_fgmres_without_preconditioner_is_gmres():
    P, N, f, tol, ent = _problem(31)
    xg, xf = np.zeros(N * N), np.zeros(N * N)
    g = O.gmres_solve(xg, f, N, N, P.coeff, ent, 20, tol, 2000)
    h = O.fgmres_solve(xf, f, N, N, P.coeff, ent, 20, tol, 2000)
    assert g == h and g[2] == 0
    assert np.array_equal(xg, xf)


def test_flexible_solvers_with_a_varying_preconditioner():
    P, N, f, tol, ent = _problem()
    out = {}
    for name in ("pcg", "fcg", "gmres", "fgmres"):
        pc = O.InnerCgPC(N, N, P.coeff, ent, SCHEDULE)
        x = np.zeros(N * N)
        if name == "pcg":
            r = O.cg_solve(x, f, N, N, P.coeff, ent, tol, 3000, pc=pc)
        elif name == "fcg":
            r = O.fcg_solve(x, f, N, N, P.coeff, ent, tol, 3000, pc)
        elif name == "gmres":
            r = O.gmres_solve(x, f, N, N, P.coeff, ent, 30, tol, 3000, pc=pc)
        else:
            r = O.fgmres_solve(x, f, N, N, P.coeff, ent, 30, tol, 3000, pc=pc)
        out[name] = (r[0], r[2], _true_rel(x, f, N_INT), pc.calls)
    # both flexible solvers converge on the true residual ...
    assert out["fcg"][1] == 0 and out["fcg"][2] < 1.01e-10
    assert out["fgmres"][1] == 0 and out["fgmres"][2] < 1.01e-10
    # ... PCG needs twice the iterations or more with the same preconditioner ...
    assert out["pcg"][0] >= 2 * out["fcg"][0]
    # ... and left-preconditioned GMRES reports convergence on M^-1 r while b - A x is large
    assert out["gmres"][1] == 0 and out["gmres"][2] > 1e-3
    # one preconditioner application per iteration (plus the initial one for FCG)
    assert out["fcg"][3] == out["fcg"][0] + 1 and out["fgmres"][3] == out["fgmres"][0]
