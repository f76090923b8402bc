"""The oracle's preconditioned pipelined CG (Ghysels & Vanroose 2014, Algorithm 4; new, no
counterpart in the reference) pinned to the reference methods it extends: with M = I its
recurrences reduce to the reference's unpreconditioned PipelinedCgSolver (u stays equal to r), and
with the vertex multigrid it solves the Poisson problem as preconditioned CG does."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_err
from fluxion_b200.workloads import dst_poisson_solve, poisson_modes_rhs, poisson_problem


def test_identity_preconditioner_reproduces_pipelined_cg():
    n = 63
    P = poisson_problem(n)
    N = n + 2
    f = poisson_modes_rhs(n, seed=5)
    tol = 1e-10 * float(np.linalg.norm(f))
    x1, x2 = np.zeros(N * N), np.zeros(N * N)
    it1, res1, reason1 = O.pipelined_cg_solve(x1, f, N, N, 1.0, P.stencil.as_triples(), tol, 500)
    it2, res2, reason2 = O.pipelined_pcg_solve(x2, f, N, N, 1.0, P.stencil.as_triples(), tol, 500,
                                               O.IdentityPC(N * N))
    assert reason1 == 0 and reason2 == 0 and it1 == it2
    assert np.max(np.abs(x1 - x2)) <= 1e-12 * np.max(np.abs(x1))


@pytest.mark.parametrize("n", [63, 127])
def test_multigrid_pipelined_pcg_matches_pcg(n):
    P = poisson_problem(n)
    N = n + 2
    f = poisson_modes_rhs(n, seed=7)
    tol = 1e-10 * float(np.linalg.norm(f))
    st = P.stencil.as_triples()
    mg = O.Multigrid(N, N, P.h, P.h, 2, 2, 0.8, mode=1, op_coeff=1.0, entries=st)
    xc, xp = np.zeros(N * N), np.zeros(N * N)
    itc, _, rc = O.cg_solve(xc, f, N, N, 1.0, st, tol, 100, pc=mg)
    itp, resp, rp = O.pipelined_pcg_solve(xp, f, N, N, 1.0, st, tol, 100, mg)
    assert rc == 0 and rp == 0 and abs(itc - itp) <= 1 and resp < tol
    u_ref = dst_poisson_solve(f, n)
    assert rel_err(xp, u_ref) < 1e-8 and rel_err(xc, u_ref) < 1e-8


def test_max_iterations_reported():
    n = 63
    P = poisson_problem(n)
    N = n + 2
    f = poisson_modes_rhs(n, seed=9)
    x = np.zeros(N * N)
    it, res, reason = O.pipelined_pcg_solve(x, f, N, N, 1.0, P.stencil.as_triples(), 1e-30, 3,
                                            O.IdentityPC(N * N))
    assert reason == 1 and it == 3 and res > 0


def test_oracle_fp32_cycle_is_single_precision_and_close_to_fp64():
    """The oracle's FP32 vertex cycle: every value it returns is a float32 value, it differs from
    the FP64 cycle (it does compute in single precision) by less than 1e-5 relative, and as a
    preconditioner it takes CG to the FP64 tolerance in the FP64 cycle's iterations (within one)."""
    import numpy as np
    from fluxion_b200.workloads import poisson_problem, poisson_uniform_rhs
    from oracle import oracle as O
    n = 127
    P = poisson_problem(n)
    N = n + 2
    f = poisson_uniform_rhs(n, seed=8)
    mk = lambda f32: O.Multigrid(N, N, P.h, P.h, 2, 2, 0.8, mode=1, op_coeff=1.0,
                                 entries=P.stencil.as_triples(), coarse_max=15, coarse_sweeps=200, f32=f32)
    z64, z32 = np.zeros(N * N), np.zeros(N * N)
    mk(False).v_cycle(z64, f)
    mk(True).v_cycle_f32(z32, f)
    assert np.array_equal(z32.astype(np.float32).astype(np.float64), z32)
    e = np.linalg.norm(z32 - z64) / np.linalg.norm(z64)
    assert 0.0 < e < 1e-5, e
    tol = 1e-10 * np.linalg.norm(f)
    its = []
    for f32 in (False, True):
        x = np.zeros(N * N)
        it, _, reason = O.cg_solve(x, f, N, N, 1.0, P.stencil.as_triples(), tol, 100, pc=mk(f32))
        assert reason == 0
        its.append(it)
    assert abs(its[0] - its[1]) <= 1, its
