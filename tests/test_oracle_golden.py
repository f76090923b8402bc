"""Pin the CPU oracle to the reference's own known-answer tests.

Every case below restates an assertion from the reference test suite
(crates/backend-cpu/src/ops.rs tests, crates/runtime/tests/solvers.rs,
analytical.rs, properties.rs, crates/core/src/*.rs tests) and checks the
oracle against it.  These run without a GPU.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import gaussian_ic, quadratic_field, sin_sin_field

from fluxion_b200.core import (Boundaries, BoundaryCondition, DType, Grid, InvalidGrid,
                               InvalidStencil, Stencil)

ZD = O.ZERO_DIRICHLET


# ---------------------------------------------------------------- core types

def test_grid_known_answers():
    # crates/core/src/grid.rs:68-95
    g = Grid.new(10, 20, 0.1, 0.2)
    assert g.len() == 200 and g.idx(3, 5) == 3 * 20 + 5
    s = Grid.square(100, 0.01)
    assert s.rows == 100 and s.cols == 100 and abs(s.dx - 0.01) < np.finfo(float).eps
    for bad in [(2, 10, 1.0, 1.0), (10, 2, 1.0, 1.0), (10, 10, 0.0, 1.0), (10, 10, -1.0, 1.0),
                (10, 10, float("nan"), 1.0), (10, 10, float("inf"), 1.0)]:
        with pytest.raises(InvalidGrid):
            Grid.new(*bad)


def test_stencil_known_answers():
    # crates/core/src/stencil.rs:245-362
    s = Stencil.laplacian_2d_5pt(1.0, 1.0)
    assert abs(sum(e.weight for e in s.entries())) < 1e-14
    assert s.len() == 5
    c = [e for e in s.entries() if e.dr == 0 and e.dc == 0][0]
    assert abs(c.weight + 4.0) < 1e-14
    s = Stencil.laplacian_2d_5pt(0.1, 0.2)
    assert abs(sum(e.weight for e in s.entries())) < 1e-10
    east = [e for e in s.entries() if e.dr == 0 and e.dc == 1][0]
    assert abs(east.weight - 1.0 / (0.1 * 0.1)) < 1e-14
    with pytest.raises(InvalidStencil):
        Stencil([])
    s9 = Stencil.laplacian_2d_9pt(1.0, 1.0)
    assert abs(sum(e.weight for e in s9.entries())) < 1e-14
    assert Stencil.laplacian_2d_9pt(0.1, 0.2).len() == 9
    c9 = [e for e in s9.entries() if e.dr == 0 and e.dc == 0][0]
    assert abs(c9.weight + 10.0 / 3.0) < 1e-14
    for e in s9.entries():
        expected = {(0, 0): -20.0}.get((abs(e.dr), abs(e.dc)),
                                       1.0 if (abs(e.dr), abs(e.dc)) == (1, 1) else 4.0)
        assert abs(e.weight * 6.0 - expected) < 1e-12
    assert abs(sum(e.weight for e in Stencil.laplacian_2d_9pt(0.05, 0.1).entries())) < 1e-10


def test_boundaries_and_dtype():
    # crates/core/src/boundary.rs:46-121, dtype.rs:17-44
    bc = Boundaries.zero_dirichlet()
    assert all(s == BoundaryCondition.Dirichlet(0.0) for s in bc.sides())
    assert Boundaries.periodic().top == BoundaryCondition.Periodic()
    r = BoundaryCondition.Robin(1.0, 1.0, 0.0)
    assert r.kind.name == "ROBIN"
    assert DType.F32.size_bytes() == 4 and DType.F64.size_bytes() == 8


def test_poisson_stencil_is_negative_laplacian():
    h = 1.0 / 17
    s = Stencil.poisson_neg_laplacian(h, h)
    lap = Stencil.laplacian_2d_5pt(h, h)
    # v + S v == -lap(v) entry by entry
    for a, b in zip(s.entries(), lap.entries()):
        extra = 1.0 if (a.dr, a.dc) == (0, 0) else 0.0
        assert abs((a.weight + extra) + b.weight) <= 1e-12 * abs(b.weight)


# ---------------------------------------------------------------- CPU backend ops

def test_fill_and_norm():
    # ops.rs:1201-1209
    x = np.zeros(16)
    O.fill(x, 3.0)
    assert abs(O.norm_l2(x) - 12.0) < 1e-12


def test_axpy_basic():
    # ops.rs:1211-1223
    x = np.array([1.0, 2.0, 3.0])
    y = np.array([10.0, 20.0, 30.0])
    O.axpy(2.0, x, y)
    assert np.all(np.abs(y - [12.0, 24.0, 36.0]) < 1e-14)


def test_laplacian_on_quadratic_field():
    # ops.rs:1225-1266: Laplacian(x^2 + y^2) = 4 on rows/cols 2..n-2
    n = 32
    h = 1.0 / (n - 1)
    data = quadratic_field(n, h)
    out = np.zeros(n * n)
    O.apply_stencil(data, out, n, n, h, h, O.laplacian_5pt(h, h), ZD)
    o = out.reshape(n, n)
    assert np.all(np.abs(o[2:n - 2, 2:n - 2] - 4.0) < 1e-10)


def test_dirichlet_nonzero_boundary():
    # ops.rs:1268-1305
    n = 16
    h = 1.0 / (n - 1)
    data = np.full(n * n, 50.0)
    out = np.zeros(n * n)
    O.apply_stencil(data, out, n, n, h, h, O.laplacian_5pt(h, h), [(O.BC_DIRICHLET, 100.0, 0, 0)] * 4)
    o = out.reshape(n, n)
    assert np.all(np.abs(o[0] - 100.0) < 1e-12) and np.all(np.abs(o[-1] - 100.0) < 1e-12)


def test_neumann_zero_flux_preserves_neighbor():
    # ops.rs:1307-1338
    n = 16
    h = 1.0 / (n - 1)
    data = np.full(n * n, 42.0)
    out = np.zeros(n * n)
    O.apply_stencil(data, out, n, n, h, h, O.laplacian_5pt(h, h), [(O.BC_NEUMANN, 0.0, 0, 0)] * 4)
    assert np.all(np.abs(out.reshape(n, n)[0] - 42.0) < 1e-10)


def test_periodic_rejected():
    # ops.rs:9-23
    n = 8
    with pytest.raises(O.OracleError):
        O.apply_stencil(np.zeros(n * n), np.zeros(n * n), n, n, 1.0, 1.0, O.laplacian_5pt(1, 1),
                        [(O.BC_PERIODIC, 0, 0, 0)] * 4)


def test_field_reductions_known_answers():
    # crates/runtime/tests/solvers.rs:899-975 and :1117-1149
    n = 16
    x = np.zeros(n * n)
    O.fill(x, 3.0)
    assert abs(O.reduce_sum(x) - 3.0 * n * n) < 1e-10
    seq = np.arange(n * n, dtype=np.float64)
    assert abs(O.reduce_max(seq) - (n * n - 1)) < 1e-10 and abs(O.reduce_min(seq)) < 1e-10
    a, b = np.full(n * n, 2.0), np.full(n * n, 3.0)
    assert abs(O.dot(a, b) - 6.0 * n * n) < 1e-10
    one = np.ones(32 * 32)
    h = 1.0 / 31
    assert abs(O.reduce_sum(one) * h * h - 1.0) < 0.1  # Field::integral
    a, b, c, d = (np.full(n * n, v) for v in (1.0, 2.0, 3.0, 4.0))
    d1, d2 = O.dot2(a, b, c, d)
    assert abs(d1 - 2.0 * n * n) < 1e-8 and abs(d2 - 12.0 * n * n) < 1e-8


def test_extended_vector_ops_known_answers():
    # crates/runtime/tests/solvers.rs:976-1115
    n = 256
    x, y, z = np.full(n, 3.0), np.full(n, 7.0), np.zeros(n)
    O.pointwise_mult(x, y, z)
    assert np.all(np.abs(z - 21.0) < 1e-10)
    x, y = np.full(n, 21.0), np.full(n, 7.0)
    O.pointwise_div(x, y, z)
    assert np.all(np.abs(z - 3.0) < 1e-10)
    x, y, w = np.full(n, 2.0), np.full(n, 3.0), np.zeros(n)
    O.waxpy(5.0, x, 10.0, y, w)
    assert np.all(np.abs(w - 40.0) < 1e-10)
    x, y = np.full(n, 10.0), np.full(n, 3.0)
    O.aypx(2.0, x, y)
    assert np.all(np.abs(y - 16.0) < 1e-10)
    x = np.full(n, 4.0)
    O.reciprocal(x)
    assert np.all(np.abs(x - 0.25) < 1e-10)
    x = np.full(n, -7.0)
    O.abs_val(x)
    assert np.all(np.abs(x - 7.0) < 1e-10)


@pytest.mark.parametrize("c", [492.4908687776044, -1000.0, 0.0, 3.5])
def test_laplacian_of_constant_is_zero(c):
    # crates/runtime/tests/properties.rs:13-36 (+ the saved shrink seed c = 492.4908687776044)
    n = 32
    h = 1.0 / (n - 1)
    out = np.zeros(n * n)
    O.apply_stencil(np.full(n * n, c), out, n, n, h, h, O.laplacian_5pt(h, h), ZD)
    tol = 1e-10 * (1.0 + abs(c))
    assert np.all(np.abs(out.reshape(n, n)[1:-1, 1:-1]) < tol)


def test_laplacian_linearity():
    # crates/runtime/tests/properties.rs:38-70
    n = 32
    h = 1.0 / (n - 1)
    u = quadratic_field(n, h)
    for alpha in (-100.0, -1.5, 0.3, 77.0):
        a, b = np.zeros(n * n), np.zeros(n * n)
        O.apply_stencil(u * alpha, a, n, n, h, h, O.laplacian_5pt(h, h), ZD)
        O.apply_stencil(u, b, n, n, h, h, O.laplacian_5pt(h, h), ZD)
        ai = a.reshape(n, n)[1:-1, 1:-1]
        bi = b.reshape(n, n)[1:-1, 1:-1]
        assert np.all(np.abs(ai - alpha * bi) < 1e-8 * (1 + np.abs(alpha * bi)))


# ---------------------------------------------------------------- solvers

def _cn_rhs(n, coeff):
    """b = u + coeff*Lap(u) with u the Gaussian IC (solvers.rs:53-63)."""
    h = 1.0 / (n - 1)
    st = O.laplacian_5pt(h, h)
    u = gaussian_ic(n, h)
    b = u.copy()
    O.stencil_axpy(coeff, u.copy(), b, n, n, st, ZD)
    return h, st, u, b


def test_cg_converges():
    # solvers.rs:43-76
    n = 32
    h, st, u, b = _cn_rhs(n, -0.01)
    x = np.zeros(n * n)
    it, res, reason = O.cg_solve(x, b, n, n, -0.01, st, 1e-8, 500)
    assert reason == 0 and it < 200


def test_cg_zero_rhs():
    # solvers.rs:79-97
    n = 16
    h = 1.0 / (n - 1)
    x = np.zeros(n * n)
    it, res, reason = O.cg_solve(x, np.zeros(n * n), n, n, -0.01, O.laplacian_5pt(h, h), 1e-10, 100)
    assert reason == 0 and it == 0


def test_pcg_identity_matches_cg():
    # solvers.rs:101-154
    n = 32
    h, st, u, b = _cn_rhs(n, -0.01)
    x1, x2 = np.zeros(n * n), np.zeros(n * n)
    s1 = O.cg_solve(x1, b, n, n, -0.01, st, 1e-8, 500)
    s2 = O.cg_solve(x2, b, n, n, -0.01, st, 1e-8, 500, pc=O.IdentityPC(n * n))
    assert s1[2] == 0 and s2[2] == 0 and abs(s1[0] - s2[0]) <= 2


def test_cg_max_iterations_reason():
    # solvers.rs:1151-1176
    n = 32
    h = 1.0 / (n - 1)
    b = gaussian_ic(n, h)
    x = np.zeros(n * n)
    it, res, reason = O.cg_solve(x, b, n, n, -0.01, O.laplacian_5pt(h, h), 1e-15, 2)
    assert reason == 1 and it == 2


def test_pipelined_cg_matches_cg():
    # solvers.rs:322-379
    n = 32
    h, st, u, b = _cn_rhs(n, -0.01)
    x1, x2 = np.zeros(n * n), np.zeros(n * n)
    assert O.cg_solve(x1, b, n, n, -0.01, st, 1e-8, 500)[2] == 0
    assert O.pipelined_cg_solve(x2, b, n, n, -0.01, st, 1e-8, 500)[2] == 0
    assert np.max(np.abs(x1 - x2)) < 1e-6


@pytest.mark.parametrize("coeff,tol,maxit,pc", [(-0.01, 1e-8, 500, False), (-0.01, 1e-8, 500, True),
                                                (-0.5, 1e-6, 1000, False)])
def test_bicgstab_converges(coeff, tol, maxit, pc):
    # solvers.rs:211-320
    n = 32
    h, st, u, b = _cn_rhs(n, coeff)
    x = np.zeros(n * n)
    it, res, reason = O.bicgstab_solve(x, b, n, n, coeff, st, tol, maxit,
                                       pc=O.IdentityPC(n * n) if pc else None)
    assert reason == 0


def test_gmres_known_answers():
    # solvers.rs:1221-1446
    n = 32
    h, st, u, b = _cn_rhs(n, -0.01)
    x = np.zeros(n * n)
    assert O.gmres_solve(x, b, n, n, -0.01, st, 30, 1e-8, 500)[2] == 0
    xc, xg = np.zeros(n * n), np.zeros(n * n)
    O.cg_solve(xc, b, n, n, -0.01, st, 1e-8, 500)
    O.gmres_solve(xg, b, n, n, -0.01, st, 50, 1e-8, 500)
    assert np.max(np.abs(xc - xg)) < 1e-6
    x = np.zeros(n * n)
    assert O.gmres_solve(x, b, n, n, -0.01, st, 30, 1e-8, 500, pc=O.IdentityPC(n * n))[2] == 0
    x = np.zeros(n * n)
    it, res, reason = O.gmres_solve(x, b, n, n, -0.01, st, 5, 1e-8, 500)
    assert reason == 0 and it > 5
    h2, st2, u2, b2 = _cn_rhs(n, -0.5)
    x = np.zeros(n * n)
    assert O.gmres_solve(x, b2, n, n, -0.5, st2, 100, 1e-6, 1000)[2] == 0


def test_multigrid_depth_hierarchy():
    # solvers.rs:813-841
    for n, depth in ((64, 5), (32, 4), (8, 2)):
        h = 1.0 / (n - 1)
        assert O.Multigrid(n, n, h, h, 2, 2, 2.0 / 3.0, mode=0).depth() == depth


def test_multigrid_reduces_residual():
    # crates/runtime/tests/analytical.rs:447-521 (Jacobi smoother)
    n = 64
    h = 1.0 / (n - 1)
    b = sin_sin_field(n, h)
    mg = O.Multigrid(n, n, h, h, 3, 3, 2.0 / 3.0, mode=0)
    assert mg.depth() >= 3
    x = np.zeros(n * n)
    st = O.laplacian_5pt(h, h)
    prev = np.finfo(float).max
    for _ in range(10):
        mg.v_cycle(x, b)
        ax = np.zeros(n * n)
        O.apply_stencil(x, ax, n, n, h, h, st, ZD)
        r = b.copy()
        O.axpy(-1.0, ax, r)
        res = np.sqrt(O.dot(r, r))
        assert res < prev
        prev = res
    assert prev < 10.0


def test_pcg_multigrid_fewer_iterations():
    # solvers.rs:156-208: Crank-Nicolson step (I - dt/2 alpha Lap) with MG-PCG vs plain CG
    n = 64
    h = 1.0 / (n - 1)
    coeff = -0.5 * 0.1 * 1.0
    st = O.laplacian_5pt(h, h)
    u = gaussian_ic(n, h)
    b = u.copy()
    O.stencil_axpy(-coeff, u.copy(), b, n, n, st, ZD)  # (I + dt/2 Lap) u
    x1 = u.copy()
    mg = O.Multigrid(n, n, h, h, 2, 2, 2.0 / 3.0, mode=0)
    s_pcg = O.cg_solve(x1, b, n, n, coeff, st, 1e-8, 100, pc=mg)
    x2 = u.copy()
    s_cg = O.cg_solve(x2, b, n, n, coeff, st, 1e-8, 500)
    assert s_pcg[2] == 0 and s_cg[2] == 0 and s_pcg[0] <= s_cg[0]


def test_reference_mg_odd_levels_rejected():
    # multigrid.rs:121-135 builds 257 -> 128 for a 514 grid; prolong then indexes coarse row 128 of
    # 128 (a panic in the reference).  The oracle reports it as a dimension error.
    with pytest.raises(O.OracleError):
        O.prolong(np.zeros(128 * 128), np.zeros(257 * 257), (128, 128), (257, 257))
