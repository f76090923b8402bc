"""GPU parity of every backend op against the CPU oracle, through the C ABI.

F64 elementwise, stencil, convection-diffusion and multigrid-transfer results use the
reference's own fma nesting and are required to be BITWISE equal to the oracle.
Reductions sum in a different (compensated, fixed-tree) order: the bar is
|gpu - oracle| <= 1e-13 * sum|x_i y_i| (dot, norm^2, sum).  F32 ops are compared with a
float32 numpy restatement to 2 ulp-scale relative tolerance (4e-7 relative of the operands).
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RED_TOL = 1e-13


@pytest.fixture(scope="module")
def be():
    from fluxion_b200 import CudaBackend
    return CudaBackend.get(0)


def up(be, a):
    return be.upload_f64(np.ascontiguousarray(a, dtype=np.float64))


def rand(rng, n, lo=-1.0, hi=1.0):
    return rng.uniform(lo, hi, n)


SHAPES = [(3, 3), (4, 5), (33, 31), (67, 67), (130, 65), (257, 259)]


def _stencils(dx, dy):
    from fluxion_b200 import Stencil
    rng = np.random.default_rng(7)
    five = Stencil.laplacian_2d_5pt(dx, dy)
    nine = Stencil.laplacian_2d_9pt(dx, dy)
    # arbitrary 5 weights in a shuffled order (ops.rs:898-916 handles any order)
    wts = rng.normal(size=5)
    custom5 = Stencil([(0, 1, wts[0]), (-1, 0, wts[1]), (0, 0, wts[2]), (1, 0, wts[3]), (0, -1, wts[4])])
    # generic 3-entry stencil (entry-order path, ops.rs:869-883)
    generic = Stencil([(0, 0, 2.0), (1, 1, -0.5), (-1, 0, 0.25)])
    return {"5pt": five, "9pt": nine, "custom5": custom5, "generic": generic}


def _bcs_cases():
    from fluxion_b200 import Boundaries, BoundaryCondition as B
    return {
        "dirichlet0": Boundaries.zero_dirichlet(),
        "dirichlet100": Boundaries.uniform(B.Dirichlet(100.0)),
        "mixed": Boundaries(B.Dirichlet(1.0), B.Neumann(0.5), B.Robin(1.0, 2.0, 0.3), B.Robin(0.0, 0.0, 1.0)),
    }


# ---------------------------------------------------------------- elementwise

@pytest.mark.parametrize("n", [1, 31, 1000, 4097, 100003])
def test_elementwise_bitwise(be, n):
    rng = np.random.default_rng(n)
    x, y = rand(rng, n), rand(rng, n, 0.5, 2.0)
    cases = [
        ("axpy", lambda X, Y, Z: be.axpy(1.7, X, Y), lambda x, y, z: O.axpy(1.7, x, y), "y"),
        ("scale", lambda X, Y, Z: be.scale(Y, -0.3), lambda x, y, z: O.scale(y, -0.3), "y"),
        ("waxpy", lambda X, Y, Z: be.waxpy(0.7, X, -1.3, Y, Z), lambda x, y, z: O.waxpy(0.7, x, -1.3, y, z), "z"),
        ("aypx", lambda X, Y, Z: be.aypx(2.5, X, Y), lambda x, y, z: O.aypx(2.5, x, y), "y"),
        ("mult", lambda X, Y, Z: be.pointwise_mult(X, Y, Z), lambda x, y, z: O.pointwise_mult(x, y, z), "z"),
        ("div", lambda X, Y, Z: be.pointwise_div(X, Y, Z), lambda x, y, z: O.pointwise_div(x, y, z), "z"),
        ("max", lambda X, Y, Z: be.pointwise_max(X, Y, Z), lambda x, y, z: O.pointwise_max(x, y, z), "z"),
        ("min", lambda X, Y, Z: be.pointwise_min(X, Y, Z), lambda x, y, z: O.pointwise_min(x, y, z), "z"),
        ("recip", lambda X, Y, Z: be.reciprocal(Y), lambda x, y, z: O.reciprocal(y), "y"),
        ("abs", lambda X, Y, Z: be.abs_val(X), lambda x, y, z: O.abs_val(x), "x"),
        ("fill", lambda X, Y, Z: be.fill(Z, 3.25), lambda x, y, z: O.fill(z, 3.25), "z"),
        ("copy", lambda X, Y, Z: be.copy(X, Z), lambda x, y, z: O.copy(x, z), "z"),
    ]
    for name, g, o, which in cases:
        X, Y, Z = up(be, x), up(be, y), be.allocate(n)
        xo, yo, zo = x.copy(), y.copy(), np.zeros(n)
        g(X, Y, Z)
        o(xo, yo, zo)
        got = {"x": X, "y": Y, "z": Z}[which].to_numpy()
        want = {"x": xo, "y": yo, "z": zo}[which]
        assert np.array_equal(got.view(np.uint64), want.view(np.uint64)), name


def test_pcg_fused_update_bitwise(be):
    rng = np.random.default_rng(3)
    n = 70001
    vs = [rand(rng, n) for _ in range(7)]
    G = [up(be, v) for v in vs]
    C_ = [v.copy() for v in vs]
    be.pipelined_cg_fused(0.37, 0.81, *G)
    O.pcg_fused_update(0.37, 0.81, *C_)
    for g, c in zip(G[:6], C_[:6]):
        assert np.array_equal(g.to_numpy(), c)
    # the fused variant also returns (r.r, r.w) of the updated vectors
    G = [up(be, v) for v in vs]
    rr, rw = be.pipelined_cg_fused_dot2(0.37, 0.81, *G)
    r, w = C_[4], C_[5]
    assert abs(rr - O.dot(r, r)) <= RED_TOL * np.sum(r * r)
    assert abs(rw - O.dot(r, w)) <= RED_TOL * np.sum(np.abs(r * w))


# ---------------------------------------------------------------- reductions

@pytest.mark.parametrize("n", [0, 1, 33, 4096, 4097, 1 << 20, 3_000_017])
def test_reductions(be, n):
    rng = np.random.default_rng(11 + n)
    x, y = rand(rng, n), rand(rng, n)
    X, Y = up(be, x), up(be, y)
    if n == 0:
        assert be.reduce_sum(X) == 0.0 and be.norm_l2(X) == 0.0 and be.dot(X, Y) == 0.0
        assert be.reduce_max(X) == -np.inf and be.reduce_min(X) == np.inf
        return
    assert abs(be.dot(X, Y) - O.dot(x, y)) <= RED_TOL * np.sum(np.abs(x * y))
    assert abs(be.norm_l2(X) ** 2 - O.norm_l2(x) ** 2) <= 2 * RED_TOL * np.sum(x * x)
    assert abs(be.reduce_sum(X) - O.reduce_sum(x)) <= RED_TOL * np.sum(np.abs(x))
    assert be.reduce_max(X) == O.reduce_max(x) and be.reduce_min(X) == O.reduce_min(x)
    a, b = be.dot2(X, Y, X, X)
    o1, o2 = O.dot2(x, y, x, x)
    assert abs(a - o1) <= RED_TOL * np.sum(np.abs(x * y)) and abs(b - o2) <= RED_TOL * np.sum(x * x)
    # determinism: same inputs, same bits
    assert be.dot(X, Y) == be.dot(X, Y)


@pytest.mark.parametrize("n", [1, 4097, 1 << 20, 3_000_017])
def test_reductions_f32(be, n):
    """F32 dots: each product of two floats is exact in FP64; the sum is within 1e-13 sum|x_i y_i|
    of the exact FP64 sum of the same float32 data (math.fsum)."""
    import math
    rng = np.random.default_rng(29 + n)
    x, y = rand(rng, n).astype(np.float32), rand(rng, n).astype(np.float32)
    X, Y = be.upload_f32(x), be.upload_f32(y)
    xd, yd = x.astype(np.float64), y.astype(np.float64)
    exact_xy, exact_xx = math.fsum(xd * yd), math.fsum(xd * xd)
    assert abs(be.dot(X, Y) - exact_xy) <= RED_TOL * np.sum(np.abs(xd * yd))
    a, b = be.dot2(X, Y, X, X)
    assert abs(a - exact_xy) <= RED_TOL * np.sum(np.abs(xd * yd)) and abs(b - exact_xx) <= RED_TOL * exact_xx
    assert abs(be.norm_l2(X) ** 2 - exact_xx) <= 2 * RED_TOL * exact_xx
    assert be.dot(X, Y) == be.dot(X, Y)


@pytest.mark.parametrize("n", [4099, 1 << 20])
def test_axpy_f32_is_one_rounding(be, n):
    """F32 axpy is fma(alpha, x, y) in single precision (one rounding), on the 16-byte vector path
    and its scalar tail alike: equal to the exactly rounded FP64 result except where that double
    rounding could differ (at most one ulp)."""
    rng = np.random.default_rng(77 + n)
    x, y = rand(rng, n).astype(np.float32), rand(rng, n).astype(np.float32)
    a = np.float32(0.3712)
    X, Y = be.upload_f32(x), be.upload_f32(y)
    be.axpy(float(a), X, Y)
    got = Y.to_numpy().astype(np.float32)
    want = (np.float64(a) * x.astype(np.float64) + y.astype(np.float64)).astype(np.float32)
    ulp = np.spacing(np.abs(want))
    assert np.all(np.abs(got - want) <= ulp)
    assert np.mean(got == want) > 0.999


def test_compensated_dot_recovers_cancelled_terms(be):
    # +B and -B pairs cancel exactly; only the small terms survive.  A plain double sum
    # loses them, the compensated (twice-working-precision) sum must not.
    import math
    rng = np.random.default_rng(5)
    n = 1 << 15
    big = rng.choice([-1.0, 1.0], n) * 1e16
    small = rng.uniform(0.0, 1.0, n)
    x = np.concatenate([big, -big, small])
    rng.shuffle(x)
    exact = math.fsum(small)
    got = be.dot(up(be, x), up(be, np.ones(x.size)))
    assert abs(got - exact) <= 1e-9 * exact


def test_nan_semantics_of_max_min(be):
    x = np.array([1.0, np.nan, 3.0, -2.0])
    X = up(be, x)
    assert be.reduce_max(X) == 3.0 and be.reduce_min(X) == -2.0  # f64::max/min ignore NaN


# ---------------------------------------------------------------- stencil

@pytest.mark.parametrize("rows,cols", SHAPES)
def test_apply_stencil_bitwise(be, rows, cols):
    from fluxion_b200 import Grid
    dx, dy = 1.0 / (cols - 1), 1.0 / (rows - 1) * 1.3
    g = Grid.new(rows, cols, dx, dy)
    rng = np.random.default_rng(rows * 1000 + cols)
    x = rand(rng, rows * cols)
    coeff = rand(rng, rows * cols, 0.5, 1.5)
    X, CF = up(be, x), up(be, coeff)
    for sname, st in _stencils(dx, dy).items():
        for bname, bc in _bcs_cases().items():
            out = be.allocate(rows * cols)
            be.apply_stencil(X, out, g, st, bc)
            want = np.zeros(rows * cols)
            O.apply_stencil(x, want, rows, cols, dx, dy, st.as_triples(), bc.as_tuples())
            assert np.array_equal(out.to_numpy(), want), (sname, bname)
            be.apply_stencil_var(X, out, CF, g, st, bc)
            O.apply_stencil_var(x, want, coeff, rows, cols, dx, dy, st.as_triples(), bc.as_tuples())
            assert np.array_equal(out.to_numpy(), want), ("var", sname, bname)
        y0 = rand(rng, rows * cols)
        Y = up(be, y0)
        be.stencil_axpy(-0.7, X, Y, g, st, _bcs_cases()["dirichlet0"])
        yw = y0.copy()
        O.stencil_axpy(-0.7, x, yw, rows, cols, st.as_triples())
        assert np.array_equal(Y.to_numpy(), yw), ("axpy", sname)


def test_stencil_f32_matches_float32_restatement(be):
    from fluxion_b200 import Boundaries, Grid, Stencil
    rows, cols = 129, 257
    h = 1.0 / 256
    g = Grid.new(rows, cols, h, h)
    rng = np.random.default_rng(2)
    x = rand(rng, rows * cols).astype(np.float32)
    X = be.upload_f32(x)
    out = be.allocate(rows * cols, dtype=0)
    st = Stencil.laplacian_2d_5pt(h, h)
    be.apply_stencil(X, out, g, st, Boundaries.zero_dirichlet())
    a = x.reshape(rows, cols).astype(np.float64)
    ref = np.zeros_like(a)
    w = 1.0 / (h * h)
    ref[1:-1, 1:-1] = (-4 * w * a[1:-1, 1:-1] + w * (a[:-2, 1:-1] + a[2:, 1:-1] + a[1:-1, :-2] + a[1:-1, 2:]))
    got = out.to_numpy().reshape(rows, cols)
    scale = w * (np.abs(a[1:-1, 1:-1]) * 4 + np.abs(a[:-2, 1:-1]) + np.abs(a[2:, 1:-1]) + np.abs(a[1:-1, :-2])
                 + np.abs(a[1:-1, 2:]))
    assert np.all(np.abs(got[1:-1, 1:-1] - ref[1:-1, 1:-1]) <= 4e-7 * scale + 1e-30)
    assert np.all(got[0] == 0) and np.all(got[-1] == 0)


def test_stencil_errors(be):
    from fluxion_b200 import (BackendError, Boundaries, DimensionMismatch, Grid, InvalidArgument,
                              InvalidStencil, Stencil)
    g = Grid.square(8, 0.1)
    X, Y = be.allocate(64), be.allocate(64)
    with pytest.raises(DimensionMismatch):
        be.apply_stencil(X, be.allocate(63), g, Stencil.laplacian_2d_5pt(0.1, 0.1), Boundaries.zero_dirichlet())
    with pytest.raises(BackendError):
        be.apply_stencil(X, Y, g, Stencil.laplacian_2d_5pt(0.1, 0.1), Boundaries.periodic())
    with pytest.raises(InvalidStencil):
        be.apply_stencil(X, Y, g, Stencil([(2, 0, 1.0), (0, 0, 1.0)]), Boundaries.zero_dirichlet())
    with pytest.raises(InvalidArgument):
        be.apply_stencil(X, X, g, Stencil.laplacian_2d_5pt(0.1, 0.1), Boundaries.zero_dirichlet())
    with pytest.raises(DimensionMismatch):
        be.axpy(1.0, X, be.allocate(65))


def test_known_answers_on_gpu(be):
    # ops.rs:1201-1338 through the CUDA path
    from fluxion_b200 import Boundaries, BoundaryCondition, Grid, Stencil
    from tests.helpers import quadratic_field
    buf = be.allocate(16)
    be.fill(buf, 3.0)
    assert abs(be.norm_l2(buf) - 12.0) < 1e-12
    x, y = up(be, [1.0, 2.0, 3.0]), up(be, [10.0, 20.0, 30.0])
    be.axpy(2.0, x, y)
    assert np.allclose(y.to_numpy(), [12.0, 24.0, 36.0], atol=1e-14, rtol=0)
    n = 32
    h = 1.0 / (n - 1)
    g = Grid.square(n, h)
    out = be.allocate(n * n)
    be.apply_stencil(up(be, quadratic_field(n, h)), out, g, Stencil.laplacian_2d_5pt(h, h),
                     Boundaries.zero_dirichlet())
    assert np.all(np.abs(out.to_numpy().reshape(n, n)[2:-2, 2:-2] - 4.0) < 1e-10)
    n = 16
    h = 1.0 / (n - 1)
    g = Grid.square(n, h)
    be.apply_stencil(up(be, np.full(n * n, 50.0)), out := be.allocate(n * n), g, Stencil.laplacian_2d_5pt(h, h),
                     Boundaries.uniform(BoundaryCondition.Dirichlet(100.0)))
    o = out.to_numpy().reshape(n, n)
    assert np.all(np.abs(o[0] - 100) < 1e-12) and np.all(np.abs(o[-1] - 100) < 1e-12)
    be.apply_stencil(up(be, np.full(n * n, 42.0)), out, g, Stencil.laplacian_2d_5pt(h, h),
                     Boundaries.uniform(BoundaryCondition.Neumann(0.0)))
    assert np.all(np.abs(out.to_numpy().reshape(n, n)[0] - 42.0) < 1e-10)


# ---------------------------------------------------------------- conv-diff

@pytest.mark.parametrize("rows,cols", [(3, 3), (33, 47), (129, 129)])
def test_conv_diff_bitwise(be, rows, cols):
    from fluxion_b200 import Boundaries, Grid
    dx, dy = 1.0 / (cols - 1), 1.0 / (rows - 1)
    g = Grid.new(rows, cols, dx, dy)
    rng = np.random.default_rng(rows + cols)
    u, k, vx, vy = (rand(rng, rows * cols) for _ in range(4))
    U, K, VX, VY = (up(be, a) for a in (u, k, vx, vy))
    out = be.allocate(rows * cols)
    be.apply_conv_diff(U, out, K, VX, VY, g, Boundaries.zero_dirichlet())
    want = np.zeros(rows * cols)
    O.apply_conv_diff(u, want, k, vx, vy, rows, cols, dx, dy)
    assert np.array_equal(out.to_numpy(), want)
    y0 = rand(rng, rows * cols)
    Y = up(be, y0)
    be.conv_diff_axpy(0.3, U, Y, K, VX, VY, g, Boundaries.zero_dirichlet())
    O.conv_diff_axpy(0.3, u, y0, k, vx, vy, rows, cols, dx, dy)
    assert np.array_equal(Y.to_numpy(), y0)


# ---------------------------------------------------------------- multigrid primitives

@pytest.mark.parametrize("fine,coarse", [((64, 64), (32, 32)), ((65, 33), (33, 17)), ((8, 8), (4, 4)),
                                         ((7, 9), (4, 5))])
def test_reference_transfer_bitwise(be, fine, coarse):
    from fluxion_b200 import Grid
    fg, cg = Grid.new(*fine, 0.1, 0.1), Grid.new(*coarse, 0.2, 0.2)
    rng = np.random.default_rng(1)
    f, c = rand(rng, fg.len()), rand(rng, cg.len())
    F, Cb = up(be, f), be.allocate(cg.len())
    be.restrict(F, Cb, fg, cg)
    cw = np.zeros(cg.len())
    O.restrict(f, cw, fine, coarse)
    assert np.array_equal(Cb.to_numpy(), cw)
    F2 = up(be, f)
    be.prolong(up(be, c), F2, cg, fg)
    fw = f.copy()
    O.prolong(c, fw, coarse, fine)
    assert np.array_equal(F2.to_numpy(), fw)


def test_reference_transfer_out_of_range_is_an_error(be):
    from fluxion_b200 import DimensionMismatch, Grid
    fg, cg = Grid.new(257, 257, 0.1, 0.1), Grid.new(128, 128, 0.2, 0.2)
    with pytest.raises(DimensionMismatch):
        be.prolong(be.allocate(cg.len()), be.allocate(fg.len()), cg, fg)


@pytest.mark.parametrize("rows,cols", [(3, 3), (16, 16), (33, 65), (130, 67)])
def test_lexicographic_weighted_jacobi_bitwise(be, rows, cols):
    from fluxion_b200 import Boundaries, Grid, Stencil
    dx = 1.0 / (cols - 1)
    g = Grid.new(rows, cols, dx, dx)
    rng = np.random.default_rng(rows)
    x, b = rand(rng, rows * cols), rand(rng, rows * cols)
    for st in (Stencil.laplacian_2d_5pt(dx, dx), Stencil.laplacian_2d_9pt(dx, dx)):
        X, B = up(be, x), up(be, b)
        xo = x.copy()
        for _ in range(3):
            be.weighted_jacobi(X, B, 2.0 / 3.0, g, st, Boundaries.zero_dirichlet())
            O.weighted_jacobi(xo, b, 2.0 / 3.0, rows, cols, st.as_triples())
        assert np.array_equal(X.to_numpy(), xo)


@pytest.mark.parametrize("n", [17, 33, 129, 257])
def test_vertex_primitives_bitwise(be, n):
    rng = np.random.default_rng(n)
    h = 1.0 / (n - 1)
    a5 = [4 / h ** 2, -1 / h ** 2, -1 / h ** 2, -1 / h ** 2, -1 / h ** 2]
    x, b = rand(rng, n * n), rand(rng, n * n)
    X, B, Yb = up(be, x), up(be, b), up(be, np.zeros(n * n))
    be.jacobi_sweep(X, Yb, B, 0.8, n, n, a5)
    yo = np.zeros(n * n)
    O.jacobi_sweep(x, yo, b, 0.8, n, n, a5)
    assert np.array_equal(Yb.to_numpy(), yo)
    R = up(be, np.zeros(n * n))
    be.residual5(X, B, R, n, n, a5)
    ro = np.zeros(n * n)
    O.residual(x, b, ro, n, n, a5)
    assert np.array_equal(R.to_numpy(), ro)
    nc = (n - 1) // 2 + 1
    Cb = be.allocate(nc * nc)
    be.restrict_fw(X, Cb, (n, n), (nc, nc))
    co = np.zeros(nc * nc)
    O.restrict_fw(x, co, (n, n), (nc, nc))
    assert np.array_equal(Cb.to_numpy(), co)
    F = up(be, x)
    be.prolong_bilinear(Cb, F, (nc, nc), (n, n))
    fo = x.copy()
    O.prolong_bilinear(co, fo, (nc, nc), (n, n))
    assert np.array_equal(F.to_numpy(), fo)


def test_zero_boundaries(be):
    rows, cols = 37, 41
    x = np.random.default_rng(0).uniform(size=rows * cols)
    X = up(be, x)
    be.zero_boundaries(X, rows, cols)
    O.zero_boundaries(x, rows, cols)
    assert np.array_equal(X.to_numpy(), x)


def test_f32_upload_roundtrip_and_conversion(be):
    x = np.random.default_rng(0).uniform(size=1001)
    X = be.upload_f32(x.astype(np.float32))
    assert np.array_equal(X.to_numpy(), x.astype(np.float32))
    out = np.empty(1001)
    X.copy_to_host_f64(out)
    assert np.array_equal(out, x.astype(np.float32).astype(np.float64))
    Y = be.upload_f64(x)
    o32 = np.empty(1001, dtype=np.float32)
    Y.copy_to_host_f32(o32)
    assert np.array_equal(o32, x.astype(np.float32))
