"""The batched solver (fx_batch_*) on mixed-size batches: its operator and its V-cycle equal the
single-problem operator and conv-diff cycle bit for bit (F64 and F32 cycles), and its BiCGSTAB
matches the oracle's solve of every problem (same stop reason, iterations within one, solutions
within 1e-8, the tolerance met on the residual the oracle recomputes); a graph-replayed batch
gives the same bits as one launched directly."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu

NU = 1e-2


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


def _batch(dev, sides, seed=0, nu=NU, cycle_dtype=None):
    from fluxion_b200.batch import BatchSolver
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    be = dev.backend()
    vx, vy, f = [], [], []
    for k, s in enumerate(sides):
        a, b = stream_velocity(s - 2, seed + 2 * k)
        vx.append(a)
        vy.append(b)
        f.append(poisson_uniform_rhs(s - 2, seed + 2 * k + 1))
    VX, VY = be.upload_f64(np.concatenate(vx)), be.upload_f64(np.concatenate(vy))
    B = BatchSolver(dev, sides, nu, VX, VY, cycle_dtype=cycle_dtype)
    return B, vx, vy, f, be


def _single(dev, side, vx, vy, nu=NU):
    from fluxion_b200 import ConvDiffOperator, Field, Grid
    g = Grid.square(side, 1.0 / (side - 1))
    VX, VY = Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev)
    return g, ConvDiffOperator(g, VX, VY, -nu, sigma=0.0, coeff=1.0), (VX, VY)


SIDES = [65, 129, 33, 257, 65, 17, 129]


def test_batched_operator_equals_single_problem_operator(dev):
    from fluxion_b200 import DType, Field
    B, vx, vy, f, be = _batch(dev, SIDES, seed=3)
    rng = np.random.default_rng(4)
    v = rng.uniform(-1, 1, B.offsets[-1])
    out = be.allocate(B.offsets[-1], DType.F64)
    B.apply(be.upload_f64(v), out)
    got = out.to_numpy()
    for p, s in enumerate(SIDES):
        g, op, keep = _single(dev, s, vx[p], vy[p])
        w = Field.zeros(g, DType.F64, dev)
        op.apply(Field.from_f64(g, v[B.offsets[p]:B.offsets[p + 1]], dev), w)
        assert np.array_equal(got[B.offsets[p]:B.offsets[p + 1]], w.to_vec_f64()), p


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_batched_cycle_equals_single_problem_cycle(dev, dtype):
    from fluxion_b200 import ConvDiffMultigrid, DType, Field
    dt = DType.F32 if dtype == "f32" else DType.F64
    B, vx, vy, f, be = _batch(dev, SIDES, seed=5, cycle_dtype=dt)
    assert B.depths == [3, 4, 2, 5, 3, 1, 4]
    r = np.concatenate(f)
    z = be.allocate(B.offsets[-1], DType.F64)
    for _ in range(2):  # the second application starts from the buffers the first left
        B.precondition(z, be.upload_f64(r))
    got = z.to_numpy()
    for p, s in enumerate(SIDES):
        g, op, keep = _single(dev, s, vx[p], vy[p])
        mg = ConvDiffMultigrid(op, dtype=dt)
        zz = Field.zeros(g, DType.F64, dev)
        mg.apply(zz, Field.from_f64(g, f[p], dev))
        assert mg.depth() == B.depths[p]
        assert np.array_equal(got[B.offsets[p]:B.offsets[p + 1]], zz.to_vec_f64()), p


def test_batched_bicgstab_matches_oracle_on_16_problems(dev):
    from fluxion_b200 import DType
    sides = [65, 129, 257, 33, 65, 129, 513, 65, 257, 129, 33, 65, 129, 257, 65, 129]
    B, vx, vy, f, be = _batch(dev, sides, seed=11)
    b = be.upload_f64(np.concatenate(f))
    x = be.allocate(B.offsets[-1], DType.F64)
    stats, run = B.bicgstab(x, b, 1e-10, 200)
    xs = x.to_numpy()
    for p, s in enumerate(sides):
        h = 1.0 / (s - 1)
        oop = O.cd_op(s, s, h, h, vx[p], vy[p], kappa=None, kappa_s=-NU, sigma=0.0, coeff=1.0)
        tol = 1e-10 * np.linalg.norm(f[p])
        xo = np.zeros(s * s)
        it, _, reason = O.bicgstab_solve_op(xo, f[p], oop, tol, 200, O.CdMultigrid(oop))
        st = stats[p]
        xp = xs[B.offsets[p]:B.offsets[p + 1]]
        assert st.converged() and reason == 0, (p, st, it, reason)
        assert abs(st.iterations - it) <= 1, (p, st.iterations, it)
        assert np.linalg.norm(O.op_apply(oop, xp) - f[p]) < 1.01 * tol
        assert rel_err(xp, xo) < 1e-8
    assert run == max(st.iterations for st in stats) + 1


def test_graph_replay_equals_direct_launches_and_max_iterations(dev):
    from fluxion_b200 import ConvergenceReason, DType
    sides = [65, 129, 33, 257]
    B, vx, vy, f, be = _batch(dev, sides, seed=21)
    b = be.upload_f64(np.concatenate(f))
    outs = []
    for use_graph in (True, False, True):
        x = be.allocate(B.offsets[-1], DType.F64)
        stats, _ = B.bicgstab(x, b, 1e-10, 200, use_graph=use_graph)
        outs.append((x.to_numpy(), [(s.iterations, s.residual) for s in stats]))
    assert all(np.array_equal(o[0], outs[0][0]) and o[1] == outs[0][1] for o in outs)
    x = be.allocate(B.offsets[-1], DType.F64)
    stats, run = B.bicgstab(x, b, 1e-14, 2)
    assert all(s.reason == ConvergenceReason.MaxIterations and s.iterations == 2 for s in stats)
