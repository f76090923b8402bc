"""Time steppers over the CUDA path: the reference's own tests of CrankNicolsonSolver, ImexSolver,
BdfSolver and the explicit DiffusionSolver (crates/runtime/tests/solvers.rs, analytical.rs,
src/solver.rs), restated; one Crank-Nicolson step against the same step assembled from the
oracle's operations; and graph-replayed explicit steps against eager ones."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import gaussian_ic, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


def _setup(n, dev):
    from fluxion_b200 import Boundaries, Field, Grid
    h = 1.0 / (n - 1)
    g = Grid.square(n, h)
    data = gaussian_ic(n, h)
    return g, h, Boundaries.zero_dirichlet(), data, Field.from_f64(g, data, dev)


def test_crank_nicolson_known_answers(dev):
    from fluxion_b200 import DType, Field
    from fluxion_b200.steppers import CrankNicolsonSolver
    g, h, bc, data, u = _setup(32, dev)
    s = CrankNicolsonSolver.new(g, 0.01, 0.01, bc, dev, 1e-8, 200)  # solvers.rs:436-460
    st = s.step(u, None)
    assert st.converged() and s.steps_done() == 1
    s = CrankNicolsonSolver.with_multigrid(g, 0.01, 0.01, bc, dev, 1e-8, 200, 2, 2, 2.0 / 3.0)  # :463-507
    u = Field.from_f64(g, data, dev)
    s.step_n(u, 200)
    peak = u.to_vec_f64().max()
    assert np.isfinite(peak) and 0.0 < peak < data.max() and s.steps_done() == 200
    assert abs(s.sim_time() - 2.0) < 1e-12
    s = CrankNicolsonSolver.new(g, 0.01, 0.01, bc, dev, 1e-8, 200)  # :510-533
    u = Field.zeros(g, DType.F64, dev)
    src = Field.zeros(g, DType.F64, dev)
    src.fill(1.0)
    assert s.step(u, src).converged() and u.norm_l2() > 1e-10


def test_chebyshev_fewer_iterations_than_jacobi(dev):
    """solvers.rs:842-893 and analytical.rs:523-575: PCG on a Crank-Nicolson step converges
    with either smoother of the reference multigrid, in no more iterations with Chebyshev."""
    from fluxion_b200 import Field, SmootherKind
    from fluxion_b200.steppers import CrankNicolsonSolver
    g, h, bc, data, _ = _setup(64, dev)
    stats = {}
    for sm in (SmootherKind.Jacobi, SmootherKind.Chebyshev):
        s = CrankNicolsonSolver.with_multigrid_smoother(g, 1.0, 0.1, bc, dev, 1e-8, 100, 2, 2, 2.0 / 3.0, sm)
        stats[sm] = s.step(Field.from_f64(g, data, dev), None)
        assert stats[sm].converged()
    assert stats[SmootherKind.Chebyshev].iterations <= stats[SmootherKind.Jacobi].iterations
    s = CrankNicolsonSolver.with_multigrid_smoother(g, 0.01, 0.01, bc, dev, 1e-10, 200, 3, 3, 2.0 / 3.0,
                                                    SmootherKind.Chebyshev)
    assert s.step(Field.from_f64(g, data, dev), None).converged()


def test_imex_known_answers(dev):
    from fluxion_b200 import Field
    from fluxion_b200.steppers import ImexSolver
    g, h, bc, data, u = _setup(32, dev)
    s = ImexSolver.new(g, 0.01, 0.0, 0.0, 0.01, bc, dev, 1e-8, 200)  # solvers.rs:1449-1486
    s.step_n(u, 50)
    peak = u.to_vec_f64().max()
    assert np.isfinite(peak) and peak < data.max() and s.steps_done() == 50
    s = ImexSolver.new(g, 0.01, 0.5, 0.0, 0.001, bc, dev, 1e-8, 200)  # :1489-1518
    u = Field.from_f64(g, data, dev)
    n0 = u.norm_l2()
    s.step_n(u, 20)
    n1 = u.norm_l2()
    assert np.isfinite(n1) and 0.0 < n1 < 2.0 * n0
    s = ImexSolver.with_multigrid(g, 0.01, 0.0, 0.0, 0.01, bc, dev, 1e-8, 200, 2, 2, 2.0 / 3.0)  # :1521-1544
    assert s.step(Field.from_f64(g, data, dev)).converged()


def test_bdf_known_answers(dev):
    from fluxion_b200 import Field
    from fluxion_b200.steppers import BdfSolver
    g, h, bc, data, _ = _setup(32, dev)
    for order in (1, 2):  # solvers.rs:1805-1880
        s = BdfSolver.new(g, 0.01, 0.01, order, bc, dev, 1e-8, 200)
        u = Field.from_f64(g, data, dev)
        s.step_n(u, 50)
        peak = u.to_vec_f64().max()
        assert np.isfinite(peak) and peak < data.max() and s.steps_done() == 50 and s.order() == order
    s = BdfSolver.with_multigrid(g, 0.01, 0.01, 4, bc, dev, 1e-8, 200, 2, 2, 2.0 / 3.0)  # :1883-1905
    assert s.step(Field.from_f64(g, data, dev)).converged()
    with pytest.raises(ValueError):
        BdfSolver.new(g, 0.01, 0.01, 5, bc, dev, 1e-8, 200)


def test_crank_nicolson_step_matches_oracle(dev):
    """One multigrid-preconditioned step, on the GPU and from the oracle's operations in the
    order of implicit.rs:178-226."""
    from fluxion_b200.steppers import CrankNicolsonSolver
    n = 64
    g, h, bc, data, u = _setup(n, dev)
    alpha, dt = 1.0, 0.1
    s = CrankNicolsonSolver.with_multigrid(g, alpha, dt, bc, dev, 1e-10, 100, 2, 2, 2.0 / 3.0)
    st = s.step(u, None)
    hda = 0.5 * dt * alpha
    lap = O.laplacian_5pt(h, h)
    rhs = data.copy()
    O.stencil_axpy(hda, data.copy(), rhs, n, n, lap)
    mg = O.Multigrid(n, n, h, h, 2, 2, 2.0 / 3.0, mode=0)
    x = data.copy()
    it, _, reason = O.cg_solve(x, rhs, n, n, -hda, lap, 1e-10, 100, pc=mg)
    assert st.converged() and reason == 0 and abs(st.iterations - it) <= 1
    assert rel_err(u.to_vec_f64(), x) < 1e-9


def test_diffusion_solver_known_answers(dev):
    """solver.rs:676-800 (unit tests) and solvers.rs rk2/rk4 diffusion tests."""
    from fluxion_b200 import Boundaries, DType, Field, Grid
    from fluxion_b200.steppers import DiffusionSolver, TimeScheme
    g, h, bc, data, u = _setup(64, dev)
    s = DiffusionSolver.new(g, 0.01, None, dev)
    s.step_n(u, 100)
    peak = u.to_vec_f64().max()
    assert 0.0 < peak < data.max()
    assert abs(s.dt() - 0.4 * h * h / (4 * 0.01)) < 1e-18
    n = 32
    g32 = Grid.square(n, 1.0 / (n - 1))
    u = Field.from_f64(g32, np.ones(n * n), dev)
    s = DiffusionSolver.new(g32, 0.01, None, dev)
    s.step_n(u, 10)
    assert s.steps_done() == 10
    s.step_n(u, 5)
    assert s.steps_done() == 15
    u = Field.zeros(g32, DType.F64, dev)
    src = Field.from_f64(g32, np.full(n * n, 100.0), dev)
    s = DiffusionSolver.new(g32, 0.01, None, dev)
    s.step_n_with_source(u, 50, src)
    assert u.max() > 0.0
    hh = 1.0 / (n - 1)
    t = np.arange(n) * hh
    X, Y = np.meshgrid(t, t)
    sin = (np.sin(np.pi * X) * np.sin(np.pi * Y)).ravel()
    for scheme in (TimeScheme.Rk2, TimeScheme.Rk4):
        u = Field.from_f64(g32, sin, dev)
        s = DiffusionSolver.build(g32, 0.01, None, Boundaries.zero_dirichlet(), scheme, dev)
        s.step_n(u, 200)
        nrm = u.norm_l2()
        assert np.isfinite(nrm) and 0.0 < nrm < np.linalg.norm(sin) and s.scheme() == scheme


@pytest.mark.parametrize("scheme", ["Euler", "Rk2", "Rk4"])
def test_graph_replay_equals_eager_steps(dev, scheme):
    """The recorded-and-replayed step (solver.rs:259-325 on CUDA graphs) is the same sequence of
    kernels as the eager step: bitwise equal after 25 steps."""
    from fluxion_b200 import Boundaries, Field
    from fluxion_b200.steppers import DiffusionSolver, TimeScheme
    g, h, bc, data, _ = _setup(64, dev)
    ue, ug = Field.from_f64(g, data, dev), Field.from_f64(g, data, dev)
    se = DiffusionSolver.build(g, 0.01, None, Boundaries.zero_dirichlet(), TimeScheme[scheme], dev)
    sg = DiffusionSolver.build(g, 0.01, None, Boundaries.zero_dirichlet(), TimeScheme[scheme], dev)
    sg.enable_graph()
    se.step_n(ue, 25)
    sg.step_n(ug, 10)
    sg.step_n(ug, 15)
    assert sg.steps_done() == se.steps_done() == 25
    assert np.array_equal(ug.to_vec_f64(), ue.to_vec_f64())
