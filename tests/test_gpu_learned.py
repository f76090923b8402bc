"""The learned smoother on the GPU against its torch FP64 oracle (oracle/learned.py): one learned
step (tensor-core network), the training samples cut from plain V-cycle iterates, the loss and its
gradient (forward and backward kernels), the untrained network reproducing the Jacobi cycle bit
for bit, the device-side fallback to the plain cycle, and what training gains.

Tolerances: the network runs in BF16 with FP32 accumulation on the GPU and in FP64 with the same
BF16 roundings in the oracle, so a hidden activation can land one BF16 step apart where the two
sums straddle a rounding boundary.  The network output is compared within 1e-2 relative (L2),
the loss within 1e-4 and the gradient within 2e-3 relative (L2)."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import learned as OL
from tests.helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


def _cd(n, nu, dev, seed):
    from fluxion_b200 import ConvDiffOperator, Field, Grid
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    N, h = n + 2, 1.0 / (n + 1)
    g = Grid.square(N, h)
    vx, vy = stream_velocity(n, seed)
    f = poisson_uniform_rhs(n, seed + 1)
    op = ConvDiffOperator(g, Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev), -nu, sigma=0.0, coeff=1.0)
    oop = O.cd_op(N, N, h, h, vx, vy, kappa=None, kappa_s=-nu, sigma=0.0, coeff=1.0)
    return g, N, h, vx, vy, f, op, oop


def _random_params(lsm, seed, scale3=0.2):
    rng = np.random.default_rng(seed)
    p = lsm.params
    p[OL.NP - 145:OL.NP - 1] = rng.normal(0.0, scale3, 144)  # W3
    p[OL.NP - 1] = 0.01                                      # b3
    p[432:448] = rng.normal(0.0, 0.05, 16)                   # b1
    p[448 + 2304:448 + 2320] = rng.normal(0.0, 0.05, 16)     # b2
    lsm.params = p
    return lsm.params


def _q_grid(oop, x, f, vx, vy, nu, h, N):
    d = OL.cd_diag(vx, vy, nu, h, h).reshape(N, N)
    q = ((f - O.op_apply(oop, x)) * (1.0 / d.ravel())).reshape(N, N)
    q[0, :] = q[-1, :] = q[:, 0] = q[:, -1] = 0.0
    return q, d


def test_learned_step_matches_oracle(dev):
    from fluxion_b200 import DType, Field
    from fluxion_b200.learned import LearnedSmoother
    n, nu, omega = 93, 1e-2, 0.8
    g, N, h, vx, vy, f, op, oop = _cd(n, nu, dev, 11)
    lsm = LearnedSmoother(dev, seed=3)
    params = _random_params(lsm, 4)
    x0 = np.zeros((N, N))
    x0[1:-1, 1:-1] = np.random.default_rng(5).uniform(-1e-2, 1e-2, (n, n))
    x = Field.from_f64(g, x0.ravel(), dev)
    lsm.smooth(op, x, Field.from_f64(g, f, dev), omega, 1)
    q, d = _q_grid(oop, x0.ravel(), f, vx, vy, nu, h, N)
    want, c_ref, s = OL.smooth_step(params, x0, q, vx.reshape(N, N), vy.reshape(N, N), d, omega, h, h)
    got = x.to_vec_f64().reshape(N, N)
    c_gpu = (got - x0 - omega * q)[1:-1, 1:-1] / s
    c_o = c_ref[1:-1, 1:-1]
    assert np.all(got[0, :] == 0) and np.all(got[:, 0] == 0)  # the ring is not touched
    assert np.abs(c_o).max() > 1e-2  # the network output is not trivial
    assert rel_err(c_gpu.ravel(), c_o.ravel()) < 1e-2
    assert np.abs(c_gpu - c_o).max() < 3e-2 * np.abs(c_o).max()


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_untrained_learned_cycle_is_the_jacobi_cycle(dev, dtype):
    """A network as created (last layer zero) makes every learned step the weighted-Jacobi sweep, so
    the learned cycle equals the plain cycle bit for bit; the check passes and nothing falls back."""
    from fluxion_b200 import ConvDiffMultigrid, DType, Field
    from fluxion_b200.learned import LearnedSmoother
    g, N, h, vx, vy, f, op, oop = _cd(127, 1e-3, dev, 21)
    dt = DType.F32 if dtype == "f32" else DType.F64
    plain, learned = ConvDiffMultigrid(op, dtype=dt), ConvDiffMultigrid(op, dtype=dt)
    learned.set_learned(LearnedSmoother(dev, seed=1), min_points=1, fallback_ratio=10.0)
    r = Field.from_f64(g, f, dev)
    za, zb = Field.zeros(g, DType.F64, dev), Field.zeros(g, DType.F64, dev)
    plain.apply(za, r)
    learned.apply(zb, r)
    assert np.array_equal(za.to_vec_f64(), zb.to_vec_f64())
    assert learned.learned_stats() == (1, 0)


def test_fallback_recomputes_the_plain_cycle(dev):
    """With a trained-looking (random) network and a check no cycle can pass, every application falls
    back on the device and z is the plain cycle's, bit for bit."""
    from fluxion_b200 import ConvDiffMultigrid, DType, Field
    from fluxion_b200.learned import LearnedSmoother
    g, N, h, vx, vy, f, op, oop = _cd(127, 1e-3, dev, 23)
    lsm = LearnedSmoother(dev, seed=2)
    _random_params(lsm, 9)
    plain, learned = ConvDiffMultigrid(op), ConvDiffMultigrid(op)
    r = Field.from_f64(g, f, dev)
    za, zb, zc = (Field.zeros(g, DType.F64, dev) for _ in range(3))
    plain.apply(za, r)
    learned.set_learned(lsm, min_points=1, fallback_ratio=10.0)
    learned.apply(zc, r)  # the learned cycle itself (passes the loose check)
    assert not np.array_equal(za.to_vec_f64(), zc.to_vec_f64())
    learned.set_learned(lsm, min_points=1, fallback_ratio=1e-30)
    for _ in range(2):
        learned.apply(zb, r)
        assert np.array_equal(za.to_vec_f64(), zb.to_vec_f64())
    assert learned.learned_stats() == (3, 2)


def test_samples_match_oracle(dev):
    from fluxion_b200 import DType, Field
    from fluxion_b200.learned import SmootherSamples
    n, nu, omega = 63, 1e-3, 0.8
    g, N, h, vx, vy, f, op, oop = _cd(n, nu, dev, 31)
    rng = np.random.default_rng(32)
    x0 = np.zeros((N, N))
    e0 = np.zeros((N, N))
    x0[1:-1, 1:-1] = rng.uniform(-1, 1, (n, n))
    e0[1:-1, 1:-1] = rng.uniform(-1, 1, (n, n))
    origins = [(4, 4), (10, 20), (44, 44), (30, 6)]
    S = SmootherSamples(dev, 16)
    S.add_patches(op, Field.from_f64(g, x0.ravel(), dev), Field.from_f64(g, e0.ravel(), dev),
                  Field.from_f64(g, f, dev), omega, origins)
    assert len(S) == 4
    q, d = _q_grid(oop, x0.ravel(), f, vx, vy, nu, h, N)
    s = float(np.sqrt(np.sum(q[1:-1, 1:-1] ** 2) / (n * n)))
    for k, (y0, x0_) in enumerate(origins):
        inp, th, te, nh, ne = S.get(k)
        wi, wth, wte, wnh, wne = OL.extract(q, e0, vx.reshape(N, N), vy.reshape(N, N), d, s, omega, h, h, y0, x0_)
        # BF16 inputs: equal, or one BF16 step apart where FP64 rounding differs at a boundary
        assert np.all(np.abs(inp - wi) <= 2.0 ** -7 * np.abs(wi) + 1e-30)
        assert np.mean(inp == wi) > 0.99
        assert rel_err(th.ravel().astype(np.float64), wth.ravel()) < 1e-6
        assert rel_err(te.ravel().astype(np.float64), wte.ravel()) < 1e-6
        assert abs(nh - wnh) <= 1e-6 * wnh and abs(ne - wne) <= 1e-6 * wne


def test_loss_and_gradient_match_oracle(dev):
    from fluxion_b200.learned import LearnedSmoother, SmootherSamples
    g, N, h, vx, vy, f, op, oop = _cd(95, 1e-3, dev, 41)
    from fluxion_b200 import Field
    S = SmootherSamples(dev, 64)
    added = S.add_problem(op, Field.from_f64(g, f, dev), iterates=3, patches_per_iterate=8, seed=7)
    assert added == 24 == len(S)
    lsm = LearnedSmoother(dev, seed=5)
    params = _random_params(lsm, 6)
    idx = list(range(24))
    data = [S.get(i) for i in idx]
    for lam in (0.0, 1.0):
        loss, grad = lsm.loss_grad(S, idx, lam=lam)
        wl, wg = OL.loss_and_grad(params, *(np.stack([d[j] for d in data]) for j in range(3)),
                                  np.array([d[3] for d in data]), np.array([d[4] for d in data]), lam)
        assert abs(loss - wl) <= 1e-4 * wl
        assert rel_err(grad.astype(np.float64), wg) < 2e-3
        # every layer's gradient is live, and the same batch gives the same bits
        for lo, hi in ((0, 432), (448, 2752), (2768, 2912)):
            assert np.linalg.norm(wg[lo:hi]) > 0 and rel_err(grad[lo:hi].astype(np.float64), wg[lo:hi]) < 5e-3
        l2, g2 = lsm.loss_grad(S, idx, lam=lam)
        assert l2 == loss and np.array_equal(g2, grad)


def test_training_beats_the_jacobi_step_and_learned_fgmres_converges(dev):
    """Training on samples from plain V-cycles (95^2 and 127^2, nu = 1e-3 and 1e-2) lowers the loss of
    held-out samples (another problem) below the Jacobi step's (the untrained network's).  The
    trained smoother inside FGMRES(30) with the per-cycle fallback reaches the tolerance on the true
    residual; its iterations are reported beside the plain cycle's."""
    from fluxion_b200 import ConvDiffMultigrid, DType, FgmresSolver, Field
    from fluxion_b200.learned import LearnedSmoother, SmootherSamples
    S = SmootherSamples(dev, 4096)
    for k, (n, nu) in enumerate([(95, 1e-3), (127, 1e-3), (95, 1e-2), (127, 1e-2)]):
        g, N, h, vx, vy, f, op, oop = _cd(n, nu, dev, 100 + 10 * k)
        S.add_problem(op, Field.from_f64(g, f, dev), iterates=4, patches_per_iterate=64, seed=k)
    H = SmootherSamples(dev, 512)
    g, N, h, vx, vy, f, op, oop = _cd(127, 1e-3, dev, 999)
    H.add_problem(op, Field.from_f64(g, f, dev), iterates=4, patches_per_iterate=64, seed=99)
    lsm = LearnedSmoother(dev, seed=11)
    held = list(range(len(H)))
    jacobi_loss, _ = lsm.loss_grad(H, held, want_grad=False)
    hist = lsm.train(S, epochs=30, batch=128, lr=2e-3, seed=3)
    trained_loss, _ = lsm.loss_grad(H, held, want_grad=False)
    print(f"held-out loss: Jacobi step {jacobi_loss:.4f}, learned {trained_loss:.4f}; "
          f"training loss {hist[0]:.4f} -> {hist[-1]:.4f}")
    assert hist[-1] < hist[0]
    assert trained_loss < jacobi_loss
    tol = 1e-10 * np.linalg.norm(f)
    b = Field.from_f64(g, f, dev)
    its = {}
    for name in ("plain", "learned"):
        mg = ConvDiffMultigrid(op)
        if name == "learned":
            mg.set_learned(lsm, min_points=1024, fallback_ratio=0.9)
        x = Field.zeros(g, DType.F64, dev)
        st = FgmresSolver(g, dev, 30, tol, 300).solve_op(x, b, op, mg)
        assert st.converged(), (name, st)
        assert np.linalg.norm(O.op_apply(oop, x.to_vec_f64()) - f) < 1.01 * tol
        its[name] = (st.iterations, mg.learned_stats() if name == "learned" else None)
    print("FGMRES(30) iterations (plain, learned [applications, fallbacks]):", its)


def test_checkpoint_reload_gives_the_same_smoothing(dev, tmp_path):
    from fluxion_b200 import Field
    from fluxion_b200.learned import LearnedSmoother
    n, nu = 61, 1e-2
    g, N, h, vx, vy, f, op, oop = _cd(n, nu, dev, 17)
    a = LearnedSmoother(dev, seed=5)
    params = _random_params(a, 6)
    a.save(tmp_path / "lsm.bin")
    b = LearnedSmoother(dev, seed=99)
    b.load(tmp_path / "lsm.bin")
    assert np.array_equal(b.params, params)
    outs = []
    for m in (a, b):
        x = Field.from_f64(g, np.zeros(N * N), dev)
        m.smooth(op, x, Field.from_f64(g, f, dev), 0.8, 2)
        outs.append(x.to_vec_f64())
    assert np.array_equal(outs[0], outs[1])


def test_patience_switches_the_learned_cycle_off(dev):
    """With a check no learned cycle passes and a patience of 2, the first two applications fall
    back and the learned cycle is then off: every z is the plain cycle's, so the FGMRES solve is
    the plain one bit for bit, and only two applications were checked."""
    from fluxion_b200 import ConvDiffMultigrid, DType, FgmresSolver, Field
    from fluxion_b200.learned import LearnedSmoother
    g, N, h, vx, vy, f, op, oop = _cd(127, 1e-3, dev, 29)
    lsm = LearnedSmoother(dev, seed=4)
    _random_params(lsm, 10)
    tol = 1e-10 * np.linalg.norm(f)
    outs = []
    for patience in (None, 2):
        mg = ConvDiffMultigrid(op)
        if patience:
            mg.set_learned(lsm, min_points=1, fallback_ratio=1e-30)
            mg.set_learned_patience(patience)
        x = Field.zeros(g, DType.F64, dev)
        st = FgmresSolver(g, dev, 30, tol, 300).solve_op(x, Field.from_f64(g, f, dev), op, mg)
        outs.append((st.iterations, x.to_vec_f64()))
        if patience:
            assert st.converged()
            assert mg.learned_disabled()
            assert mg.learned_stats() == (2, 2)
            mg.set_learned_patience(patience)  # switches it back on
            assert not mg.learned_disabled()
    assert outs[0][0] == outs[1][0]
    assert np.array_equal(outs[0][1], outs[1][1])
