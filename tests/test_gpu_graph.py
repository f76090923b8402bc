"""Graph capture and replay (HipGraph, crates/backend-hip/src/graph.rs) through the C ABI."""
import numpy as np
import pytest

from fluxion_b200 import Boundaries, DType, Grid, Stencil

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def be():
    from fluxion_b200 import CudaBackend
    return CudaBackend.get(0)


def test_graph_capture_and_replay(be):
    # crates/backend-hip/tests/graph.rs:8-38
    buf = be.allocate(256, DType.F64)
    be.graph_begin()
    be.fill(buf, 10.0)
    be.scale(buf, 0.5)
    graph = be.graph_end()
    be.fill(buf, 0.0)
    graph.launch()
    be.synchronize()
    assert np.all(np.abs(buf.to_numpy().astype(np.float64) - 5.0) < 1e-12)


def test_graph_replay_multiple_times(be):
    # crates/backend-hip/tests/graph.rs:40-72
    buf = be.allocate(1024, DType.F64)
    be.fill(buf, 1.0)
    be.graph_begin()
    be.scale(buf, 2.0)
    graph = be.graph_end()
    for _ in range(10):
        graph.launch()
    be.synchronize()
    assert abs(buf.to_numpy().astype(np.float64)[0] - 1024.0) < 1e-8


@pytest.mark.parametrize("dtype", [DType.F64, DType.F32])
def test_graph_replays_stencil_sequence_bitwise(be, dtype):
    """A captured stencil-AXPY / AXPY / scale step replayed three times gives exactly what running
    the step three times does."""
    n = 257
    g = Grid.square(n, 1.0 / (n - 1))
    st = Stencil.laplacian_2d_5pt(g.dx, g.dy)
    bc = Boundaries.zero_dirichlet()
    rng = np.random.default_rng(3)
    x0 = rng.uniform(-1, 1, n * n)
    up = be.upload_f64 if dtype == DType.F64 else be.upload_f32

    def step(x, y):
        be.stencil_axpy(1e-5, x, y, g, st, bc)
        be.axpy(0.25, y, x)
        be.scale(y, 0.5)

    xa, ya = up(x0), up(x0[::-1].copy())
    for _ in range(3):
        step(xa, ya)
    xb, yb = up(x0), up(x0[::-1].copy())
    be.graph_begin()
    step(xb, yb)
    graph = be.graph_end()
    for _ in range(3):
        graph.launch()
    be.synchronize()
    assert np.array_equal(xa.to_numpy().astype(np.float64), xb.to_numpy().astype(np.float64))
    assert np.array_equal(ya.to_numpy().astype(np.float64), yb.to_numpy().astype(np.float64))


def test_host_value_op_fails_capture_and_context_recovers(be):
    """A reduction returns a host value, so it cannot be recorded: it fails, ending the capture
    reports the failure, and the context keeps working afterwards."""
    from fluxion_b200.backend import BackendUnavailable
    a = be.upload_f64(np.arange(100.0))
    be.graph_begin()
    be.scale(a, 2.0)
    with pytest.raises(Exception):
        be.dot(a, a)
    with pytest.raises(Exception):
        be.graph_end()
    be.fill(a, 3.0)
    assert abs(be.dot(a, a) - 900.0) < 1e-12


def test_stream_switch_refused_while_capturing(be):
    """Switching the context's stream in the middle of a capture is refused (the old stream cannot
    be waited for, and the capture must end on the stream it began on); the capture itself is
    unharmed and replays correctly."""
    import torch
    from fluxion_b200.backend import InvalidArgument
    buf = be.allocate(512, DType.F64)
    s = torch.cuda.Stream()
    be.graph_begin()
    be.fill(buf, 4.0)
    with pytest.raises(InvalidArgument):
        be.set_stream(s.cuda_stream)
    be.scale(buf, 0.25)
    graph = be.graph_end()
    be.fill(buf, 0.0)
    graph.launch()
    be.synchronize()
    assert np.all(buf.to_numpy().astype(np.float64) == 1.0)
    be.set_stream(s.cuda_stream)  # outside a capture the switch is allowed
    be.set_stream(None)


def test_buffer_freed_during_capture_stays_owned_by_the_graph(be):
    """A pool buffer freed while its operations are being recorded is still addressed by the graph:
    its memory must not return to the pool (and reach a new buffer) before the graph is destroyed."""
    n = 1 << 16
    y = be.allocate(n, DType.F64)
    t = be.allocate(n, DType.F64)
    be.graph_begin()
    be.fill(t, 1.0)
    be.axpy(2.0, t, y)
    t.free()
    graph = be.graph_end()
    others = [be.allocate(n, DType.F64) for _ in range(4)]  # would reuse t's block if it were free
    for o in others:
        be.fill(o, 7.0)
    for _ in range(3):
        graph.launch()
    be.synchronize()
    assert np.all(y.to_numpy().astype(np.float64) == 6.0)
    for o in others:
        assert np.all(o.to_numpy().astype(np.float64) == 7.0)
    del graph  # fx_graph_destroy: the held memory returns to the pool only now
