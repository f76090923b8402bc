"""Lanes: several contexts on one GPU, each with its own stream, driven from host threads.
Independent convection-diffusion solves run side by side on four lanes and give, bit for bit and
in the same number of iterations, the solutions the same problems give one after another on a
single lane; pool buffers start zeroed after reuse, and are ready on a stream the context
switches to after creating them."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _solve(dev, n, seed):
    from fluxion_b200 import (BiCgStabSolver, ConvDiffMultigrid, ConvDiffOperator, DType, Field,
                              Grid)
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    N, h = n + 2, 1.0 / (n + 1)
    g = Grid.square(N, h)
    vx, vy = stream_velocity(n, seed)
    f = poisson_uniform_rhs(n, seed + 1)
    VX, VY, b = Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev), Field.from_f64(g, f, dev)
    x = Field.zeros(g, DType.F64, dev)
    op = ConvDiffOperator(g, VX, VY, -1e-2, sigma=0.0, coeff=1.0)
    mg = ConvDiffMultigrid(op, 2, 2, 0.8, 15, 200)
    st = BiCgStabSolver(g, dev, 1e-10 * float(np.linalg.norm(f)), 200).solve_op(x, b, op, mg)
    assert st.converged()
    return st.iterations, x.to_vec_f64()


PROBLEMS = [(63, 11), (255, 13), (127, 15), (511, 17), (255, 19), (63, 21), (127, 23), (511, 25)]


def test_concurrent_lanes_match_sequential_solves():
    import torch
    from fluxion_b200 import Device
    seq = [_solve(Device.Cuda(0), n, s) for n, s in PROBLEMS]
    out = [None] * len(PROBLEMS)
    errors = []

    def work(lane):
        try:
            dev = Device.Cuda(0, lane=lane)
            assert dev.backend() is not Device.Cuda(0).backend()
            for i in range(lane - 1, len(PROBLEMS), 4):
                out[i] = _solve(dev, *PROBLEMS[i])
        except Exception as e:  # re-raised below
            errors.append(e)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(1, 5)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    torch.cuda.synchronize()
    assert not errors, errors
    for (it_s, xs), (it_c, xc) in zip(seq, out):
        assert it_s == it_c
        assert np.array_equal(xs, xc)


def test_pool_buffers_are_zeroed_and_follow_a_stream_switch():
    import torch
    from fluxion_b200 import DType, Device, Field, Grid
    dev = Device.Cuda(0, lane=7)
    assert str(dev) == "cuda:0/lane7" and Device.Cuda(0, 7) == dev and Device.Cuda(0) != dev
    g = Grid.square(1025, 1.0 / 1024)
    for _ in range(3):  # the pool hands the dropped block back out: it must be cleared each time
        u = Field.zeros(g, DType.F64, dev)
        assert not u.to_vec_f64().any()
        u.fill(3.5)
        del u
    data = np.random.default_rng(4).uniform(-1, 1, 1025 * 1025)
    v = Field.from_f64(g, data, dev)
    s = torch.cuda.Stream()
    be = dev.backend()
    be.set_stream(s.cuda_stream)
    try:
        w = Field.zeros(g, DType.F64, dev)
        assert np.array_equal(v.to_vec_f64(), data) and not w.to_vec_f64().any()
    finally:
        be.set_stream(None)
    assert np.array_equal(v.to_vec_f64(), data)
    out = torch.empty(data.size, dtype=torch.float64, pin_memory=True).numpy()
    v.copy_to_host(out)
    assert np.array_equal(out, data)
    out32 = np.empty(data.size, dtype=np.float32)
    v.copy_to_host(out32)
    assert np.array_equal(out32, data.astype(np.float32))
    from fluxion_b200 import DimensionMismatch
    with pytest.raises(DimensionMismatch):
        v.copy_to_host(np.empty(data.size - 1))


def test_async_copies_on_other_streams_ordered_by_events():
    """fx_write_f64_async / fx_copy_to_host_f64_async on two copy streams, ordered against the
    library's stream by events, move exactly the data (a round trip through an AXPY)."""
    import torch
    from fluxion_b200 import DType, Device, Field, Grid
    dev = Device.Cuda(0)
    be = dev.backend()
    g = Grid.square(1025, 1.0 / 1024)
    n = 1025 * 1025
    src = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    src[:] = np.random.default_rng(9).uniform(-1, 1, n)
    dst = torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    lib = torch.cuda.ExternalStream(be.stream()) if be.stream() else torch.cuda.current_stream()
    a, y = Field.zeros(g, DType.F64, dev), Field.zeros(g, DType.F64, dev)
    y.fill(1.0)
    be.synchronize()
    a.write_async(src, up.cuda_stream)
    e1 = torch.cuda.Event()
    e1.record(up)
    lib.wait_event(e1)
    y.axpy(2.0, a)  # y = 1 + 2 src on the library's stream
    e2 = torch.cuda.Event()
    e2.record(lib)
    down.wait_event(e2)
    y.copy_to_host_async(dst, down.cuda_stream)
    down.synchronize()
    assert np.array_equal(dst, 1.0 + 2.0 * src)
