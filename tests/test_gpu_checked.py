"""The checked build (libfluxion_cuda_checked.so, FX_CHECKED): kernels that test every index they
compute against the extent of the array addressed and record, never trap on, an out-of-range one.

- The status word records exactly what a check saw (a test hook runs one check and makes no
  memory access, so nothing out of range is ever touched) and a read clears it.
- The small-grid parity suites (3 x 3 up to 257 x 259 grids, the fused and reference cycles, the
  solvers, the conv-diff cycle, the batch, the learned smoother, graphs, steppers) run again on
  the checked library in a child process, each test followed by a read of the status words
  (tests/conftest.py): every result still matches the oracle and no index was out of range.
- Determinism: the same solves run twice give the same bits."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SUITES = [
    "tests/test_gpu_ops.py",
    "tests/test_gpu_solvers.py",
    "tests/test_gpu_convdiff.py",
    "tests/test_gpu_batch.py",
    "tests/test_gpu_learned.py",
    "tests/test_gpu_flexible.py",
    "tests/test_gpu_graph.py",
    "tests/test_gpu_steppers.py",
    "tests/test_gpu_failures.py",
    "tests/test_gpu_checked.py::test_status_word_records_a_check",
]


def _status(be):
    from fluxion_b200 import _lib as L
    cnt, line, idx, ext = C.c_size_t(), C.c_int(), C.c_longlong(), C.c_longlong()
    name = C.create_string_buffer(256)
    assert L.lib().fx_checked_status(be.ctx, C.byref(cnt), name, 256, C.byref(line), C.byref(idx),
                                     C.byref(ext)) == 0
    return cnt.value, name.value.decode(), line.value, idx.value, ext.value


def test_status_word_records_a_check():
    from fluxion_b200 import CudaBackend
    from fluxion_b200 import _lib as L
    be = CudaBackend.get(0)
    checked = L.lib().fx_checked_build() == 1
    assert checked == (os.environ.get("FLUXION_CHECKED") == "1")
    assert _status(be)[0] == 0
    assert L.lib().fx_test_check_index(be.ctx, 3, 5) == 0  # in range: nothing recorded
    assert _status(be)[0] == 0
    assert L.lib().fx_test_check_index(be.ctx, 7, 5) == 0
    assert L.lib().fx_test_check_index(be.ctx, -1, 5) == 0  # the first event of the unit is kept
    cnt, name, line, idx, ext = _status(be)
    if checked:
        assert (cnt, name, idx, ext) == (1, "fx_context.cu", 7, 5) and line > 0
    else:
        assert cnt == 0
    assert _status(be)[0] == 0  # the read cleared the word


@pytest.mark.skipif(os.environ.get("FLUXION_CHECKED") == "1", reason="runs the suites on the checked library")
def test_small_grid_suites_on_the_checked_build():
    lib = os.path.join(ROOT, "fluxion_b200", "libfluxion_cuda_checked.so")
    assert os.path.exists(lib), "build it with fluxion_b200.build.build(checked=True)"
    env = dict(os.environ, FLUXION_CHECKED="1")
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-p", "no:cacheprovider", "-m", "gpu", *SUITES],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1200)
    tail = (r.stdout + r.stderr)[-3000:]
    assert r.returncode == 0, tail
    assert " passed" in r.stdout and "failed" not in r.stdout, tail


def test_solves_are_deterministic():
    """The MG-PCG solve, the conv-diff FGMRES solve and the batched BiCGSTAB, each run twice from
    the same inputs: the same iterations and the same bits."""
    from fluxion_b200 import (CgSolver, ConvDiffMultigrid, ConvDiffOperator, DType, Device, FgmresSolver, Field,
                              Grid, Multigrid)
    from fluxion_b200.batch import BatchSolver
    from fluxion_b200.workloads import poisson_problem, poisson_uniform_rhs, stream_velocity
    dev = Device.best()
    be = dev.backend()
    n = 255
    P = poisson_problem(n)
    f = poisson_uniform_rhs(n, seed=5)
    out = []
    for _ in range(2):
        x = Field.zeros(P.grid, DType.F64, dev)
        st = CgSolver(P.grid, dev, 1e-10 * np.linalg.norm(f), 100).solve_preconditioned(
            x, Field.from_f64(P.grid, f, dev), P.coeff, P.stencil, None, Multigrid.vertex(P.grid, None, dev))
        out.append((st.iterations, st.residual, x.to_vec_f64()))
    assert out[0][:2] == out[1][:2] and np.array_equal(out[0][2], out[1][2])

    N = n + 2
    g = Grid.square(N, 1.0 / (n + 1))
    vx, vy = stream_velocity(n, 6)
    VX, VY = Field.from_f64(g, vx, dev), Field.from_f64(g, vy, dev)  # the operator borrows them
    op = ConvDiffOperator(g, VX, VY, -1e-3, sigma=0.0, coeff=1.0)
    out = []
    for _ in range(2):
        x = Field.zeros(g, DType.F64, dev)
        st = FgmresSolver(g, dev, 30, 1e-10 * np.linalg.norm(f), 300).solve_op(x, Field.from_f64(g, f, dev), op,
                                                                             ConvDiffMultigrid(op))
        out.append((st.iterations, st.residual, x.to_vec_f64()))
    assert out[0][:2] == out[1][:2] and np.array_equal(out[0][2], out[1][2])

    sides = [65, 129, 33, 257]
    vxs, vys, fs = [], [], []
    for k, s in enumerate(sides):
        a, b = stream_velocity(s - 2, 30 + k)
        vxs.append(a)
        vys.append(b)
        fs.append(poisson_uniform_rhs(s - 2, 40 + k))
    BVX, BVY = be.upload_f64(np.concatenate(vxs)), be.upload_f64(np.concatenate(vys))  # borrowed by the batch
    B = BatchSolver(dev, sides, 1e-2, BVX, BVY)
    rhs = be.upload_f64(np.concatenate(fs))
    out = []
    for _ in range(2):
        x = be.allocate(B.offsets[-1], DType.F64)
        stats, _ = B.bicgstab(x, rhs, 1e-10, 200)
        out.append(([(s.iterations, s.residual) for s in stats], x.to_numpy()))
    assert out[0][0] == out[1][0] and np.array_equal(out[0][1], out[1][1])
