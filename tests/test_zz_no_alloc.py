"""fx_dot_f64_noalloc: the dot product for callers that cannot let the library allocate.

Some callers own all device memory themselves (an application with its own pool that
accounts for every byte, or a loop that must never reach the allocator), so the library
must not cudaMalloc scratch on their behalf.  fx_dot_f64_noalloc keeps its reduction scratch
in a fixed static device array instead.  This test calls it through the C ABI on plain device
pointers and checks it against fx_dot (the context-scratch reduction) to the tolerance the
other reduction tests use, |a - b| <= 1e-13 * sum|x_i y_i|, on two calls in a row (the
scratch keeps the previous call's contents, so the second call checks that nothing leaks
from the first).  It lives in a file of its own that pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RED_TOL = 1e-13
MAX_N = 4096 * 2048


def _dp(buf):
    """A buffer's device address as the `const double *` the binding expects."""
    return C.cast(buf.device_ptr(), C.POINTER(C.c_double))


def _setup():
    from fluxion_b200 import CudaBackend
    from fluxion_b200 import _lib as L
    return CudaBackend.get(0), L.lib(), L


def test_noalloc_dot_matches_context_dot_twice():
    be, lib, L = _setup()
    rng = np.random.default_rng(2024)
    for n in (1, 4097, 1_000_003, MAX_N):
        x = rng.uniform(-1.0, 1.0, n)
        y = rng.uniform(-1.0, 1.0, n)
        X, Y = be.upload_f64(x), be.upload_f64(y)
        want = be.dot(X, Y)
        bound = RED_TOL * float(np.sum(np.abs(x * y)))
        got = []
        for _ in range(2):
            out = C.c_double(np.nan)
            st = lib.fx_dot_f64_noalloc(_dp(X), _dp(Y), n,
                                        C.byref(out), C.c_void_p(be.stream()))
            assert st == L.FX_OK, L.last_error()
            got.append(out.value)
        for g in got:
            assert abs(g - want) <= bound, (n, g, want)
        assert got[0] == got[1]  # deterministic across calls


def test_noalloc_dot_second_problem_after_first():
    # a different, smaller problem right after a larger one: no stale partials may leak in
    be, lib, L = _setup()
    rng = np.random.default_rng(7)
    for n in (MAX_N, 3):
        x, y = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
        X, Y = be.upload_f64(x), be.upload_f64(y)
        out = C.c_double()
        assert lib.fx_dot_f64_noalloc(_dp(X), _dp(Y), n, C.byref(out),
                                      None) == L.FX_OK
        assert abs(out.value - be.dot(X, Y)) <= RED_TOL * float(np.sum(np.abs(x * y)))


def test_noalloc_dot_rejects_sizes_beyond_the_limit():
    be, lib, L = _setup()
    X = be.upload_f64(np.ones(8))
    out = C.c_double()
    st = lib.fx_dot_f64_noalloc(_dp(X), _dp(X), MAX_N + 1, C.byref(out),
                                None)
    assert st == L.FX_ERR_INVALID_ARGUMENT
    assert "exceeds the static scratch limit" in L.last_error()
    assert lib.fx_dot_f64_noalloc(None, None, 0, C.byref(out), None) == L.FX_OK and out.value == 0.0
