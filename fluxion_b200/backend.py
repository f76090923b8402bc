"""``CudaBackend`` / ``CudaBuffer``: the reference's backend trait over the C ABI.

Mirrors ``fluxion_core::Backend`` (crates/core/src/backend.rs:43-406) and
``BackendBuffer`` (:13-36) method for method, plus the GPU backend's non-trait
fast paths (crates/backend-hip/src/backend.rs:463-668).  Every call goes through
``libfluxion_cuda.so``; status codes become the reference's ``CoreError``
variants.  One backend (context + stream) per device, created on first use like
the reference's ``OnceLock`` singletons (crates/runtime/src/storage.rs:118-138).
"""
from __future__ import annotations

import ctypes as C
import re
import threading
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _lib as L
from .core import (BackendError, Boundaries, CoreError, DimensionMismatch, DType, Grid, InvalidGrid,
                   InvalidStencil, Stencil)


class InvalidArgument(CoreError):
    def __init__(self, msg: str):
        super().__init__(f"invalid argument: {msg}")


class BackendUnavailable(CoreError):
    """crates/runtime/src/error.rs:11-12 (RuntimeError::BackendUnavailable)."""

    def __init__(self, msg: str):
        super().__init__(f"backend not available: {msg}")


def check(status: int) -> None:
    """Raise the CoreError variant matching a C-ABI status."""
    if status == L.FX_OK:
        return
    msg = L.last_error()
    if status == L.FX_ERR_DIMENSION_MISMATCH:
        m = re.search(r"expected (\d+), got (\d+)", msg)
        if m:
            raise DimensionMismatch(int(m.group(1)), int(m.group(2)))
        raise DimensionMismatch(-1, -1)
    if status == L.FX_ERR_INVALID_GRID:
        raise InvalidGrid(msg)
    if status == L.FX_ERR_INVALID_STENCIL:
        raise InvalidStencil(msg)
    if status == L.FX_ERR_INVALID_ARGUMENT:
        raise InvalidArgument(msg)
    if status == L.FX_ERR_NO_DEVICE:
        raise BackendUnavailable(msg)
    raise BackendError(msg)


# ------------------------------------------------------------------ marshalling

def grid_c(g: Grid) -> L.FxGrid:
    return L.FxGrid(g.rows, g.cols, g.dx, g.dy)


class StencilC:
    """Keeps the ctypes arrays of an ``fx_stencil`` alive for the duration of a call."""

    def __init__(self, s: Stencil):
        tr = s.as_triples()
        n = len(tr)
        self.dr = (C.c_int * n)(*[t[0] for t in tr])
        self.dc = (C.c_int * n)(*[t[1] for t in tr])
        self.w = (C.c_double * n)(*[t[2] for t in tr])
        self.s = L.FxStencil(n, self.dr, self.dc, self.w)

    @property
    def ptr(self):
        return C.byref(self.s)


def bcs_c(b: Optional[Boundaries]) -> L.FxBoundaries:
    out = L.FxBoundaries()
    b = b or Boundaries.zero_dirichlet()
    for i, side in enumerate(b.sides()):
        out.side[i].kind = int(side.kind)
        out.side[i].a = side.a
        out.side[i].b = side.b
        out.side[i].g = side.g
    return out


_NP = {DType.F64: np.float64, DType.F32: np.float32}


# ------------------------------------------------------------------ buffer

class CudaBuffer:
    """Device buffer owned by the library (HipBuffer's role, backend-hip/src/buffer.rs)."""

    __slots__ = ("backend", "handle", "_len", "_dtype", "__weakref__")

    def __init__(self, backend: "CudaBackend", handle: int, length: int, dtype: DType):
        self.backend = backend
        self.handle = handle
        self._len = length
        self._dtype = dtype

    def len(self) -> int:
        return self._len

    def __len__(self) -> int:
        return self._len

    def is_empty(self) -> bool:
        return self._len == 0

    def dtype(self) -> DType:
        return self._dtype

    def device_ptr(self) -> int:
        return L.lib().fx_buf_device_ptr(self.handle) or 0

    def copy_to_host_f64(self, dst: np.ndarray) -> None:
        """BackendBuffer::copy_to_host_f64; a length mismatch raises (the reference panics)."""
        if dst.dtype != np.float64 or not dst.flags.c_contiguous:
            raise InvalidArgument("destination must be a contiguous float64 array")
        if dst.size != self._len:
            raise AssertionError("destination length mismatch")
        check(L.lib().fx_copy_to_host_f64(self.backend.ctx, self.handle,
                                          dst.ctypes.data_as(C.POINTER(C.c_double)), dst.size))

    def copy_to_host_f32(self, dst: np.ndarray) -> None:
        if dst.dtype != np.float32 or not dst.flags.c_contiguous:
            raise InvalidArgument("destination must be a contiguous float32 array")
        if dst.size != self._len:
            raise AssertionError("destination length mismatch")
        check(L.lib().fx_copy_to_host_f32(self.backend.ctx, self.handle,
                                          dst.ctypes.data_as(C.POINTER(C.c_float)), dst.size))

    def to_numpy(self) -> np.ndarray:
        out = np.empty(self._len, dtype=_NP[self._dtype])
        if self._dtype == DType.F64:
            self.copy_to_host_f64(out)
        else:
            self.copy_to_host_f32(out)
        return out

    def write(self, data: np.ndarray) -> None:
        """Host -> this buffer, converting to the buffer's dtype."""
        if data.dtype == np.float64:
            a = np.ascontiguousarray(data)
            check(L.lib().fx_write_f64(self.backend.ctx, self.handle,
                                       a.ctypes.data_as(C.POINTER(C.c_double)), a.size))
        else:
            a = np.ascontiguousarray(data, dtype=np.float32)
            check(L.lib().fx_write_f32(self.backend.ctx, self.handle,
                                       a.ctypes.data_as(C.POINTER(C.c_float)), a.size))

    def write_async(self, data: np.ndarray, stream: int = 0) -> None:
        """Enqueue the copy of a contiguous float64 host array (page-locked for a true DMA) into this
        F64 buffer on `stream` (a cudaStream_t handle; 0 = the backend's stream) without waiting
        (fx_write_f64_async).  The caller orders it against the work that reads it with events."""
        if data.dtype != np.float64 or not data.flags.c_contiguous:
            raise InvalidArgument("write_async takes a contiguous float64 array")
        check(L.lib().fx_write_f64_async(self.backend.ctx, self.handle,
                                         data.ctypes.data_as(C.POINTER(C.c_double)), data.size, stream or None))

    def copy_to_host_async(self, out: np.ndarray, stream: int = 0) -> None:
        """Enqueue the copy of this F64 buffer into a contiguous float64 host array on `stream`
        without waiting (fx_copy_to_host_f64_async)."""
        if out.dtype != np.float64 or not out.flags.c_contiguous:
            raise InvalidArgument("copy_to_host_async takes a contiguous float64 array")
        check(L.lib().fx_copy_to_host_f64_async(self.backend.ctx, self.handle,
                                                out.ctypes.data_as(C.POINTER(C.c_double)), out.size,
                                                stream or None))

    def free(self) -> None:
        if self.handle:
            L.lib().fx_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __repr__(self):
        return f"CudaBuffer(len={self._len}, dtype={self._dtype.name})"


# ------------------------------------------------------------------ backend

class CudaGraph:
    """A recorded and instantiated sequence of this backend's operations (HipGraph,
    backend-hip/src/graph.rs:14-108): `launch` replays it on the backend's stream; the graph is
    destroyed with the object, as HipGraph is on Drop."""

    def __init__(self, backend: "CudaBackend", handle: int):
        self.backend = backend
        self.h = handle

    def launch(self) -> None:
        check(L.lib().fx_graph_launch(self.backend.ctx, self.h))

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_graph_destroy(self.h)
                self.h = None
        except Exception:
            pass


class CudaBackend:
    """The B200 backend: one CUDA context and stream per device."""

    _instances: Dict[tuple, "CudaBackend"] = {}
    _lock = threading.Lock()

    def __init__(self, ordinal: int = 0, lane: int = 0):
        lib = L.lib()
        h = C.c_void_p()
        check(lib.fx_ctx_create(int(ordinal), C.byref(h)))
        self.ctx = h.value
        self.ordinal = ordinal
        self.lane = lane

    @classmethod
    def get(cls, ordinal: int = 0, lane: int = 0) -> "CudaBackend":
        """The context of (device, lane): one per pair, created on first use, each with its own
        non-blocking stream."""
        with cls._lock:
            b = cls._instances.get((ordinal, lane))
            if b is None:
                b = cls(ordinal, lane)
                cls._instances[(ordinal, lane)] = b
            return b

    @staticmethod
    def device_count() -> int:
        n = C.c_int(0)
        st = L.lib().fx_device_count(C.byref(n))
        return n.value if st == L.FX_OK else 0

    def name(self) -> str:
        return L.lib().fx_backend_name().decode()

    def synchronize(self) -> None:
        check(L.lib().fx_ctx_synchronize(self.ctx))

    def launch_count(self) -> int:
        return int(L.lib().fx_ctx_launch_count(self.ctx))

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        check(L.lib().fx_ctx_set_stream(self.ctx, stream_ptr or None))

    def set_pdl(self, enabled: bool) -> None:
        """Programmatic dependent launch for this context's kernels (on by default)."""
        check(L.lib().fx_ctx_set_pdl(self.ctx, 1 if enabled else 0))

    def stream(self) -> int:
        return L.lib().fx_ctx_get_stream(self.ctx) or 0

    # -------------------------------------------------------------- graphs (HipGraph, graph.rs)

    def graph_begin(self) -> None:
        """Start recording this backend's stream (HipGraph::begin_capture, graph.rs:35-46)."""
        check(L.lib().fx_graph_begin(self.ctx))

    def graph_end(self) -> "CudaGraph":
        """Stop recording and instantiate (HipGraph::end_capture, graph.rs:48-70)."""
        h = C.c_void_p()
        check(L.lib().fx_graph_end(self.ctx, C.byref(h)))
        return CudaGraph(self, h.value)

    # -------------------------------------------------------------- memory

    def allocate(self, length: int, dtype: DType = DType.F64) -> CudaBuffer:
        h = C.c_void_p()
        check(L.lib().fx_alloc(self.ctx, int(length), int(dtype), C.byref(h)))
        return CudaBuffer(self, h.value, int(length), DType(dtype))

    def upload_f64(self, data) -> CudaBuffer:
        a = np.ascontiguousarray(data, dtype=np.float64).ravel()
        h = C.c_void_p()
        check(L.lib().fx_upload_f64(self.ctx, a.ctypes.data_as(C.POINTER(C.c_double)), a.size, C.byref(h)))
        return CudaBuffer(self, h.value, a.size, DType.F64)

    def upload_f32(self, data) -> CudaBuffer:
        a = np.ascontiguousarray(data, dtype=np.float32).ravel()
        h = C.c_void_p()
        check(L.lib().fx_upload_f32(self.ctx, a.ctypes.data_as(C.POINTER(C.c_float)), a.size, C.byref(h)))
        return CudaBuffer(self, h.value, a.size, DType.F32)

    def wrap(self, device_ptr: int, length: int, dtype: DType) -> CudaBuffer:
        """Non-owning view of existing device memory (e.g. a torch tensor's storage)."""
        h = C.c_void_p()
        check(L.lib().fx_wrap(self.ctx, C.c_void_p(device_ptr), int(length), int(dtype), C.byref(h)))
        return CudaBuffer(self, h.value, int(length), DType(dtype))

    # -------------------------------------------------------------- trait ops

    def apply_stencil(self, inp, out, grid: Grid, stencil: Stencil, boundaries: Boundaries):
        s = StencilC(stencil)
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_apply_stencil(self.ctx, inp.handle, out.handle, C.byref(g), s.ptr, C.byref(b)))

    def apply_stencil_var(self, inp, out, coeff, grid, stencil, boundaries):
        s = StencilC(stencil)
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_apply_stencil_var(self.ctx, inp.handle, out.handle, coeff.handle, C.byref(g), s.ptr,
                                           C.byref(b)))

    def stencil_axpy(self, alpha, x, y, grid, stencil, boundaries):
        s = StencilC(stencil)
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_stencil_axpy(self.ctx, float(alpha), x.handle, y.handle, C.byref(g), s.ptr, C.byref(b)))

    def copy(self, src, dst):
        check(L.lib().fx_copy(self.ctx, src.handle, dst.handle))

    def fill(self, buf, value):
        check(L.lib().fx_fill(self.ctx, buf.handle, float(value)))

    def axpy(self, alpha, x, y):
        check(L.lib().fx_axpy(self.ctx, float(alpha), x.handle, y.handle))

    def scale(self, buf, alpha):
        check(L.lib().fx_scale(self.ctx, buf.handle, float(alpha)))

    def _scalar(self, fn, *args) -> float:
        out = C.c_double()
        check(fn(self.ctx, *args, C.byref(out)))
        return out.value

    def norm_l2(self, buf) -> float:
        return self._scalar(L.lib().fx_norm_l2, buf.handle)

    def reduce_sum(self, buf) -> float:
        return self._scalar(L.lib().fx_reduce_sum, buf.handle)

    def reduce_max(self, buf) -> float:
        return self._scalar(L.lib().fx_reduce_max, buf.handle)

    def reduce_min(self, buf) -> float:
        return self._scalar(L.lib().fx_reduce_min, buf.handle)

    def dot(self, x, y) -> float:
        return self._scalar(L.lib().fx_dot, x.handle, y.handle)

    def dot2(self, a, b, c, d) -> Tuple[float, float]:
        ab, cd = C.c_double(), C.c_double()
        check(L.lib().fx_dot2(self.ctx, a.handle, b.handle, c.handle, d.handle, C.byref(ab), C.byref(cd)))
        return ab.value, cd.value

    def restrict(self, fine, coarse, fine_grid: Grid, coarse_grid: Grid):
        fg, cg = grid_c(fine_grid), grid_c(coarse_grid)
        check(L.lib().fx_restrict(self.ctx, fine.handle, coarse.handle, C.byref(fg), C.byref(cg)))

    def prolong(self, coarse, fine, coarse_grid: Grid, fine_grid: Grid):
        fg, cg = grid_c(fine_grid), grid_c(coarse_grid)
        check(L.lib().fx_prolong(self.ctx, coarse.handle, fine.handle, C.byref(cg), C.byref(fg)))

    def weighted_jacobi(self, x, b, omega, grid, stencil, boundaries):
        s = StencilC(stencil)
        g, bc = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_weighted_jacobi(self.ctx, x.handle, b.handle, float(omega), C.byref(g), s.ptr,
                                         C.byref(bc)))

    def pointwise_mult(self, x, y, z):
        check(L.lib().fx_pointwise_mult(self.ctx, x.handle, y.handle, z.handle))

    def pointwise_div(self, x, y, z):
        check(L.lib().fx_pointwise_div(self.ctx, x.handle, y.handle, z.handle))

    def pointwise_max(self, x, y, z):
        check(L.lib().fx_pointwise_max(self.ctx, x.handle, y.handle, z.handle))

    def pointwise_min(self, x, y, z):
        check(L.lib().fx_pointwise_min(self.ctx, x.handle, y.handle, z.handle))

    def waxpy(self, alpha, x, beta, y, w):
        check(L.lib().fx_waxpy(self.ctx, float(alpha), x.handle, float(beta), y.handle, w.handle))

    def aypx(self, alpha, x, y):
        check(L.lib().fx_aypx(self.ctx, float(alpha), x.handle, y.handle))

    def reciprocal(self, buf):
        check(L.lib().fx_reciprocal(self.ctx, buf.handle))

    def abs_val(self, buf):
        check(L.lib().fx_abs_val(self.ctx, buf.handle))

    def apply_conv_diff(self, u, out, kappa, vx, vy, grid, boundaries):
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_apply_conv_diff(self.ctx, u.handle, out.handle, kappa.handle, vx.handle, vy.handle,
                                         C.byref(g), C.byref(b)))

    def conv_diff_axpy(self, alpha, u, out, kappa, vx, vy, grid, boundaries):
        g, b = grid_c(grid), bcs_c(boundaries)
        check(L.lib().fx_conv_diff_axpy(self.ctx, float(alpha), u.handle, out.handle, kappa.handle, vx.handle,
                                        vy.handle, C.byref(g), C.byref(b)))

    # -------------------------------------------------------------- non-trait fast paths

    def zero_boundaries(self, buf, rows: int, cols: int):
        check(L.lib().fx_zero_boundaries(self.ctx, buf.handle, int(rows), int(cols)))

    def pipelined_cg_fused(self, alpha, beta, z, t, p, x, r, w, q):
        check(L.lib().fx_pcg_fused_update(self.ctx, float(alpha), float(beta), z.handle, t.handle, p.handle,
                                          x.handle, r.handle, w.handle, q.handle))

    def pipelined_cg_fused_dot2(self, alpha, beta, z, t, p, x, r, w, q) -> Tuple[float, float]:
        rr, rw = C.c_double(), C.c_double()
        check(L.lib().fx_pcg_fused_update_dot2(self.ctx, float(alpha), float(beta), z.handle, t.handle,
                                               p.handle, x.handle, r.handle, w.handle, q.handle,
                                               C.byref(rr), C.byref(rw)))
        return rr.value, rw.value

    # -------------------------------------------------------------- vertex multigrid primitives

    @staticmethod
    def _a5(a5: Sequence[float]):
        return (C.c_double * 5)(*[float(v) for v in a5])

    def jacobi_sweep(self, x_in, x_out, b, omega, rows, cols, a5):
        check(L.lib().fx_jacobi_sweep(self.ctx, x_in.handle, x_out.handle, b.handle, float(omega), int(rows),
                                      int(cols), self._a5(a5)))

    def residual5(self, x, b, r, rows, cols, a5):
        check(L.lib().fx_residual5(self.ctx, x.handle, b.handle, r.handle, int(rows), int(cols), self._a5(a5)))

    def restrict_fw(self, fine, coarse, fine_dims, coarse_dims):
        check(L.lib().fx_restrict_fw(self.ctx, fine.handle, coarse.handle, int(fine_dims[0]), int(fine_dims[1]),
                                     int(coarse_dims[0]), int(coarse_dims[1])))

    def prolong_bilinear(self, coarse, fine, coarse_dims, fine_dims):
        check(L.lib().fx_prolong_bilinear(self.ctx, coarse.handle, fine.handle, int(coarse_dims[0]),
                                          int(coarse_dims[1]), int(fine_dims[0]), int(fine_dims[1])))

    def __repr__(self):
        return f"CudaBackend(cuda:{self.ordinal})"
