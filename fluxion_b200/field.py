"""``Device`` and ``Field``: the runtime layer of fluxion over the CUDA backend.

``Device`` follows crates/runtime/src/device.rs:3-37 (CUDA variant, probed by
``Device.best()``); ``Field`` follows crates/runtime/src/field.rs:15-1050, one
backend call per method.  There is no CPU or wgpu arm: a Field lives on a B200.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional, Tuple

import numpy as np

import ctypes as C

from . import _lib as L
from .backend import BackendUnavailable, CudaBackend, CudaBuffer, check
from .core import Boundaries, DimensionMismatch, DType, Grid, Stencil


class DeviceMismatch(Exception):
    """crates/runtime/src/error.rs:8-9."""

    def __init__(self, a, b):
        super().__init__(f"device mismatch: {a} vs {b}")


@dataclass(frozen=True)
class Device:
    """crates/runtime/src/device.rs:3-11 (only the CUDA variant exists here).

    ``lane`` selects one of several independent contexts on the same GPU, each with its own
    stream (new; the reference has one stream per device): work on different lanes may run
    concurrently, so independent problems can share the GPU from several host threads.  A field
    belongs to its lane; operations never mix lanes."""

    ordinal: int = 0
    lane: int = 0

    @staticmethod
    def Cuda(ordinal: int = 0, lane: int = 0) -> "Device":  # noqa: N802 - reference variant name
        return Device(int(ordinal), int(lane))

    @staticmethod
    def best() -> "Device":
        """device.rs:18-37 probes CUDA first; this build has no fallback device."""
        if CudaBackend.device_count() > 0:
            return Device(0)
        raise BackendUnavailable("no CUDA device")

    def backend(self) -> CudaBackend:
        return CudaBackend.get(self.ordinal, self.lane)

    def __str__(self):
        return f"cuda:{self.ordinal}" + (f"/lane{self.lane}" if self.lane else "")


class Field:
    """A scalar field on a structured grid, stored on the device (field.rs:15-18)."""

    __slots__ = ("storage", "_grid", "_device")

    def __init__(self, storage: CudaBuffer, grid: Grid, device: Device):
        self.storage = storage
        self._grid = grid
        self._device = device

    # ---------------------------------------------------------- constructors

    @staticmethod
    def zeros(grid: Grid, dtype: DType = DType.F64, device: Optional[Device] = None) -> "Field":
        device = device or Device.best()
        return Field(device.backend().allocate(grid.len(), dtype), grid, device)

    @staticmethod
    def from_f64(grid: Grid, data, device: Optional[Device] = None) -> "Field":
        device = device or Device.best()
        a = np.ascontiguousarray(data, dtype=np.float64).ravel()
        if a.size != grid.len():
            raise DimensionMismatch(grid.len(), a.size)
        return Field(device.backend().upload_f64(a), grid, device)

    @staticmethod
    def from_f32(grid: Grid, data, device: Optional[Device] = None) -> "Field":
        device = device or Device.best()
        a = np.ascontiguousarray(data, dtype=np.float32).ravel()
        if a.size != grid.len():
            raise DimensionMismatch(grid.len(), a.size)
        return Field(device.backend().upload_f32(a), grid, device)

    # ---------------------------------------------------------- accessors

    def grid(self) -> Grid:
        return self._grid

    def device(self) -> Device:
        return self._device

    def dtype(self) -> DType:
        return self.storage.dtype()

    def to_vec_f64(self) -> np.ndarray:
        out = np.empty(self.storage.len(), dtype=np.float64)
        self.storage.copy_to_host_f64(out)
        return out

    def copy_to_host(self, out: np.ndarray) -> None:
        """This field into an existing contiguous host array of its length (f64 or f32,
        converted on the device); with page-locked memory the copy is a direct DMA."""
        if out.size != self.storage.len() or not out.flags.c_contiguous:
            raise DimensionMismatch(self.storage.len(), out.size)
        if out.dtype == np.float64:
            self.storage.copy_to_host_f64(out)
        elif out.dtype == np.float32:
            self.storage.copy_to_host_f32(out)
        else:
            raise TypeError(f"host array must be float64 or float32, not {out.dtype}")

    def to_vec_f32(self) -> np.ndarray:
        out = np.empty(self.storage.len(), dtype=np.float32)
        self.storage.copy_to_host_f32(out)
        return out

    def write(self, data) -> None:
        self.storage.write(np.asarray(data))

    def write_async(self, data: np.ndarray, stream: int = 0) -> None:
        """Enqueue the copy of a contiguous float64 host array (page-locked for a true DMA) into
        this F64 field on `stream` (a cudaStream_t handle; 0 = the backend's stream) without
        waiting (fx_write_f64_async).  The caller orders it against the solves with events."""
        if data.dtype != np.float64 or not data.flags.c_contiguous:
            raise TypeError("write_async takes a contiguous float64 array")
        check(L.lib().fx_write_f64_async(self._b.ctx, self.storage.handle,
                                         data.ctypes.data_as(C.POINTER(C.c_double)), data.size, stream or None))

    def copy_to_host_async(self, out: np.ndarray, stream: int = 0) -> None:
        """Enqueue the copy of this F64 field into a contiguous float64 host array on `stream`
        without waiting (fx_copy_to_host_f64_async)."""
        if out.dtype != np.float64 or not out.flags.c_contiguous:
            raise TypeError("copy_to_host_async takes a contiguous float64 array")
        check(L.lib().fx_copy_to_host_f64_async(self._b.ctx, self.storage.handle,
                                                out.ctypes.data_as(C.POINTER(C.c_double)), out.size,
                                                stream or None))

    @property
    def _b(self) -> CudaBackend:
        return self._device.backend()

    def _same(self, other: "Field") -> None:
        if other._device != self._device:
            raise DeviceMismatch(other._device, self._device)

    # ---------------------------------------------------------- operations

    def copy_from(self, other: "Field") -> None:
        self._same(other)
        self._b.copy(other.storage, self.storage)

    def apply_stencil_into(self, stencil: Stencil, boundaries: Boundaries, output: "Field") -> None:
        self._same(output)
        self._b.apply_stencil(self.storage, output.storage, self._grid, stencil, boundaries)

    def apply_stencil_var_into(self, coeff: "Field", stencil: Stencil, boundaries: Boundaries,
                               output: "Field") -> None:
        self._same(output)
        self._same(coeff)
        self._b.apply_stencil_var(self.storage, output.storage, coeff.storage, self._grid, stencil, boundaries)

    def stencil_axpy(self, alpha: float, other: "Field", stencil: Stencil, boundaries: Boundaries) -> None:
        """self += alpha * stencil(other); boundary points of self untouched (field.rs:300-351)."""
        self._same(other)
        self._b.stencil_axpy(alpha, other.storage, self.storage, self._grid, stencil, boundaries)

    def fill(self, value: float) -> None:
        self._b.fill(self.storage, value)

    def zero_boundaries(self) -> None:
        self._b.zero_boundaries(self.storage, self._grid.rows, self._grid.cols)

    def scale(self, alpha: float) -> None:
        self._b.scale(self.storage, alpha)

    def axpy(self, alpha: float, other: "Field") -> None:
        self._same(other)
        self._b.axpy(alpha, other.storage, self.storage)

    def norm_l2(self) -> float:
        return self._b.norm_l2(self.storage)

    def sum(self) -> float:
        return self._b.reduce_sum(self.storage)

    def max(self) -> float:
        return self._b.reduce_max(self.storage)

    def min(self) -> float:
        return self._b.reduce_min(self.storage)

    def dot(self, other: "Field") -> float:
        self._same(other)
        return self._b.dot(self.storage, other.storage)

    def dot2(self, b: "Field", c: "Field", d: "Field") -> Tuple[float, float]:
        return self._b.dot2(self.storage, b.storage, c.storage, d.storage)

    def integral(self) -> float:
        return self.sum() * self._grid.dx * self._grid.dy

    @staticmethod
    def swap(a: "Field", b: "Field") -> None:
        a.storage, b.storage = b.storage, a.storage
        a._grid, b._grid = b._grid, a._grid

    def pointwise_mult(self, x: "Field", y: "Field") -> None:
        self._b.pointwise_mult(x.storage, y.storage, self.storage)

    def pointwise_div(self, x: "Field", y: "Field") -> None:
        self._b.pointwise_div(x.storage, y.storage, self.storage)

    def pointwise_max(self, x: "Field", y: "Field") -> None:
        self._b.pointwise_max(x.storage, y.storage, self.storage)

    def pointwise_min(self, x: "Field", y: "Field") -> None:
        self._b.pointwise_min(x.storage, y.storage, self.storage)

    def waxpy(self, alpha: float, x: "Field", beta: float, y: "Field") -> None:
        self._b.waxpy(alpha, x.storage, beta, y.storage, self.storage)

    def aypx(self, alpha: float, other: "Field") -> None:
        """self = other + alpha * self (field.rs:957-999)."""
        self._b.aypx(alpha, other.storage, self.storage)

    def reciprocal(self) -> None:
        self._b.reciprocal(self.storage)

    def abs_val(self) -> None:
        self._b.abs_val(self.storage)

    def apply_conv_diff_into(self, kappa: "Field", vx: "Field", vy: "Field", boundaries: Boundaries,
                             output: "Field") -> None:
        self._b.apply_conv_diff(self.storage, output.storage, kappa.storage, vx.storage, vy.storage,
                                self._grid, boundaries)

    def conv_diff_axpy(self, alpha: float, u: "Field", kappa: "Field", vx: "Field", vy: "Field",
                       boundaries: Boundaries) -> None:
        """self += alpha * (kappa Lap(u) + v . grad u)."""
        self._b.conv_diff_axpy(alpha, u.storage, self.storage, kappa.storage, vx.storage, vy.storage,
                               self._grid, boundaries)

    def __repr__(self):
        return f"Field({self._grid.rows}x{self._grid.cols}, {self.dtype().name}, {self._device})"
