"""The learned smoother of the convection-diffusion multigrid (fx_lsm_*; new: the reference
smooths with weighted Jacobi only, crates/runtime/src/multigrid.rs:245-306).

A 3 -> 16 -> 16 -> 1 network of 3 x 3 convolutions (ReLU after the first two, BF16 weights and
activations, FP32 accumulation, 2913 parameters) corrects the weighted-Jacobi step: with
q = (b - A x) / diag(A) and s the RMS of q over the interior, one learned step is
x <- x + omega q + s N(q / s, vx / (dx diag), vy / (dy diag)).  Its network runs on the tensor
cores; it is trained on the GPU by the library's forward, backward and Adam kernels on samples
cut from plain V-cycle iterates (`SmootherSamples.add_problem`), with the loss
(||H e'||^2 + lam ||e'||^2) / (||H e||^2 + lam ||e||^2) of the error e' after the step, H = I - P R.  A `ConvDiffMultigrid` uses it
through `set_learned`, with a per-application residual check that falls back to the plain cycle.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L
from .backend import check
from .field import Device, Field

IN_SIDE = 25   # network input region of a sample (points per side)
PATCH = 16     # loss patch of a sample
# Weight of the whole error beside its high-frequency part in the loss.  0 by default: with a
# positive weight the network chases the smooth error, which a local correction cannot remove,
# and the trained cycles diverged (measured at 127^2 - 511^2, nu 1e-2 - 1e-4, weights 0.3 - 10).
DEFAULT_LAMBDA = 0.0


def param_count() -> int:
    n = C.c_size_t()
    check(L.lib().fx_lsm_param_count(C.byref(n)))
    return n.value


class SmootherSamples:
    """Training samples on the device (fx_lsm_data_*)."""

    def __init__(self, device: Device, capacity: int):
        self.device = device
        out = C.c_void_p()
        check(L.lib().fx_lsm_data_create(device.backend().ctx, int(capacity), C.byref(out)))
        self.h = out.value
        self.capacity = int(capacity)

    def __len__(self) -> int:
        n = C.c_size_t()
        check(L.lib().fx_lsm_data_size(self.h, C.byref(n)))
        return n.value

    def add_patches(self, op, x: Field, e: Field, b: Field, omega: float, origins: Sequence) -> None:
        """One sample per (row, col) origin of an iterate x with error e for op u = b."""
        o = np.ascontiguousarray(np.asarray(origins, dtype=np.int32).reshape(-1, 2))
        check(L.lib().fx_lsm_data_add_patches(self.h, op.h, x.storage.handle, e.storage.handle, b.storage.handle,
                                              float(omega), o.ctypes.data_as(C.POINTER(C.c_int)), o.shape[0]))

    def add_problem(self, op, b: Field, iterates: int, patches_per_iterate: int, omega: float = 0.8,
                    seed: int = 0) -> int:
        """Samples from the plain V-cycle on op u = b (u solved to 1e-12 first); returns the count."""
        n = C.c_size_t()
        check(L.lib().fx_lsm_data_add_problem(self.h, op.h, b.storage.handle, int(iterates), int(patches_per_iterate),
                                              float(omega), int(seed), C.byref(n)))
        return n.value

    def get(self, index: int):
        """(inputs [3, 25, 25], tH [16, 16], tE [16, 16], nH, nE) of one sample, float32 values."""
        inp = np.empty(3 * IN_SIDE * IN_SIDE, dtype=np.float32)
        tgt = np.empty(2 * PATCH * PATCH, dtype=np.float32)
        nrm = np.empty(2, dtype=np.float32)
        check(L.lib().fx_lsm_data_get(self.h, int(index), inp.ctypes.data_as(C.POINTER(C.c_float)),
                                      tgt.ctypes.data_as(C.POINTER(C.c_float)),
                                      nrm.ctypes.data_as(C.POINTER(C.c_float))))
        t = tgt.reshape(2, PATCH, PATCH)
        return inp.reshape(3, IN_SIDE, IN_SIDE), t[0], t[1], float(nrm[0]), float(nrm[1])

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_lsm_data_destroy(self.h)
                self.h = None
        except Exception:
            pass


class LearnedSmoother:
    """The network, its FP32 master parameters and its Adam state (fx_lsm_*)."""

    def __init__(self, device: Device, seed: int = 0):
        self.device = device
        out = C.c_void_p()
        check(L.lib().fx_lsm_create(device.backend().ctx, int(seed), C.byref(out)))
        self.h = out.value

    @property
    def params(self) -> np.ndarray:
        p = np.empty(param_count(), dtype=np.float32)
        check(L.lib().fx_lsm_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    @params.setter
    def params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(L.lib().fx_lsm_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def loss_grad(self, samples: SmootherSamples, indices: Sequence[int], want_grad: bool = True,
                  lam: float = DEFAULT_LAMBDA):
        """(mean loss with whole-error weight `lam`, its gradient or None) over the given samples."""
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.uint64))
        loss = C.c_double()
        g = np.empty(param_count(), dtype=np.float32) if want_grad else None
        check(L.lib().fx_lsm_loss_grad(self.h, samples.h, idx.ctypes.data_as(C.POINTER(C.c_size_t)), idx.size,
                                       float(lam), C.byref(loss),
                                       g.ctypes.data_as(C.POINTER(C.c_float)) if g is not None else None))
        return loss.value, g

    def train(self, samples: SmootherSamples, epochs: int, batch: int = 256, lr: float = 2e-3,
              seed: int = 0, lam: float = DEFAULT_LAMBDA) -> List[float]:
        """Adam over `epochs` shuffles; returns the mean sample loss of each epoch."""
        out = (C.c_double * max(1, int(epochs)))()
        check(L.lib().fx_lsm_train(self.h, samples.h, int(epochs), int(batch), float(lr), float(lam), int(seed),
                                   out))
        return [out[i] for i in range(int(epochs))]

    def save(self, path) -> None:
        """Write the FP32 master parameters to a checkpoint file (fluxion_b200.io format)."""
        from .io import write_smoother_params
        write_smoother_params(path, self.params)

    def load(self, path) -> None:
        """Read parameters from a checkpoint (the optimiser state restarts)."""
        from .io import read_smoother_params
        p = read_smoother_params(path)
        if p.size != param_count():
            raise ValueError(f"checkpoint holds {p.size} parameters, the network has {param_count()}")
        self.params = p

    def smooth(self, op, x: Field, b: Field, omega: float = 0.8, steps: int = 1) -> None:
        """`steps` learned smoothing steps on op x = b (x in place)."""
        check(L.lib().fx_lsm_smooth(self.h, op.h, x.storage.handle, b.storage.handle, float(omega), int(steps)))

    def __del__(self):
        try:
            if self.h:
                L.lib().fx_lsm_destroy(self.h)
                self.h = None
        except Exception:
            pass
