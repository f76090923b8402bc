"""Raw field dump (crates/io/src/raw.rs:9-77): a little-endian header rows:u64, cols:u64,
dx:f64, dy:f64, then the rows * cols values as f64, row-major -- byte for byte the reference's
format, so files move between the two implementations."""
from __future__ import annotations

import os
import struct
from typing import Tuple, Union

import numpy as np

from .core import Grid

_HEADER = struct.Struct("<QQdd")


def write_raw_array(path: Union[str, os.PathLike], grid: Grid, data: np.ndarray) -> None:
    """Write `data` (rows * cols values) on `grid` in the raw format."""
    data = np.ascontiguousarray(data, dtype="<f8").ravel()
    if data.size != grid.rows * grid.cols:
        raise ValueError(f"expected {grid.rows * grid.cols} values, got {data.size}")
    with open(path, "wb") as f:
        f.write(_HEADER.pack(grid.rows, grid.cols, grid.dx, grid.dy))
        f.write(data.tobytes())


def read_raw_array(path: Union[str, os.PathLike]) -> Tuple[Grid, np.ndarray]:
    """Read a raw file into its grid and values; a short file is an error, as in the reference
    (read_exact)."""
    with open(path, "rb") as f:
        head = f.read(_HEADER.size)
        if len(head) != _HEADER.size:
            raise EOFError("raw file shorter than its header")
        rows, cols, dx, dy = _HEADER.unpack(head)
        grid = Grid.new(rows, cols, dx, dy)
        n = rows * cols
        body = f.read(8 * n)
        if len(body) != 8 * n:
            raise EOFError(f"raw file holds {len(body) // 8} of {n} values")
    return grid, np.frombuffer(body, dtype="<f8").astype(np.float64)


def write_raw(path: Union[str, os.PathLike], field) -> None:
    """raw.rs:9-31: write a field (its values read back as f64)."""
    write_raw_array(path, field.grid(), field.to_vec_f64())


def read_raw(path: Union[str, os.PathLike], device=None):
    """raw.rs:33-77: read a raw file into an F64 field on `device`."""
    from .field import Field
    grid, data = read_raw_array(path)
    return Field.from_f64(grid, data, device)


# Checkpoint of the learned smoother's parameters: an 8-byte magic, the parameter count as a
# little-endian u64, then the FP32 master parameters in the library's order (W1, b1, W2, b2, W3, b3).
_LSM_MAGIC = b"FXLSM001"


def write_smoother_params(path: Union[str, os.PathLike], params: np.ndarray) -> None:
    p = np.ascontiguousarray(params, dtype="<f4").ravel()
    with open(path, "wb") as f:
        f.write(_LSM_MAGIC)
        f.write(struct.pack("<Q", p.size))
        f.write(p.tobytes())


def read_smoother_params(path: Union[str, os.PathLike]) -> np.ndarray:
    with open(path, "rb") as f:
        if f.read(8) != _LSM_MAGIC:
            raise ValueError("not a learned-smoother checkpoint")
        head = f.read(8)
        if len(head) != 8:
            raise EOFError("checkpoint shorter than its header")
        (n,) = struct.unpack("<Q", head)
        body = f.read(4 * n)
        if len(body) != 4 * n:
            raise EOFError(f"checkpoint holds {len(body) // 4} of {n} parameters")
    return np.frombuffer(body, dtype="<f4").astype(np.float32)
