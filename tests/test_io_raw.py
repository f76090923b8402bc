"""The raw field format (crates/io/src/raw.rs:9-77): header rows:u64, cols:u64, dx:f64, dy:f64
little-endian, then row-major f64 values; round trips are bit for bit; short files and invalid
grids are errors."""
import struct

import numpy as np
import pytest

from fluxion_b200.core import Grid, InvalidGrid
from fluxion_b200.io import read_raw_array, write_raw_array


def test_layout_and_round_trip(tmp_path):
    g = Grid.new(3, 5, 0.25, 0.125)
    data = np.random.default_rng(1).uniform(-1, 1, 15)
    data[0] = -0.0
    data[1] = np.inf
    p = tmp_path / "f.raw"
    write_raw_array(p, g, data)
    raw = p.read_bytes()
    assert len(raw) == 32 + 8 * 15
    assert raw[:32] == struct.pack("<QQdd", 3, 5, 0.25, 0.125)
    assert raw[32:] == data.astype("<f8").tobytes()
    g2, d2 = read_raw_array(p)
    assert (g2.rows, g2.cols, g2.dx, g2.dy) == (3, 5, 0.25, 0.125)
    assert d2.tobytes() == data.tobytes()


def test_errors(tmp_path):
    g = Grid.new(4, 4, 0.1, 0.1)
    with pytest.raises(ValueError):
        write_raw_array(tmp_path / "a.raw", g, np.zeros(15))
    p = tmp_path / "short.raw"
    write_raw_array(p, g, np.zeros(16))
    p.write_bytes(p.read_bytes()[:-8])
    with pytest.raises(EOFError):
        read_raw_array(p)
    (tmp_path / "hdr.raw").write_bytes(b"\x00" * 10)
    with pytest.raises(EOFError):
        read_raw_array(tmp_path / "hdr.raw")
    bad = tmp_path / "bad.raw"
    bad.write_bytes(struct.pack("<QQdd", 0, 4, 0.1, 0.1))
    with pytest.raises(InvalidGrid):
        read_raw_array(bad)


def test_smoother_checkpoint_roundtrip(tmp_path):
    import numpy as np
    import pytest
    from fluxion_b200.io import read_smoother_params, write_smoother_params
    p = np.random.default_rng(1).normal(size=2913).astype(np.float32)
    path = tmp_path / "lsm.bin"
    write_smoother_params(path, p)
    assert path.stat().st_size == 16 + 4 * 2913
    assert np.array_equal(read_smoother_params(path), p)
    raw = path.read_bytes()
    (tmp_path / "bad.bin").write_bytes(b"XXXXXXXX" + raw[8:])
    with pytest.raises(ValueError):
        read_smoother_params(tmp_path / "bad.bin")
    (tmp_path / "short.bin").write_bytes(raw[:100])
    with pytest.raises(EOFError):
        read_smoother_params(tmp_path / "short.bin")
