"""A field written with write_raw and read back with read_raw (crates/io/src/raw.rs) is the same
field, bit for bit, on the same grid."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_field_round_trip(tmp_path):
    from fluxion_b200 import Device, Field, Grid
    from fluxion_b200.io import read_raw, write_raw
    dev = Device.best()
    g = Grid.new(33, 65, 1.0 / 64, 1.0 / 32)
    data = np.random.default_rng(3).uniform(-1, 1, 33 * 65)
    f = Field.from_f64(g, data, dev)
    write_raw(tmp_path / "u.raw", f)
    h = read_raw(tmp_path / "u.raw", dev)
    assert h.grid() == g
    assert np.array_equal(h.to_vec_f64(), data)
