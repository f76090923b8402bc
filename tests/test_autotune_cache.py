"""The autotuner's JSON cache (fluxion_b200/autotune.py) on CPU: keys are canonical, a stored
choice survives a reload from the file, and the batch sample keeps the batch's mix of sizes."""
import json

from fluxion_b200.autotune import TuneCache, _sample


def test_cache_roundtrip(tmp_path):
    p = tmp_path / "tune.json"
    c = TuneCache(str(p))
    k1 = TuneCache.key(kind="batch_convdiff", nu=0.01, sample_sizes={"65": 2, "129": 1}, device="B200")
    k2 = TuneCache.key(device="B200", sample_sizes={"129": 1, "65": 2}, nu=0.01, kind="batch_convdiff")
    assert k1 == k2
    assert c.get(k1) is None
    c.put(k1, {"chunk": 2048, "sweeps": 2, "cycle_dtype": "f32", "ms": 1.5})
    again = TuneCache(str(p))
    assert again.get(k2) == {"chunk": 2048, "sweeps": 2, "cycle_dtype": "f32", "ms": 1.5}
    assert json.load(open(p))[k1]["chunk"] == 2048


def test_sample_keeps_the_size_mix():
    sides = [65] * 50 + [129] * 30 + [1025] * 4
    idx = _sample(sides, 12, seed=1)
    assert len(idx) == 12 and len(set(idx)) == 12
    got = sorted({sides[i] for i in idx})
    assert got == [65, 129, 1025]
    assert _sample(sides, 1000) == list(range(len(sides)))
