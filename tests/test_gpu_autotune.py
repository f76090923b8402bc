"""The fused vertex cycle's layout knobs and their autotuner: every candidate layout (strip row
chunks per launch, largest level in the one-block tail) computes the same cycle bit for bit,
equal to the oracle's in F64, and the autotuner keeps the fastest candidate it timed."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CANDIDATES = [(p, t) for p in (50, 100, 200) for t in (9 * 1024, 2 * 1024)]


@pytest.fixture(scope="module")
def dev():
    from fluxion_b200 import Device
    return Device.best()


@pytest.mark.parametrize("n", [255, 1023])
def test_every_layout_gives_the_same_cycle(dev, n):
    from fluxion_b200 import DType, Field, Multigrid
    from fluxion_b200.workloads import poisson_modes_rhs, poisson_problem
    P = poisson_problem(n)
    N = n + 2
    f = poisson_modes_rhs(n, 7)
    r = Field.from_f64(P.grid, f, dev)
    omg = O.Multigrid(N, N, P.h, P.h, 2, 2, 0.8, mode=1, op_coeff=1.0, entries=P.stencil.as_triples())
    zo = np.zeros(N * N)
    omg.v_cycle(zo, f)
    for dt in (DType.F64, DType.F32):
        mg = Multigrid.vertex(P.grid, None, dev, dtype=dt)
        ref = None
        for pct, top in CANDIDATES:
            mg.set_tuning(pct, top)
            assert mg.get_tuning() == {"chunk_pct": pct, "tail_top_points": top}
            z = Field.zeros(P.grid, DType.F64, dev)
            mg.precondition(z, r)
            zv = z.to_vec_f64()
            if ref is None:
                ref = zv
                if dt == DType.F64:
                    assert np.array_equal(zv, zo)
            assert np.array_equal(zv, ref), (dt, pct, top)


def test_autotune_keeps_the_fastest_candidate(dev):
    from fluxion_b200 import DType, Field, Multigrid
    from fluxion_b200.workloads import poisson_modes_rhs, poisson_problem
    n = 1023
    P = poisson_problem(n)
    r = Field.from_f64(P.grid, poisson_modes_rhs(n, 7), dev)
    z = Field.zeros(P.grid, DType.F64, dev)
    mg = Multigrid.vertex(P.grid, None, dev, dtype=DType.F32)
    z0 = Field.zeros(P.grid, DType.F64, dev)
    mg.precondition(z0, r)
    res = mg.autotune(z, r, reps=3)
    assert len(res["candidates_ms"]) == len(CANDIDATES)
    k = int(np.argmin(res["candidates_ms"]))
    assert (res["chunk_pct"], res["tail_top_points"]) == CANDIDATES[k]
    assert res["ms"] == min(res["candidates_ms"]) > 0
    assert mg.get_tuning() == {"chunk_pct": res["chunk_pct"], "tail_top_points": res["tail_top_points"]}
    z1 = Field.zeros(P.grid, DType.F64, dev)
    mg.precondition(z1, r)
    assert np.array_equal(z1.to_vec_f64(), z0.to_vec_f64())


def test_batch_autotune_chooses_a_converging_candidate_and_caches_it(tmp_path):
    """The batch tuner times whole solves of a sample for each (chunk, sweeps, cycle dtype), keeps
    the fastest whose problems all converge, and a second call with the same key reads the JSON
    cache instead of timing."""
    import numpy as np
    from fluxion_b200 import Device
    from fluxion_b200.autotune import TuneCache, tune_batch
    from fluxion_b200.workloads import poisson_uniform_rhs, stream_velocity
    dev = Device.best()
    sides = [33, 65, 129, 65, 33, 129, 65, 257]
    vx, vy, f = [], [], []
    for k, s in enumerate(sides):
        a, b = stream_velocity(s - 2, 300 + k)
        vx.append(a)
        vy.append(b)
        f.append(poisson_uniform_rhs(s - 2, 400 + k))
    path = str(tmp_path / "tune.json")
    best = tune_batch(dev, sides, 1e-2, vx, vy, f, sample=6, chunks=(1024, 4096), sweeps=(1, 2),
                      dtypes=("f64", "f32"), cache=TuneCache(path))
    assert not best["cached"] and len(best["candidates"]) == 8
    assert any(c["ok"] for c in best["candidates"])
    chosen = [c for c in best["candidates"] if c["chunk"] == best["chunk"] and c["sweeps"] == best["sweeps"]
              and c["cycle_dtype"] == best["cycle_dtype"]][0]
    assert chosen["ok"] and chosen["ms"] == min(c["ms"] for c in best["candidates"] if c["ok"])
    again = tune_batch(dev, sides, 1e-2, vx, vy, f, sample=6, chunks=(1024, 4096), sweeps=(1, 2),
                       dtypes=("f64", "f32"), cache=TuneCache(path))
    assert again["cached"] and (again["chunk"], again["sweeps"], again["cycle_dtype"]) == \
        (best["chunk"], best["sweeps"], best["cycle_dtype"])


def test_vertex_mg_tuning_through_the_cache(tmp_path):
    import numpy as np
    from fluxion_b200 import DType, Device, Field, Multigrid
    from fluxion_b200.autotune import TuneCache, tune_vertex_mg
    from fluxion_b200.workloads import poisson_problem, poisson_uniform_rhs
    dev = Device.best()
    P = poisson_problem(1023)
    mg = Multigrid.vertex(P.grid, None, dev, dtype=DType.F32)
    r = Field.from_f64(P.grid, poisson_uniform_rhs(1023, 5), dev)
    z = Field.zeros(P.grid, DType.F64, dev)
    path = str(tmp_path / "mg.json")
    a = tune_vertex_mg(mg, z, r, cache=TuneCache(path), reps=3, dtype="f32", coarse_max=15, coarse_sweeps=200)
    mg2 = Multigrid.vertex(P.grid, None, dev, dtype=DType.F32)
    b = tune_vertex_mg(mg2, z, r, cache=TuneCache(path), reps=3, dtype="f32", coarse_max=15, coarse_sweeps=200)
    assert not a["cached"] and b["cached"]
    assert mg2.get_tuning() == {"chunk_pct": a["chunk_pct"], "tail_top_points": a["tail_top_points"]}
