"""The multi-rank split of the batched workload (fluxion_b200/batch.py), on CPU with gloo and two
ranks: the partition covers every problem exactly once with balanced loads, each rank computes
only its own problems, and one collective gives every rank all results in problem order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fluxion_b200.batch import gather_results, loads, partition_by_points


def _sizes(n=1024, seed=2024):
    ks = np.random.default_rng(seed).integers(6, 11, size=n)
    return [int(2 ** k + 1) ** 2 for k in ks]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_partition_covers_and_balances(world):
    pts = _sizes()
    parts = partition_by_points(pts, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(pts)))
    ld = loads(pts, parts)
    assert max(ld) - min(ld) <= max(pts)          # LPT bound
    assert max(ld) <= sum(pts) / world + max(pts)
    assert parts == partition_by_points(pts, world)  # deterministic


def test_partition_edge_cases():
    assert partition_by_points([], 2) == [[], []]
    assert partition_by_points([5], 3) == [[0], [], []]
    with pytest.raises(ValueError):
        partition_by_points([1, 2], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pts = _sizes(64, seed=7)
        mine = partition_by_points(pts, world)[rank]
        # each rank "solves" only its problems: a deterministic per-problem result
        local = {i: (i, rank, float(np.sqrt(pts[i]))) for i in mine}
        allres = gather_results(local, len(pts))
        q.put((rank, mine, allres))
    finally:
        dist.destroy_process_group()


def test_two_rank_split_and_gather():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    pts = _sizes(64, seed=7)
    parts = partition_by_points(pts, world)
    for rank, mine, allres in out:
        assert mine == parts[rank]
        assert [r[0] for r in allres] == list(range(64))
        for i, (idx, owner, val) in enumerate(allres):
            assert owner == (0 if i in parts[0] else 1) and val == float(np.sqrt(pts[i]))
    assert out[0][2] == out[1][2]
