"""Multi-rank host logic of the independent-units sharding, run as two gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from master_thesis_b200 import sharding


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 2), (8, 4), (5, 8), (1000, 3)])
def test_shard_covers_every_unit_once(n, world):
    seen = []
    sizes = []
    for r in range(world):
        lo, hi = sharding.shard(n, r, world)
        seen += list(range(lo, hi))
        sizes.append(hi - lo)
    assert seen == list(range(n))
    assert max(sizes) - min(sizes) <= 1


def test_shard_rejects_bad_rank():
    with pytest.raises(ValueError):
        sharding.shard(4, 2, 2)


def test_reductions_without_process_group():
    assert sharding.max_over_ranks([1.0, 2.0]) == [1.0, 2.0]
    assert sharding.sum_over_ranks([3.0]) == [3.0]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        jobs = ["image%d" % k for k in range(5)]
        mine = sharding.owned(jobs, rank, world)
        mx = sharding.max_over_ranks([10.0 * (rank + 1), -rank])
        sm = sharding.sum_over_ranks([len(mine), 1])
        q.put((rank, mine, mx, sm))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=10) for _ in range(world))
    assert res[0][1] + res[1][1] == ["image%d" % k for k in range(5)]
    for _, _, mx, sm in res:
        assert mx == [20.0, 0.0]
        assert sm == [5.0, 2.0]
