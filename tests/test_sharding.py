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


# One image and one gradient split over gloo ranks. Each rank's part comes from the oracle (the
# CPU restatement of the reference's path tracer) for its pixel tile or sample range, so this
# checks the host logic of the split (partition, scaling, collectives, assembly) on the CPU; the
# GPU tests check that the library's parts equal the oracle's.
W, H, SPP, DEPTH, SEED = 24, 16, 5, 5, 31


def _split_setup(root):
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    from oracle import oracle as O
    s = scenes.cornell(4, root)
    sd = swr.load_scene(s["scene"], s["basepath"])
    cam = swr.load_camera(s["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    return O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org)


def _split_rank_main(rank, world, port, q, root, spp):
    import datetime
    import numpy as np
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        osc, ocam = _split_setup(root)
        calls = []

        def part(pb, pc, sb, sc):
            calls.append((pb, pc, sb, sc))
            _, pp = O.render_reference(osc, ocam, W, H, spp, DEPTH, SEED, pb, pb + pc, threads=2,
                                       samples=(sb, sb + sc))
            return torch.from_numpy(pp)

        tiles = sharding.render_split(part, W, H, spp, rank, world, split="tiles").numpy()
        by_spp = sharding.render_split(part, W, H, spp, rank, world, split="spp").numpy()
        dl = np.random.default_rng(3).normal(size=(H * W, 3)).astype(np.float32)

        def adj(sb, sc):
            ga, ge = O.adjoint_physical64(osc, ocam, W, H, spp, DEPTH, SEED, dl, rr_depth=3, rr_q=0.8, threads=2,
                                          samples=(sb, sb + sc))
            return torch.from_numpy(ga), torch.from_numpy(ge)

        shapes = [(osc.v0.shape[0], 3), (osc.obj_box.shape[0], 3)]
        ga, ge = sharding.adjoint_split(adj, spp, rank, world, shapes, dtype=torch.float64)
        q.put((rank, calls, tiles, by_spp, ga.numpy(), ge.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,spp", [(2, SPP), (3, SPP), (3, 2)])
def test_image_and_gradient_split_over_gloo_ranks(tmp_path, world, spp):
    import numpy as np
    from oracle import oracle as O
    root = str(tmp_path)
    osc, ocam = _split_setup(root)
    _, whole = O.render_reference(osc, ocam, W, H, spp, DEPTH, SEED)
    dl = np.random.default_rng(3).normal(size=(H * W, 3)).astype(np.float32)
    ga1, ge1 = O.adjoint_physical64(osc, ocam, W, H, spp, DEPTH, SEED, dl, rr_depth=3, rr_q=0.8)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_split_rank_main, args=(r, world, port, q, root, spp)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(world)), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    whole = whole.reshape(H, W, 3)
    for rank, calls, tiles, by_spp, ga, ge in res:
        # every rank holds the whole image: tiles bit-identical, sample ranges to float rounding
        assert np.array_equal(tiles, whole)
        assert np.allclose(by_spp, whole, rtol=1e-5, atol=1e-7)
        assert np.allclose(ga, ga1, rtol=1e-9, atol=1e-12) and np.allclose(ge, ge1, rtol=1e-9, atol=1e-12)
        # each rank rendered only its own share (an empty sample share makes no call)
        tlo, thi = sharding.shard(W * H, rank, world)
        slo, shi = sharding.shard(spp, rank, world)
        want = [(tlo, thi - tlo, 0, spp)] + ([(0, W * H, slo, shi - slo)] if shi > slo else [])
        assert calls == want
    assert ga1.any() and whole.any()


def test_split_rejects_unknown_mode():
    with pytest.raises(ValueError):
        sharding.render_split(lambda *a: None, 2, 2, 1, 0, 1, split="rows")
