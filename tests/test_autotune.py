"""Autotuner: the grid search keeps the fastest configuration and caches it per workload key."""
import json

import pytest

from master_thesis_b200 import autotune


def test_search_picks_fastest_and_caches(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    cost = {(1, 4): 3.0, (1, 8): 1.0, (2, 4): 2.0, (2, 8): 5.0}
    calls = []
    monkeypatch.setattr(autotune, "_time", lambda fn, reps: (fn(), cost[calls[-1]])[1])

    def run(cfg):
        calls.append((cfg["wave_size"], cfg["refill"]))
    best = autotune._search("k", dict(wave_size=[1, 2], refill=[4, 8]), run, 1, False)
    assert best == dict(wave_size=1, refill=8)
    db = json.loads((tmp_path / "tune.json").read_text())
    assert db["k"]["best"] == best and len(db["k"]["tried"]) == 4
    n = len(calls)
    assert autotune._search("k", dict(wave_size=[1, 2], refill=[4, 8]), run, 1, False) == best
    assert len(calls) == n  # served from the cache
    autotune._search("k", dict(wave_size=[1, 2], refill=[4, 8]), run, 1, True)
    assert len(calls) == 2 * n  # forced re-tune


@pytest.mark.gpu
def test_tune_render_on_gpu(tmp_path, monkeypatch):
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    sd, cam = scenes.random_scene(3, 2000)
    sc = swr.Scene(sd)
    c = swr.make_camera(cam["position"], cam["angle"], 64, 48, fov_deg=40)
    best = autotune.tune_render(sc, c, 64, 48, 4, 4, mode=swr.MODE_PHYSICAL,
                                grid=dict(wave_size=[1 << 12, 1 << 14], refill=[8]))
    assert best["wave_size"] in (1 << 12, 1 << 14) and best["refill"] == 8
    img = sc.render(c, 64, 48, 4, 4, mode=swr.MODE_PHYSICAL, **best)
    assert float(img.max()) > 0


@pytest.mark.gpu
def test_tune_per_lane_kernels_on_gpu(tmp_path, monkeypatch):
    """The bidirectional tracer and the RayTrace frame: the tuned launch shape renders the same
    image as the library's defaults."""
    import numpy as np
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import rt, scenes
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    s = scenes.cornell(2, str(tmp_path))
    sc = swr.Scene(swr.load_scene(s["scene"], s["basepath"]))
    cam = swr.load_camera(s["camera"], 48, 32)
    b = autotune.tune_bdpt(sc, cam, 48, 32, 4, 5, 5, 5, grid=dict(shade_batch=[1, 20 | (16 << 8)], refill=[4]))
    assert b["shade_batch"] in (1, 20 | (16 << 8))
    img = sc.render_bdpt(cam, 48, 32, 4, 5, 5, 5, seed=3, **b)
    ref = sc.render_bdpt(cam, 48, 32, 4, 5, 5, 5, seed=3)
    assert torch.equal(img, ref)
    r = autotune.tune_rt(sc, cam, 48, 32, 3, 5, grid=dict(shade_batch=[4, 16], refill=[4], blocks_per_sm=[0, 6]))
    a = rt.render(sc, cam, 48, 32, 3, 5, want_rgb=False, **r)[1]
    d = rt.render(sc, cam, 48, 32, 3, 5, want_rgb=False)[1]
    assert torch.equal(a, d) and int(a.max()) > 0
    db = json.loads((tmp_path / "tune.json").read_text())
    assert any(k.startswith("bdpt|") for k in db) and any(k.startswith("rt|") for k in db)


def test_grids_name_the_tunable_knobs():
    assert set(autotune.BUILD_GRID) == {"width", "max_leaf"} and 4 in autotune.BUILD_GRID["width"]
    assert set(autotune.RENDER_GRID) == {"wave_size", "refill", "block_size", "trace_blocks"}
    assert len(autotune.RENDER_GRID["block_size"]) > 1 and len(autotune.RENDER_GRID["trace_blocks"]) > 1


@pytest.mark.gpu
def test_tune_build_on_gpu(tmp_path, monkeypatch):
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    sd, cam = scenes.random_scene(4, 3000)
    c = swr.make_camera(cam["position"], cam["angle"], 64, 48, fov_deg=40)
    best = autotune.tune_build(sd, c, 64, 48, 4, 4, mode=swr.MODE_PHYSICAL)
    assert best["width"] in (4, 8) and best["max_leaf"] in (2, 3)
    db = json.loads((tmp_path / "tune.json").read_text())
    (entry,) = [v for k, v in db.items() if k.startswith("build|")]
    assert len(entry["tried"]) == 4 and entry["best"] == best
    # the chosen tree renders the same image as the default one (same closest hits)
    a = swr.Scene(sd, **best).render(c, 64, 48, 4, 4, mode=swr.MODE_PHYSICAL)
    b = swr.Scene(sd).render(c, 64, 48, 4, 4, mode=swr.MODE_PHYSICAL)
    assert torch.equal(a, b)


@pytest.mark.gpu
def test_tune_batch_build_on_gpu(tmp_path, monkeypatch):
    """The batch's tree options (BVH width, leaf size) are tuned on the batch itself and cached;
    the chosen trees render the same batch images as the default ones."""
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    monkeypatch.setattr(autotune, "CACHE", str(tmp_path / "tune.json"))
    datas, jobs = [], []
    for k, (n, side, spp) in enumerate([(2000, 32, 4), (6000, 48, 2), (800, 24, 8)]):
        sd, cam = scenes.random_scene(40 + k, n)
        datas.append(sd)
        jobs.append(dict(cam=swr.make_camera(cam["position"], cam["angle"], side, side, fov_deg=40), width=side,
                         height=side, spp=spp, depth=4, seed=k, mode=swr.MODE_PHYSICAL))
    best = autotune.tune_batch_build(datas, jobs)
    assert best["width"] in (4, 8) and best["max_leaf"] in (2, 3)
    db = json.loads((tmp_path / "tune.json").read_text())
    (entry,) = [v for k, v in db.items() if k.startswith("batchbuild|")]
    assert len(entry["tried"]) == 4 and entry["best"] == best
    imgs = []
    for opts in (best, {}):
        b = swr.Batch()
        scs = [swr.Scene(sd, **opts) for sd in datas]
        outs = [torch.empty((j["height"], j["width"], 3), dtype=torch.float32, device="cuda") for j in jobs]
        b.render([dict(j, scene=sc, out=o) for j, sc, o in zip(jobs, scs, outs)])
        torch.cuda.synchronize()
        imgs.append([o.cpu() for o in outs])
        b.close()
        for sc in scs:
            sc.close()
    for x, y in zip(*imgs):
        assert torch.equal(x, y)
