"""Autotuner for the BVH shape and the wavefront's launch shape.

For a workload it times a small grid of the tunable knobs with CUDA events, keeps the fastest, and
caches the choice in a JSON file keyed by the workload's shape and the GPU name:
  - the tree (tune_build, tune_batch_build): children per wide node (BVH width 4 or 8; the node record keeps 8
    slots) and triangles per leaf, each candidate built and rendered;
  - the launch (tune_render, tune_batch): paths in flight (wave size), the idle-lane refill
    threshold of the traversal, the shading kernel's block size and the traversal's register
    budget (resident blocks per SM).

    bo = tune_build(scene_data, cam, width, height, spp, depth, mode=...)  # -> dict of Scene kwargs
    cfg = tune_render(scene, cam, width, height, spp, depth, mode=...)   # -> dict of render kwargs
    bo = tune_batch_build(scene_datas, jobs)                             # -> dict of Scene kwargs
    cfg = tune_batch(batch, jobs)                                        # -> dict of batch kwargs
    cfg = tune_bdpt(scene, cam, width, height, spp, vj, lj, md)          # -> dict of render_bdpt kwargs
    cfg = tune_rt(scene, cam, width, height, spp, vision_jumps)          # -> dict of rt.render kwargs

For the per-lane kernels (the bidirectional tracer, the RayTrace frame) the knobs are the number
of lanes of a warp that run their stage code together, the idle-lane refill threshold and the
register budget.
"""
import itertools
import json
import os
import time

import torch

CACHE = os.environ.get("SWR_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "swr_b200", "tune.json"))

BUILD_GRID = dict(width=[4, 8], max_leaf=[2, 3])
RENDER_GRID = dict(wave_size=[1 << 22, 1 << 23, 1 << 24, 1 << 25, 1 << 26, 1 << 27], refill=[4, 8, 16], block_size=[128, 256, 512],
                   trace_blocks=[0, 10])
BATCH_GRID = dict(wave_size=[1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25], refill=[4, 8, 16])
BDPT_GRID = dict(shade_batch=[12 | (16 << 8), 20 | (16 << 8), 24 | (16 << 8), 20 | (8 << 8), 20 | (24 << 8)],
                 refill=[4, 8], blocks_per_sm=[0])
RT_GRID = dict(shade_batch=[8, 12, 16, 20], refill=[2, 4], blocks_per_sm=[0, 6])


def _load():
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(db):
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    tmp = CACHE + ".tmp"
    with open(tmp, "w") as f:
        json.dump(db, f, indent=1, sort_keys=True)
    os.replace(tmp, CACHE)


def _time(fn, reps):
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _search(key, grid, run, reps, force):
    db = _load()
    if key in db and not force:
        return db[key]["best"]
    names = sorted(grid)
    results = []
    for values in itertools.product(*[grid[n] for n in names]):
        cfg = dict(zip(names, values))
        results.append((_time(lambda: run(cfg), reps), cfg))
    results.sort(key=lambda r: r[0])
    db[key] = {"best": results[0][1], "ms": results[0][0], "tried": [[ms, c] for ms, c in results],
               "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    _store(db)
    return results[0][1]


def tune_build(data, cam, width, height, spp, depth, mode=0, rr_depth=0, rr_survive=1.0, reps=2, force=False,
               grid=None, builder="host"):
    """Tree options for a scene (SceneData): each candidate of the grid is built and one image
    with the library's default launch shape is timed; returns the fastest as Scene kwargs."""
    from .api import Scene
    key = "build|%s|%s|tris=%d|objs=%d|px=%d|spp=%d|depth=%d|mode=%d" % (
        torch.cuda.get_device_name(), builder, data.num_triangles, data.num_objects, width * height, spp, depth,
        mode)
    out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
    built = {}

    def run(cfg):
        k = tuple(sorted(cfg.items()))
        if k not in built:
            for sc in built.values():
                sc.close()
            built.clear()
            built[k] = Scene(data, builder=builder, **cfg)
        built[k].render(cam, width, height, spp, depth, mode=mode, rr_depth=rr_depth, rr_survive=rr_survive,
                        out=out)
    try:
        return _search(key, grid or BUILD_GRID, run, reps, force)
    finally:
        for sc in built.values():
            sc.close()


def tune_render(scene, cam, width, height, spp, depth, mode=0, rr_depth=0, rr_survive=1.0, reps=2, force=False,
                grid=None):
    st = scene.stats()
    key = "render|%s|tris=%d|px=%d|spp=%d|depth=%d|mode=%d" % (torch.cuda.get_device_name(), st["triangles"],
                                                              width * height, spp, depth, mode)
    out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")

    def run(cfg):
        scene.render(cam, width, height, spp, depth, mode=mode, rr_depth=rr_depth, rr_survive=rr_survive, out=out,
                     **cfg)
    return _search(key, grid or RENDER_GRID, run, reps, force)


def tune_batch_build(datas, jobs, reps=1, force=False, grid=None, builder="host"):
    """Tree options for the scenes of a batch: datas[i] is the SceneData of jobs[i] (jobs as for
    Batch.render, without their "scene"). Each candidate of the grid builds every scene with the
    same options and times one batched render with the library's default launch shape; returns
    the fastest as Scene kwargs."""
    from .api import Batch, Scene
    tris = sum(d.num_triangles for d in datas)
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    key = "batchbuild|%s|%s|jobs=%d|tris=%d|samples=%d" % (torch.cuda.get_device_name(), builder, len(jobs), tris,
                                                          samples)
    outs = [torch.empty((j["height"], j["width"], 3), dtype=torch.float32, device="cuda") for j in jobs]
    batch = Batch()
    built = {}

    def release():
        for scs in built.values():
            for sc in scs:
                sc.close()
        built.clear()

    def run(cfg):
        k = tuple(sorted(cfg.items()))
        if k not in built:
            release()
            built[k] = [Scene(d, builder=builder, **cfg) for d in datas]
        batch.render([dict(j, scene=sc, out=o) for j, sc, o in zip(jobs, built[k], outs)])
    try:
        return _search(key, grid or BUILD_GRID, run, reps, force)
    finally:
        release()
        batch.close()


def tune_batch(batch, jobs, reps=1, force=False, grid=None):
    tris = sum(j["scene"].stats()["triangles"] for j in jobs)
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    key = "batch|%s|jobs=%d|tris=%d|samples=%d" % (torch.cuda.get_device_name(), len(jobs), tris, samples)
    outs = [torch.empty((j["height"], j["width"], 3), dtype=torch.float32, device="cuda") for j in jobs]
    jj = [dict(j, out=o) for j, o in zip(jobs, outs)]

    def run(cfg):
        batch.render(jj, **cfg)
    return _search(key, grid or BATCH_GRID, run, reps, force)


def tune_bdpt(scene, cam, width, height, spp, vision_jumps, light_jumps, max_depth, reps=2, force=False, grid=None):
    st = scene.stats()
    key = "bdpt|%s|tris=%d|px=%d|spp=%d|jumps=%d/%d/%d" % (torch.cuda.get_device_name(), st["triangles"],
                                                          width * height, spp, vision_jumps, light_jumps, max_depth)
    out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")

    def run(cfg):
        scene.render_bdpt(cam, width, height, spp, vision_jumps, light_jumps, max_depth, out=out, **cfg)
    return _search(key, grid or BDPT_GRID, run, reps, force)


def tune_rt(scene, cam, width, height, spp, vision_jumps, reps=2, force=False, grid=None):
    from . import rt
    st = scene.stats()
    key = "rt|%s|tris=%d|px=%d|spp=%d|jumps=%d" % (torch.cuda.get_device_name(), st["triangles"], width * height,
                                                   spp, vision_jumps)
    out = torch.empty((height, width, 4), dtype=torch.uint8, device="cuda")

    def run(cfg):
        rt.render(scene, cam, width, height, spp, vision_jumps, rgba=out, want_rgb=False, **cfg)
    return _search(key, grid or RT_GRID, run, reps, force)
