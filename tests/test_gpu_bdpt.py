"""GPU bidirectional path tracer (swr_render_bdpt through the C ABI) against the reference's own
BidirectionalPathTracer samples (golden fixtures, Philox shim) and against the oracle."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from helpers import GOLDEN_CASES, golden, golden_camera, golden_scene
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL = 1e-4  # double transcendentals: CUDA's against glibc's


def _close(a, b):
    return np.all(np.abs(a - b) <= RTOL * np.maximum(np.abs(b), 1e-6) + 1e-7)


def _render(sc, cam, W, H, spp, vj, lj, md, seed, refill=0, shade_batch=0, chunk=0):
    samples = torch.empty((W * H, spp, 4), dtype=torch.float32, device="cuda")
    img = sc.render_bdpt(cam, W, H, spp, vj, lj, md, seed=seed, samples=samples, refill=refill,
                         shade_batch=shade_batch, chunk=chunk)
    torch.cuda.synchronize()
    return img.cpu().numpy().reshape(-1, 3), samples.cpu().numpy()


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_bdpt_matches_reference_golden(name):
    g = golden(name)
    W, H, spp, vj, lj, md, seed = [int(x) for x in g["bdpt_params"]]
    sc = swr.Scene(golden_scene(g))
    img, ps = _render(sc, golden_camera(g), W, H, spp, vj, lj, md, seed)
    mine = (ps[..., :3].astype(np.float64) * (2.0 * np.pi)).astype(np.float32)
    ref = g["bdpt_per_sample"][..., :3]
    assert _close(mine, ref)
    # pixel: the reference sums the contributions in sample order and scales by 2 pi / spp
    assert _close(img, ref.astype(np.float64).sum(1).astype(np.float32) / spp)
    assert (np.abs(ref).sum(-1) > 0).mean() > 0.05


@pytest.mark.parametrize("refill,shade_batch,chunk", [(0, 0, 0), (1, 1, 0), (32, 1, 0), (4, 16, 0),
                                                     (2, 32 | (1 << 8), 0), (0, 0, 100), (8, 8 | (24 << 8), 7)])
def test_gpu_bdpt_matches_oracle_on_terrain(tmp_path, refill, shade_batch, chunk):
    """Launch shapes and chunkings (chunk: samples per chunk of the vertex tables, rounded down
    to whole pixels; 100 and 7 give many chunks) all give the oracle's result."""
    s = scenes.terrain(3, str(tmp_path), cells=64, tile=16, spheres=6, sphere_subdiv=2, lights=3)
    sd = swr.load_scene(s["scene"], s["basepath"])
    W, H, spp, vj, lj, md, seed = 40, 28, 3, 6, 4, 7, 5
    cam = swr.load_camera(s["camera"], W, H)
    img, ps = _render(swr.Scene(sd), cam, W, H, spp, vj, lj, md, seed, refill, shade_batch, chunk)
    vi, pi, org = swr.camera_arrays(cam)
    ops, opp = O.render_bdpt(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, spp, vj, lj, md, seed)
    assert _close(ps[..., :3], ops[..., :3])
    assert _close(img, opp)
    assert np.abs(opp).max() > 0


def test_gpu_bdpt_rejects_bad_requests():
    g = golden("ref_cornell_box_with_blocks")
    sd = golden_scene(g)
    sc = swr.Scene(sd)
    cam = golden_camera(g)
    for args in [(8, 8, 1, 17, 5, 5), (8, 8, 1, 5, 17, 5), (8, 8, 1, 5, 5, 0), (8, 8, 1, 0, 5, 5)]:
        with pytest.raises(swr.SwrError):
            sc.render_bdpt(cam, *args)
    dark = swr.SceneData(sd.vpos, sd.vnrm, sd.tri, sd.tri_obj, sd.obj_first_vertex, sd.materials.copy(),
                         tri_rank=sd.tri_rank)
    dark.materials["light_source"] = 0
    with pytest.raises(swr.SwrError) as e:
        swr.Scene(dark).render_bdpt(cam, 8, 8, 1, 5, 5, 5)
    assert "light source" in str(e.value)
