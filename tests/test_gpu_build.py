"""Device BVH build (swr_build_opts.builder = SWR_BUILD_DEVICE): a different tree over the same
conservative boxes, so closest hits and renders must be bit-identical to the host-built scene's
and to the reference's golden hits."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from helpers import GOLDEN_CASES, golden, golden_scene, rays_uniform
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _hits(sc, ro, rd):
    h = sc.trace(torch.from_numpy(ro).cuda(), torch.from_numpy(rd).cuda())
    torch.cuda.synchronize()
    return h.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_device_build_golden_hits(name):
    g = golden(name)
    sc = swr.Scene(golden_scene(g), builder="device")
    h = _hits(sc, g["ray_o"], g["ray_d"])
    assert np.array_equal(h[:, 0], g["hit_id"])
    assert np.array_equal(h[:, 1], g["hit_obj"])
    assert np.array_equal(h[:, 2], g["hit_d2"].view(np.uint32))


@pytest.mark.parametrize("tris,radius,max_leaf", [(60000, 16, 3), (20000, 4, 1), (5000, 64, 2)])
def test_device_build_matches_host_build(tris, radius, max_leaf):
    sd, _ = scenes.random_scene(77 + tris, tris)
    host = swr.Scene(sd)
    dev = swr.Scene(sd, builder="device", radius=radius, max_leaf=max_leaf)
    st = dev.stats()
    assert st["triangles"] == sd.num_triangles and 1 <= st["nodes"] < sd.num_triangles
    ro, rd = rays_uniform(200000, sd.vpos.min(0) - 0.2, sd.vpos.max(0) + 0.2, seed=3)
    assert np.array_equal(_hits(host, ro, rd), _hits(dev, ro, rd))


def _tiny_scene(k, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-1, 1, (3 * k, 3)).astype(np.float32)
    nrm = np.tile(np.array([0, 0, 1], np.float32), (3 * k, 1))
    mats = np.zeros(1, swr.MAT_DTYPE)
    mats["color"] = 0.5
    mats["diffuse_t"] = 1.0
    mats["reflect_t"] = 1.0
    mats["transparent_t"] = 1.0
    mats["refraction_index"] = 1.0
    return swr.SceneData(pos, nrm, np.arange(3 * k).reshape(k, 3), np.zeros(k), [0, 3 * k], mats)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 7, 9, 25])
def test_device_build_tiny_scenes_vs_oracle(k):
    sd = _tiny_scene(k, 100 + k)
    sc = swr.Scene(sd, builder="device")
    assert sc.stats()["nodes"] >= 1
    ro, rd = rays_uniform(8192, sd.vpos.min(0) - 0.3, sd.vpos.max(0) + 0.3, seed=k)
    h = _hits(sc, ro, rd)
    otri, od2, _ = O.OracleScene.from_scene_data(sd).trace(ro, rd)
    assert np.array_equal(h[:, 0], otri)
    assert np.array_equal(h[:, 2], od2.view(np.uint32))
    assert (otri != 0xFFFFFFFF).any()


def test_device_build_render_identical(tmp_path):
    s = scenes.terrain(5, str(tmp_path), cells=128, tile=16, spheres=8, sphere_subdiv=3, lights=2)
    sd = swr.load_scene(s["scene"], s["basepath"])
    W, H = 96, 64
    cam = swr.load_camera(s["camera"], W, H)
    a = swr.Scene(sd).render(cam, W, H, 8, 6, seed=4)
    b = swr.Scene(sd, builder="device").render(cam, W, H, 8, 6, seed=4)
    torch.cuda.synchronize()
    assert torch.equal(a, b) and float(a.max()) > 0


def test_device_build_rejects_bad_options():
    g = golden("ref_white_room")
    with pytest.raises(swr.SwrError):
        swr.Scene(golden_scene(g), builder="device", radius=300)
    with pytest.raises(swr.SwrError):
        swr.Scene(golden_scene(g), builder="device", max_leaf=4)
