"""GPU closest-hit kernel (swr_trace_closest, through the C ABI) against the reference's golden
hits and against the oracle: hit triangle ids and squared distances must be bit-identical."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from helpers import GOLDEN_CASES, golden, golden_scene, rays_uniform
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _gpu_trace(sc, ro, rd):
    h = sc.trace(torch.from_numpy(ro).cuda(), torch.from_numpy(rd).cuda())
    torch.cuda.synchronize()
    h = h.cpu().numpy().view(np.uint32)
    return h[:, 0], h[:, 1], h[:, 2].view(np.float32), h[:, 3].view(np.float32)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_hits_match_reference_golden(name):
    g = golden(name)
    sd = golden_scene(g)
    sc = swr.Scene(sd)
    tri, obj, d2, t = _gpu_trace(sc, g["ray_o"], g["ray_d"])
    assert np.array_equal(tri, g["hit_id"])
    assert np.array_equal(obj, g["hit_obj"])
    assert np.array_equal(d2.view(np.uint32), g["hit_d2"].view(np.uint32))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_hits_match_oracle_random_rays(name):
    g = golden(name)
    sd = golden_scene(g)
    sc = swr.Scene(sd)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(200000, sd.vpos.min(0) - 0.3, sd.vpos.max(0) + 0.3, seed=5)
    tri, _, d2, t = _gpu_trace(sc, ro, rd)
    otri, od2, ot = osc.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))
    assert np.array_equal(t.view(np.uint32), ot.view(np.uint32))


def test_gpu_host_buffers_and_empty():
    g = golden("ref_cornell_box_with_ball")
    sc = swr.Scene(golden_scene(g))
    hits = sc.trace(g["ray_o"], g["ray_d"])  # numpy in, numpy out: staged through the device
    assert np.array_equal(hits[:, 0], g["hit_id"])
    empty = sc.trace(g["ray_o"][:0], g["ray_d"][:0])
    assert empty.shape == (0, 4)


def test_gpu_terrain_tiles_vs_oracle(tmp_path):
    """A small terrain scene (tiles of heightfield + icospheres + lights), seeded rays."""
    s = scenes.terrain(9, str(tmp_path), cells=64, tile=16, spheres=8, sphere_subdiv=2, lights=2)
    sd = swr.load_scene(s["scene"], s["basepath"])
    assert sd.num_triangles == s["triangles"] and sd.ranks_exact
    sc = swr.Scene(sd)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(50000, sd.vpos.min(0), sd.vpos.max(0), seed=21)
    tri, _, d2, _ = _gpu_trace(sc, ro, rd)
    otri, od2, _ = osc.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))


def test_gpu_trace_stats_counts():
    g = golden("ref_cornell_box_with_ball")
    sc = swr.Scene(golden_scene(g))
    ro = torch.from_numpy(g["ray_o"]).cuda()
    rd = torch.from_numpy(g["ray_d"]).cuda()
    counts = torch.zeros((ro.shape[0], 2), dtype=torch.int32, device="cuda")
    h = sc.trace(ro, rd, counts=counts)
    torch.cuda.synchronize()
    c = counts.cpu().numpy()
    assert np.array_equal(h.cpu().numpy().view(np.uint32)[:, 0], g["hit_id"])
    assert (c[:, 0] >= 1).all() and c[:, 1].mean() > 0


def test_gpu_terrain_microbench_rays_vs_oracle(tmp_path):
    """The default bench's closest-hit microbenchmark: the full terrain (2,424,840 triangles) and
    16M rays from scenes.uniform_rays; every 64th ray's hit (262,144 rays spread over the whole
    set) must be bit-identical to the oracle's."""
    s = scenes.terrain(2024, str(tmp_path), cells=1024, tile=16, spheres=64, sphere_subdiv=4, lights=4)
    sd = swr.load_scene(s["scene"], s["basepath"])
    assert sd.num_triangles == 2424840 and sd.ranks_exact
    sc = swr.Scene(sd)
    ro, rd = scenes.uniform_rays(1 << 24, sd.vpos.min(0), sd.vpos.max(0), seed=16)
    h = sc.trace(ro, rd)
    torch.cuda.synchronize()
    h = h[::64].cpu().numpy().view(np.uint32)
    osc = O.OracleScene.from_scene_data(sd)
    otri, od2, ot = osc.trace(ro[::64].cpu().numpy(), rd[::64].cpu().numpy())
    assert np.array_equal(h[:, 0], otri)
    assert np.array_equal(h[:, 2], od2.view(np.uint32))
    assert np.array_equal(h[:, 3], ot.view(np.uint32))
    assert 0.05 < float((otri != 0xFFFFFFFF).mean()) < 0.95


def test_gpu_ties_on_a_large_single_mesh(tmp_path):
    """Shared-edge and shared-vertex hits (exact ties in squared distance) on a 51,200-triangle
    single mesh with exact reference ranks: the GPU picks the same triangle as the oracle."""
    from helpers import grid_mesh_scene, rays_down_onto_grid_lines
    path, base = grid_mesh_scene(str(tmp_path))
    sd = swr.load_scene(path, base)
    assert sd.ranks_exact
    sc = swr.Scene(sd)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_down_onto_grid_lines(20000, 160, seed=8)
    tri, _, d2, _ = _gpu_trace(sc, ro, rd)
    otri, od2, _ = osc.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))
    ro2, rd2 = rays_uniform(20000, (-1.2, -0.5, -1.2), (1.2, 1.0, 1.2), seed=9)
    tri2, _, _, _ = _gpu_trace(sc, ro2, rd2)
    assert np.array_equal(tri2, osc.trace(ro2, rd2)[0])
