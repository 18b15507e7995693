"""CPU build of the kernels' traversal and shading code (tests/native/twin.cpp) against the oracle
and the reference's golden outputs: checks the wide-BVH construction, the quantised traversal
with its pruning, and the shading arithmetic without a GPU."""
import numpy as np
import pytest

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from helpers import (GOLDEN_CASES, Twin, golden, golden_camera, golden_scene, ref_pixel_from_samples,
                     rays_uniform)
from oracle import oracle as O


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_twin_hits_match_reference_golden(name):
    g = golden(name)
    tw = Twin(golden_scene(g))
    tri, d2, _ = tw.trace(g["ray_o"], g["ray_d"])
    assert np.array_equal(tri, g["hit_id"])
    assert np.array_equal(d2.view(np.uint32), g["hit_d2"].view(np.uint32))


@pytest.mark.parametrize("name", GOLDEN_CASES)
@pytest.mark.parametrize("max_leaf,postpone", [(1, False), (3, False), (3, True)])
def test_twin_hits_match_oracle_random_rays(name, max_leaf, postpone):
    g = golden(name)
    sd = golden_scene(g)
    tw = Twin(sd, max_leaf=max_leaf)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(20000, sd.vpos.min(0) - 0.3, sd.vpos.max(0) + 0.3, seed=11)
    tri, d2, t = tw.trace(ro, rd, postpone=postpone)
    otri, od2, ot = osc.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))
    assert np.array_equal(t.view(np.uint32), ot.view(np.uint32))


@pytest.mark.parametrize("width", [2, 4, 6])
def test_twin_narrow_trees_match_oracle(tmp_path, width):
    """Wide nodes built with at most `width` children (the 8-slot record keeps the rest empty):
    the same closest hits, a deeper tree, more node visits than 8-wide."""
    from master_thesis_b200 import scenes
    s = scenes.terrain(5, str(tmp_path), cells=32, tile=16, spheres=4, sphere_subdiv=2, lights=1)
    sd = swr.load_scene(s["scene"], s["basepath"])
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(20000, sd.vpos.min(0) - 0.1, sd.vpos.max(0) + 0.1, seed=12)
    otri, od2, _ = osc.trace(ro, rd)
    wide = Twin(sd)
    narrow = Twin(sd, width=width)
    tri, d2, _ = narrow.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))
    assert narrow.depth > wide.depth and narrow.num_nodes > wide.num_nodes
    words = narrow.node_words().reshape(-1, 20)
    children = np.array([bin(int(w[3]) >> 24).count("1") for w in words]) + \
        np.array([sum(((int(w[6 + i // 4]) >> (8 * (i % 4))) & 0xFF) != 0 for i in range(8)) for w in words])
    assert children.max() <= width


def test_twin_axis_aligned_and_degenerate_rays():
    """Rays with zero direction components, rays starting on box faces and through shared edges
    (exact ties between the two triangles of a quad)."""
    g = golden("ref_cornell_box_with_blocks")
    sd = golden_scene(g)
    tw = Twin(sd)
    osc = O.OracleScene.from_scene_data(sd)
    rng = np.random.default_rng(3)
    n = 6000
    ro = np.zeros((n, 4), np.float32)
    rd = np.zeros((n, 4), np.float32)
    ro[:, :3] = rng.uniform(-1.1, 1.1, (n, 3)).astype(np.float32)
    # snap some origins to the walls' planes and some coordinates to 0
    ro[:1000, 0] = np.float32(1.0)
    ro[1000:2000, 1] = np.float32(-1.0)
    ro[2000:3000, 2] = 0.0
    axes = rng.integers(0, 3, n)
    rd[np.arange(n), axes] = rng.choice([-1.0, 1.0, -0.0], n)
    # diagonal rays through the quads' shared edges
    rd[3000:4000, :3] = np.float32([-1.0, 1.0, 1.0]) / np.float32(np.sqrt(3.0))
    rd[4000:5000, :3] = np.float32([-1.0, -1.0, 0.0])
    rd[5000:, :3] = rng.normal(size=(1000, 3)).astype(np.float32)
    rd[:, :3] /= np.maximum(np.linalg.norm(rd[:, :3], axis=1, keepdims=True), 1e-30)
    tri, d2, _ = tw.trace(ro, rd)
    otri, od2, _ = osc.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_twin_reference_radiance_matches_golden(name):
    g = golden(name)
    tw = Twin(golden_scene(g))
    W, H, spp, depth, seed = [int(x) for x in g["params"]]
    ps = tw.render(golden_camera(g), W, H, spp, depth, seed)
    assert np.array_equal(ps.view(np.uint32), g["per_sample"].view(np.uint32))
    assert np.array_equal(ref_pixel_from_samples(ps, spp).view(np.uint32), g["per_pixel"].view(np.uint32))


def test_twin_physical_mode_matches_fp64_oracle(tmp_path):
    s = scenes.cornell(3, str(tmp_path))
    sd = swr.load_scene(s["scene"], s["basepath"])
    tw = Twin(sd)
    osc = O.OracleScene.from_scene_data(sd)
    W, H = 24, 18
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=True)
    vi, pi, org = swr.camera_arrays(cam)
    ps = tw.render(cam, W, H, 32, 5, 77, mode=1, rr_depth=3, rr_q=0.8)
    pp64, _ = O.render_physical64(osc, O.camera(vi, pi, org), W, H, 32, 5, 77, rr_depth=3, rr_q=0.8)
    m = ps[..., :3].astype(np.float64).mean(1)
    # same paths, float vs double arithmetic: agreement to float rounding
    assert np.max(np.abs(m - pp64) / (np.abs(pp64) + 1e-3)) < 1e-4


def test_host_builder_output_independent_of_thread_count(tmp_path):
    """The host builder splits passes over large ranges and subtrees across threads; the tree,
    its records and the slot order are the same for any thread count (a 524k-triangle terrain,
    large enough for the split passes)."""
    import ctypes
    from master_thesis_b200 import _native as N
    from helpers import build_twin
    s = scenes.terrain(2, str(tmp_path), cells=512, tile=32, spheres=8, sphere_subdiv=2, lights=2)
    sd = swr.load_scene(s["scene"], s["basepath"])
    L = ctypes.CDLL(build_twin())
    P = ctypes.c_void_p
    L.twin_create.restype = P
    L.twin_create.argtypes = [P, P]
    L.twin_destroy.argtypes = [P]
    L.twin_node_words.argtypes = [P, P]
    L.twin_node_words.restype = ctypes.c_uint32
    L.twin_slot_ids.argtypes = [P, P]
    L.twin_slot_ids.restype = ctypes.c_uint32
    d = sd.desc()
    out = []
    for threads in (1, 3, 0):
        o = N.BuildOpts(0, 0, threads, 0, 0, 0)
        h = L.twin_create(ctypes.byref(d), ctypes.byref(o))
        assert h
        words = np.empty(L.twin_node_words(h, None), np.uint32)
        L.twin_node_words(h, words.ctypes.data)
        ids = np.empty(L.twin_slot_ids(h, None), np.uint32)
        L.twin_slot_ids(h, ids.ctypes.data)
        L.twin_destroy(h)
        out.append((words, ids))
    assert sd.num_triangles > 2 ** 19
    assert np.array_equal(np.sort(out[0][1]), np.arange(sd.num_triangles, dtype=np.uint32))
    for words, ids in out[1:]:
        assert np.array_equal(words, out[0][0]) and np.array_equal(ids, out[0][1])


def _degenerate_scene(kind, rng):
    """Triangles whose box centres are equal (stacked copies, copies on a lattice) or lie on one
    line, as two objects."""
    n = 1500
    if kind == "stacked":  # copies of a few triangles: every centroid equal inside a copy group
        base = rng.uniform(-1, 1, (4, 3, 3))
        v = base[rng.integers(0, 4, n)]
    elif kind == "collinear":  # triangles whose centroids lie on one line along x
        x = rng.uniform(-1, 1, n)
        v = np.stack([np.stack([x, np.zeros(n), np.zeros(n)], 1),
                      np.stack([x + 0.01, np.full(n, 0.3), np.zeros(n)], 1),
                      np.stack([x + 0.02, np.zeros(n), np.full(n, 0.3)], 1)], 1)
    else:  # "points": one triangle shape placed on a coarse lattice, many copies at each place
        c = np.round(rng.uniform(-1, 1, (n, 3)) * 3) / 3
        v = c[:, None, :] + rng.uniform(-0.2, 0.2, (1, 3, 3))
    v = v.astype(np.float32).reshape(-1, 3)
    nrm = np.tile(np.float32([0, 1, 0]), (v.shape[0], 1))
    tri = np.arange(v.shape[0], dtype=np.uint32).reshape(-1, 3)
    tri_obj = (np.arange(n) >= n // 2).astype(np.uint32)
    from master_thesis_b200.api import MAT_DTYPE, SceneData
    mats = np.zeros(2, MAT_DTYPE)
    mats["color"] = 0.5
    mats["diffuse_t"] = 1.0
    mats["refraction_index"] = 1.0
    return SceneData(v, nrm, tri, tri_obj, np.array([0, 3 * (n // 2), 3 * n], np.uint32), mats,
                     tri_rank=np.arange(n, dtype=np.uint32))


@pytest.mark.parametrize("kind", ["stacked", "collinear", "points"])
@pytest.mark.parametrize("sah_bins", [0, 8])
def test_twin_degenerate_geometry_matches_oracle(kind, sah_bins):
    """The host builder's fallbacks (equal centroids: median split; empty centroid extents) and
    the sparse SAH sweep of small ranges, through the traversal, against the oracle."""
    rng = np.random.default_rng(len(kind) + sah_bins)
    sd = _degenerate_scene(kind, rng)
    tw = Twin(sd, sah_bins=sah_bins)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(20000, sd.vpos.min(0) - 0.2, sd.vpos.max(0) + 0.2, seed=5)
    tri, d2, t = tw.trace(ro, rd)
    otri, od2, ot = osc.trace(ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(d2.view(np.uint32), od2.view(np.uint32))
    assert np.mean(otri != 0xFFFFFFFF) > 0.01
