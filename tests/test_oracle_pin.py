"""The oracle (C restatement) is pinned to the reference's own outputs: the golden fixtures were
produced by the reference's code (tests/golden/make_golden.py); here the oracle must reproduce
them bit for bit. When the compiled reference is available it is also compared live."""
import os

import numpy as np
import pytest

from helpers import GOLDEN_CASES, golden, golden_camera, golden_scene, ref_pixel_from_samples, rays_uniform
from oracle import oracle as O
from oracle import refdump


PHILOX_KAT = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
              ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
              ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
               (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]


def test_philox_known_answers():
    """Philox-4x32-10 known-answer vectors (Salmon et al. 2011) for the Python restatement, the
    oracle's C generator and the kernels' generator (host build of swr_exact.cuh)."""
    import ctypes
    from helpers import build_twin
    twin = ctypes.CDLL(build_twin())
    olib = O.lib()
    for ctr, key, want in PHILOX_KAT:
        assert _philox_py(ctr, key) == want
        c = (ctypes.c_uint32 * 4)(*ctr)
        k = (ctypes.c_uint32 * 2)(*key)
        o1 = (ctypes.c_uint32 * 4)()
        o2 = (ctypes.c_uint32 * 4)()
        olib.swo_philox(c, k, o1)
        twin.twin_philox(c, k, o2)
        assert tuple(o1) == want and tuple(o2) == want


def _philox_py(ctr, key):
    M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0, p1 = M0 * c0, M1 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF, ((p0 >> 32) ^ c3 ^ k1) & 0xFFFFFFFF, p0 & 0xFFFFFFFF
        k0, k1 = (k0 + W0) & 0xFFFFFFFF, (k1 + W1) & 0xFFFFFFFF
    return (c0, c1, c2, c3)


def _oracle_scene(name):
    g = golden(name)
    R = {"tri_v0": g["vpos"][g["tri"][:, 0]], "tri_e0": g["tri_e0"], "tri_e1": g["tri_e1"],
         "tri_den": g["tri_den"], "tri_box": g["tri_box"], "obj_box": g["obj_box"], "tri_obj": g["tri_obj"]}
    nrm = g["vnrm"][g["tri"].astype(np.int64)].reshape(-1, 9)
    mats = np.concatenate([g["mat_color"], g["mat_thresholds"], g["mat_eta"][:, None],
                           g["mat_light"][:, None].astype(np.float32), g["mat_strength"][:, None]], 1)
    sc = O.OracleScene(R["tri_v0"], R["tri_e0"], R["tri_e1"], R["tri_den"], R["tri_box"], R["obj_box"],
                       R["tri_obj"], g["tri_rank"], nrm, mats,
                       vtx=g["vpos"][g["tri"].astype(np.int64)].reshape(-1, 9))
    return g, sc


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_hits_match_reference(name):
    g, sc = _oracle_scene(name)
    tri, d2, _ = sc.trace(g["ray_o"], g["ray_d"])
    assert np.array_equal(tri, g["hit_id"])
    assert np.array_equal(d2.view(np.uint32), g["hit_d2"].view(np.uint32))
    assert (tri != 0xFFFFFFFF).mean() > 0.3


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_radiance_matches_reference(name):
    g, sc = _oracle_scene(name)
    W, H, spp, depth, seed = [int(x) for x in g["params"]]
    cam = O.camera(g["cam_view_inv"], g["cam_proj_inv"], g["cam_origin"])
    ps, pp = O.render_reference(sc, cam, W, H, spp, depth, seed)
    assert np.array_equal(ps.view(np.uint32), g["per_sample"].view(np.uint32))
    assert np.array_equal(pp.view(np.uint32), g["per_pixel"].view(np.uint32))
    assert np.array_equal(ref_pixel_from_samples(ps, spp).view(np.uint32), g["per_pixel"].view(np.uint32))


def bdpt_reference_values(per_sample):
    """What the reference's BidirectionalPathTracer::renderPixel returns for one sample: the
    contribution scaled by 2 pi (in double, stored to float)."""
    return (per_sample[..., :3].astype(np.float64) * (2.0 * np.pi)).astype(np.float32)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_bdpt_matches_reference(name):
    g, sc = _oracle_scene(name)
    W, H, spp, vj, lj, md, seed = [int(x) for x in g["bdpt_params"]]
    cam = O.camera(g["cam_view_inv"], g["cam_proj_inv"], g["cam_origin"])
    ps, pp = O.render_bdpt(sc, cam, W, H, spp, vj, lj, md, seed)
    ref = g["bdpt_per_sample"][..., :3]
    assert np.array_equal(bdpt_reference_values(ps).view(np.uint32), ref.view(np.uint32))
    assert (np.abs(ref).sum(-1) > 0).mean() > 0.05


@pytest.mark.reference
def test_oracle_matches_live_reference_on_fresh_rays(tmp_path):
    """Fresh seeded rays through the compiled reference (not just the stored fixture)."""
    import master_thesis_b200 as swr
    ref = refdump.reference_root()
    base = os.path.join(ref, "build") + "/"
    for sc_name in ["cornell_box_with_ball", "labyrinth"]:
        scene = os.path.join(ref, "res/scene/%s.scene" % sc_name)
        D = swr.load_scene(scene, base)
        osc = O.OracleScene.from_scene_data(D)
        ro, rd = rays_uniform(20000, D.vpos.min(0) - 0.2, D.vpos.max(0) + 0.2, seed=123)
        H = refdump.trace(base, scene, np.concatenate([ro[:, :3], rd[:, :3]], 1), str(tmp_path / "h.bin"))
        tri, d2, _ = osc.trace(ro, rd)
        assert np.array_equal(tri, H["hit_id"])
        assert np.array_equal(d2.view(np.uint32), H["hit_d2"].view(np.uint32))
