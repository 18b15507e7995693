"""Regenerates the golden fixtures in tests/golden/ by running the reference's own code (the
harness in oracle/_ref/, built from the reference sources by oracle/Makefile).

For each case it stores, from the reference: the world-space scene exactly as its
GraphicsObject::init produced it (vertices, normals, triangles, materials, the tie-break visit
ranks from its BVHs), the camera matrices of GraphicsEngine::render, the closest hits of
Scene::traceRay for a seeded ray set, and PathTracer and BidirectionalPathTracer radiance per
sample (Philox shim) for a small image. Run from the repository root:  python tests/golden/make_golden.py
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle import refdump  # noqa: E402
from master_thesis_b200 import scenes  # noqa: E402
from helpers import rays_uniform  # noqa: E402

REF = refdump.reference_root()
OUT = os.path.dirname(os.path.abspath(__file__))
W, H, SPP, DEPTH, SEED = 32, 24, 4, 5, 20240601
BD_VISION, BD_LIGHT, BD_MAX = 5, 5, 5  # res/renderer/SoftwareRendererBidirectionalPathTracer.renderer
NRAYS = 4096


def ranks_from_dump(R):
    nt = R["tri_obj"].shape[0]
    ofs, nts = R["obj_first_tri"], R["obj_num_tris"]
    rank = np.zeros(nt, np.uint32)
    tord = np.split(R["tri_order"].astype(np.int64), np.cumsum(nts)[:-1])
    b = 0
    for o in R["scene_order"]:
        rank[ofs[o] + tord[o]] = b + np.arange(nts[o])
        b += int(nts[o])
    return rank


def make(name, scene, camera, basepath, tmp):
    R = refdump.dump(basepath, scene, camera, W, H, os.path.join(tmp, name + ".dump"))
    vpos = R["vpos"].reshape(-1, 3)
    lo, hi = vpos.min(0) - 0.25, vpos.max(0) + 0.25
    ro, rd = rays_uniform(NRAYS, lo, hi, seed=17)
    hits = refdump.trace(basepath, scene, np.concatenate([ro[:, :3], rd[:, :3]], 1), os.path.join(tmp, name + ".hits"))
    rend = refdump.render(basepath, scene, camera, W, H, SPP, DEPTH, SEED, 0, W * H, os.path.join(tmp, name + ".rend"))
    bd = refdump.render_bdpt(basepath, scene, camera, W, H, SPP, BD_VISION, BD_LIGHT, BD_MAX, SEED, 0, W * H,
                             os.path.join(tmp, name + ".bdpt"))
    om = R["obj_mat"].reshape(-1, 8)
    np.savez_compressed(
        os.path.join(OUT, name + ".npz"),
        vpos=vpos, vnrm=R["vnrm"].reshape(-1, 3), tri=R["tri"].reshape(-1, 3), tri_obj=R["tri_obj"],
        obj_first_vertex=np.append(R["obj_first_vertex"], vpos.shape[0]).astype(np.uint32),
        mat_color=om[:, :3], mat_thresholds=om[:, 3:6], mat_eta=om[:, 6], mat_strength=om[:, 7],
        mat_light=R["obj_light"], tri_rank=ranks_from_dump(R),
        tri_e0=R["tri_e0"].reshape(-1, 3), tri_e1=R["tri_e1"].reshape(-1, 3), tri_den=R["tri_den"].reshape(-1, 4),
        tri_box=R["tri_box"].reshape(-1, 6), obj_box=R["obj_box"].reshape(-1, 6),
        cam_view_inv=R["camera"][:16].reshape(4, 4), cam_proj_inv=R["camera"][16:32].reshape(4, 4),
        cam_origin=R["camera"][32:35], ray_o=ro, ray_d=rd, hit_id=hits["hit_id"], hit_obj=hits["hit_obj"],
        hit_d2=hits["hit_d2"], hit_pos=hits["hit_pos"].reshape(-1, 3), hit_nrm=hits["hit_nrm"].reshape(-1, 3),
        per_sample=rend["per_sample"].reshape(W * H, SPP, 4), per_pixel=rend["per_pixel"].reshape(W * H, 3),
        params=np.array([W, H, SPP, DEPTH, SEED], np.uint64),
        bdpt_per_sample=bd["per_sample"].reshape(W * H, SPP, 4),
        bdpt_params=np.array([W, H, SPP, BD_VISION, BD_LIGHT, BD_MAX, SEED], np.uint64))
    print(name, R["tri_obj"].shape[0], "triangles")


def main():
    if not refdump.available():
        sys.exit("build oracle/_ref first (make -C oracle ref)")
    base = REF + "/build/"
    cam = REF + "/res/camera/close.camera"
    with tempfile.TemporaryDirectory() as tmp:
        for sc in ["cornell_box_with_blocks", "cornell_box_with_ball", "cornell_box_with_blocks_and_ball",
                   "cornell_box_5", "white_room"]:
            make("ref_" + sc, REF + "/res/scene/%s.scene" % sc, cam, base, tmp)
        g = scenes.cornell(3, os.path.join(tmp, "c1"))
        make("gen_cornell_3", g["scene"], g["camera"], g["basepath"], tmp)


if __name__ == "__main__":
    main()
