"""The FP64 host reference gradient (oracle) is itself checked against central finite differences
of the FP64 host renderer on the same paths, before it is used to check the GPU adjoint."""
import numpy as np

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from oracle import oracle as O


def _setup(tmp_path):
    s = scenes.cornell_tessellated(4, str(tmp_path), wall_cells=4, box_cells=2)
    sd = swr.load_scene(s["scene"], s["basepath"])
    rng = np.random.default_rng(0)
    albedo = rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)
    emission = (sd.materials["color"] * sd.materials["light_strength"][:, None]).astype(np.float32)
    W, H = 12, 9
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=True)
    vi, pi, org = swr.camera_arrays(cam)
    return sd, albedo, emission, O.camera(vi, pi, org), W, H


def test_fp64_gradient_matches_fp64_finite_differences(tmp_path):
    sd, albedo, emission, cam, W, H = _setup(tmp_path)
    spp, depth, seed, rr, q = 8, 5, 3, 3, 0.8
    rng = np.random.default_rng(1)
    target = rng.uniform(0.0, 0.5, (W * H, 3))

    def loss(alb, em):
        sc = O.OracleScene.from_scene_data(sd, albedo=alb, emission=em)
        img, _ = O.render_physical64(sc, cam, W, H, spp, depth, seed, rr_depth=rr, rr_q=q)
        return float(np.sum((img - target) ** 2)), img

    L0, img = loss(albedo, emission)
    dl = (2.0 * (img - target)).astype(np.float32)
    sc = O.OracleScene.from_scene_data(sd, albedo=albedo, emission=emission)
    ga, ge = O.adjoint_physical64(sc, cam, W, H, spp, depth, seed, dl, rr_depth=rr, rr_q=q)
    # the gradient is linear in dl, and dl is float32: compare against FD of the same linear form
    dl64 = dl.astype(np.float64)
    flat = np.argsort(-np.abs(ga).ravel())[:24]
    h = 1e-4
    for k in flat:
        t, c = divmod(int(k), 3)
        ap, am = albedo.astype(np.float64).copy(), albedo.astype(np.float64).copy()
        ap[t, c] += h
        am[t, c] -= h
        scp = O.OracleScene.from_scene_data(sd, albedo=ap.astype(np.float32), emission=emission)
        scm = O.OracleScene.from_scene_data(sd, albedo=am.astype(np.float32), emission=emission)
        ip, _ = O.render_physical64(scp, cam, W, H, spp, depth, seed, rr_depth=rr, rr_q=q)
        im, _ = O.render_physical64(scm, cam, W, H, spp, depth, seed, rr_depth=rr, rr_q=q)
        # albedo is stored as float32 in the scene: use the perturbation actually applied
        dh = float(np.float32(ap[t, c])) - float(np.float32(am[t, c]))
        fd = float(np.sum(dl64 * (ip - im))) / dh
        assert abs(fd - ga[t, c]) <= 1e-6 * max(abs(fd), abs(ga[t, c])) + 1e-12, (t, c, fd, ga[t, c])
    lights = np.nonzero(sd.materials["light_source"])[0]
    for o in lights:
        for c in range(3):
            ep, em_ = emission.astype(np.float64).copy(), emission.astype(np.float64).copy()
            ep[o, c] += 1e-3
            em_[o, c] -= 1e-3
            ip = O.render_physical64(O.OracleScene.from_scene_data(sd, albedo=albedo, emission=ep.astype(np.float32)),
                                     cam, W, H, spp, depth, seed, rr_depth=rr, rr_q=q)[0]
            im = O.render_physical64(O.OracleScene.from_scene_data(sd, albedo=albedo, emission=em_.astype(np.float32)),
                                     cam, W, H, spp, depth, seed, rr_depth=rr, rr_q=q)[0]
            dh = float(np.float32(ep[o, c])) - float(np.float32(em_[o, c]))
            fd = float(np.sum(dl64 * (ip - im))) / dh
            assert abs(fd - ge[o, c]) <= 1e-6 * max(abs(fd), abs(ge[o, c])) + 1e-12
    assert np.abs(ga).max() > 0 and np.abs(ge[lights]).max() > 0
