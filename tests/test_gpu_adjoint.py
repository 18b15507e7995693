"""GPU path-replay adjoint (swr_render_adjoint through the C ABI, and the torch.autograd.Function
on top of it) against the FP64 host reference gradient and central finite differences of the GPU
renderer with shared random-number seeds."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from master_thesis_b200.diff import render_physical
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPP, DEPTH, SEED, RR, Q = 16, 5, 7, 3, 0.8
W, H = 32, 24


@pytest.fixture(scope="module")
def setup(tmp_path_factory):
    root = tmp_path_factory.mktemp("tess")
    s = scenes.cornell_tessellated(4, str(root), wall_cells=8, box_cells=5)
    sd = swr.load_scene(s["scene"], s["basepath"])
    scene = swr.Scene(sd)
    rng = np.random.default_rng(0)
    albedo = rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)
    emission = (sd.materials["color"] * sd.materials["light_strength"][:, None]).astype(np.float32)
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=True)
    target = torch.from_numpy(rng.uniform(0.0, 0.4, (H, W, 3)).astype(np.float32)).cuda()
    return sd, scene, albedo, emission, cam, target


def _render(scene, cam, albedo, emission):
    scene.set_albedo(torch.from_numpy(albedo).cuda())
    scene.set_emission(torch.from_numpy(emission).cuda())
    img = scene.render(cam, W, H, SPP, DEPTH, seed=SEED, mode=swr.MODE_PHYSICAL, rr_depth=RR, rr_survive=Q)
    torch.cuda.synchronize()
    return img


@pytest.mark.parametrize("shade_batch", [0, 1, 16, 32])
def test_adjoint_matches_fp64_reference_gradient(setup, shade_batch):
    sd, scene, albedo, emission, cam, target = setup
    img = _render(scene, cam, albedo, emission)
    dl = (2.0 * (img - target)).contiguous()
    ga, ge = scene.render_adjoint(cam, W, H, SPP, DEPTH, dl, seed=SEED, rr_depth=RR, rr_survive=Q,
                                  shade_batch=shade_batch)
    torch.cuda.synchronize()
    ga, ge = ga.cpu().numpy().astype(np.float64), ge.cpu().numpy().astype(np.float64)
    vi, pi, org = swr.camera_arrays(cam)
    osc = O.OracleScene.from_scene_data(sd, albedo=albedo, emission=emission)
    ra, re = O.adjoint_physical64(osc, O.camera(vi, pi, org), W, H, SPP, DEPTH, SEED, dl.cpu().numpy(),
                                  rr_depth=RR, rr_q=Q)
    # same paths: the float32 gradient agrees with the double one up to float accumulation
    assert np.linalg.norm(ga - ra) <= 1e-4 * np.linalg.norm(ra)
    assert np.linalg.norm(ge - re) <= 1e-4 * np.linalg.norm(re)
    assert np.abs(ra).max() > 0


def test_adjoint_matches_central_differences(setup):
    sd, scene, albedo, emission, cam, target = setup
    tgt = target.double()

    def loss(alb, em):
        return float(torch.sum((_render(scene, cam, alb, em).double() - tgt) ** 2))

    img = _render(scene, cam, albedo, emission)
    ga, ge = scene.render_adjoint(cam, W, H, SPP, DEPTH, (2.0 * (img - target)).contiguous(), seed=SEED,
                                  rr_depth=RR, rr_survive=Q)
    ga, ge = ga.cpu().numpy(), ge.cpu().numpy()
    rng = np.random.default_rng(3)
    # 64 random parameters among those that influence the image noticeably
    cand = np.argsort(-np.abs(ga).ravel())[:2000]
    picks = rng.choice(cand, 64, replace=False)
    h = 1e-3
    errs = []
    for k in picks:
        t, c = divmod(int(k), 3)
        ap, am = albedo.copy(), albedo.copy()
        ap[t, c] += h
        am[t, c] -= h
        fd = (loss(ap, emission) - loss(am, emission)) / (float(ap[t, c]) - float(am[t, c]))
        errs.append(abs(fd - ga[t, c]) / max(abs(fd), abs(ga[t, c]), 1e-12))
    assert max(errs) <= 1e-2, sorted(errs)[-5:]
    for o in np.nonzero(sd.materials["light_source"])[0]:
        for c in range(3):
            ep, em_ = emission.copy(), emission.copy()
            ep[o, c] += h
            em_[o, c] -= h
            fd = (loss(albedo, ep) - loss(albedo, em_)) / (float(ep[o, c]) - float(em_[o, c]))
            assert abs(fd - ge[o, c]) <= 1e-2 * max(abs(fd), abs(ge[o, c]), 1e-12)


def test_autograd_function(setup):
    sd, scene, albedo, emission, cam, target = setup
    a = torch.from_numpy(albedo).cuda().requires_grad_(True)
    e = torch.from_numpy(emission).cuda().requires_grad_(True)
    img = render_physical(scene, cam, a, e, W, H, SPP, DEPTH, seed=SEED, rr_depth=RR, rr_survive=Q)
    loss = torch.sum((img - target) ** 2)
    loss.backward()
    ref = _render(scene, cam, albedo, emission)
    assert torch.equal(img.detach(), ref)
    ga, ge = scene.render_adjoint(cam, W, H, SPP, DEPTH, (2.0 * (ref - target)).contiguous(), seed=SEED,
                                  rr_depth=RR, rr_survive=Q)
    assert torch.allclose(a.grad, ga, rtol=1e-5, atol=1e-9)
    assert torch.allclose(e.grad, ge, rtol=1e-5, atol=1e-9)
