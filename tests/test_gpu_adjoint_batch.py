"""Batched path-replay adjoint (swr_render_adjoint_batch) and the batched torch.autograd.Function:
every job's gradients must equal the single-scene adjoint's for that job (same paths; the float
atomic sums may add in another order)."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from master_thesis_b200.diff import render_physical, render_physical_batch

pytestmark = pytest.mark.gpu

DEPTH, RR, Q = 5, 3, 0.8


def _jobs():
    out = []
    for k, (tris, w, h, spp) in enumerate([(2000, 40, 30, 8), (12000, 64, 48, 4), (600, 24, 24, 16),
                                           (30000, 48, 36, 4)]):
        sd, cam = scenes.random_scene(500 + k, tris)
        sc = swr.Scene(sd)
        out.append(dict(scene=sc, cam=swr.make_camera(cam["position"], cam["angle"], w, h, fov_deg=40), width=w,
                        height=h, spp=spp, depth=DEPTH, seed=31 + k, rr_depth=RR, rr_survive=Q))
    return out


def _close(a, b, tol=1e-4):
    a, b = a.double().cpu(), b.double().cpu()
    return float((a - b).norm()) <= tol * max(float(b.norm()), 1e-30)


@pytest.mark.parametrize("shade_batch", [0, 1, 24])
def test_batch_adjoint_matches_single_jobs(shade_batch):
    jobs = _jobs()
    rng = np.random.default_rng(1)
    for j in jobs:
        j["dl_dimage"] = torch.from_numpy(rng.normal(size=(j["height"], j["width"], 3)).astype(np.float32)).cuda()
    batch = swr.Batch()
    for rep in range(2):  # the second call reuses the batch buffers and re-zeroes the gradients
        grads = batch.render_adjoint(jobs, shade_batch=shade_batch)
        torch.cuda.synchronize()
        for j, (ga, ge) in zip(jobs, grads):
            ra, re = j["scene"].render_adjoint(j["cam"], j["width"], j["height"], j["spp"], j["depth"],
                                               j["dl_dimage"], seed=j["seed"], rr_depth=RR, rr_survive=Q)
            torch.cuda.synchronize()
            assert float(ra.abs().max()) > 0
            assert _close(ga, ra) and _close(ge, re), rep
    batch.close()


def test_batch_adjoint_shared_scene_accumulates():
    jobs = _jobs()[:1]
    j = jobs[0]
    j["dl_dimage"] = torch.ones((j["height"], j["width"], 3), device="cuda")
    ga = torch.full((j["scene"].data.num_triangles, 3), 7.0, device="cuda")
    ge = torch.full((j["scene"].data.num_objects, 3), 7.0, device="cuda")
    two = [dict(j, grad_albedo=ga, grad_emission=ge), dict(j, seed=j["seed"] + 1, grad_albedo=ga, grad_emission=ge)]
    batch = swr.Batch()
    batch.render_adjoint(two)
    torch.cuda.synchronize()
    r1 = j["scene"].render_adjoint(j["cam"], j["width"], j["height"], j["spp"], j["depth"], j["dl_dimage"],
                                   seed=j["seed"], rr_depth=RR, rr_survive=Q)
    r2 = j["scene"].render_adjoint(j["cam"], j["width"], j["height"], j["spp"], j["depth"], j["dl_dimage"],
                                   seed=j["seed"] + 1, rr_depth=RR, rr_survive=Q)
    assert _close(ga, r1[0] + r2[0]) and _close(ge, r1[1] + r2[1])
    batch.close()


def test_batch_adjoint_rejects_reference_mode_and_deep_paths():
    j = _jobs()[0]
    j["dl_dimage"] = torch.zeros((j["height"], j["width"], 3), device="cuda")
    batch = swr.Batch()
    with pytest.raises(swr.SwrError):
        batch.render_adjoint([dict(j, depth=17)])
    batch.close()


def test_batched_autograd_matches_single_autograd():
    jobs = _jobs()
    rng = np.random.default_rng(2)
    alb = [torch.from_numpy(rng.uniform(0.1, 0.9, (j["scene"].data.num_triangles, 3)).astype(np.float32)).cuda()
           .requires_grad_() for j in jobs]
    em = [torch.from_numpy((j["scene"].data.materials["color"] * j["scene"].data.materials["light_strength"][:, None])
                           .astype(np.float32)).cuda().requires_grad_() for j in jobs]
    tgt = [torch.from_numpy(rng.uniform(0, 0.5, (j["height"], j["width"], 3)).astype(np.float32)).cuda() for j in jobs]
    batch = swr.Batch()
    imgs = render_physical_batch(batch, jobs, alb, em)
    loss = sum(((i - t) ** 2).mean() for i, t in zip(imgs, tgt))
    loss.backward()
    for j, a, e, t, img in zip(jobs, alb, em, tgt, imgs):
        a2, e2 = a.detach().clone().requires_grad_(), e.detach().clone().requires_grad_()
        ref = render_physical(j["scene"], j["cam"], a2, e2, j["width"], j["height"], j["spp"], j["depth"], seed=j["seed"],
                              rr_depth=RR, rr_survive=Q)
        assert torch.allclose(img, ref, rtol=1e-5, atol=1e-7)
        ((ref - t) ** 2).mean().backward()
        assert _close(a.grad, a2.grad) and _close(e.grad, e2.grad)
    batch.close()
