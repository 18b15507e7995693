"""Batched rendering (swr_render_batch): many uneven scenes in one shared wavefront must give each
job the image a single-scene render of that job gives (up to the order of the per-pixel sums)."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes

pytestmark = pytest.mark.gpu


def _jobs():
    rng = np.random.default_rng(5)
    out = []
    built = {}
    for k, (tris, size, spp, mode) in enumerate([(1000, 32, 4, 1), (20000, 64, 16, 1), (5000, 48, 64, 0),
                                                 (60000, 80, 4, 1), (1000, 16, 16, 0), (20000, 24, 8, 1)]):
        if tris not in built:
            sd, cam = scenes.random_scene(100 + tris, tris)
            built[tris] = (swr.Scene(sd), cam)
        sc, cam = built[tris]
        w, h = size, size * 3 // 4
        out.append(dict(scene=sc, cam=swr.make_camera(cam["position"], cam["angle"], w, h, fov_deg=40), width=w,
                        height=h, spp=spp, depth=6, seed=int(rng.integers(1 << 30)), mode=mode))
    return out


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_matches_single_renders(use_graph):
    jobs = _jobs()
    batch = swr.Batch()
    for rep in range(2):  # the second call reuses the buffers and the captured graph
        outs = batch.render(jobs, wave_size=1 << 14, use_graph=use_graph)
        torch.cuda.synchronize()
        for j, o in zip(jobs, outs):
            ref = j["scene"].render(j["cam"], j["width"], j["height"], j["spp"], j["depth"], seed=j["seed"],
                                    mode=j["mode"])
            torch.cuda.synchronize()
            a, b = o.cpu().numpy(), ref.cpu().numpy()
            assert np.allclose(a, b, rtol=1e-5, atol=1e-7), (rep, np.abs(a - b).max())
            assert b.max() > 0
    batch.close()


def test_batch_rejects_bad_jobs():
    jobs = _jobs()[:1]
    batch = swr.Batch()
    bad = dict(jobs[0])
    bad["depth"] = 0
    with pytest.raises(swr.SwrError):
        batch.render([bad])
    batch.close()


def test_batch_subwavefronts_equal_one_wavefront():
    """A batch of 2^20 samples or more runs as concurrent sub-wavefronts over ranges of the global
    sample index; its images equal those of the host-driven single wavefront bit for bit (the
    per-pixel sums are order-independent fixed point)."""
    sd, cam = scenes.random_scene(41, 8000)
    sc = swr.Scene(sd)
    jobs = []
    for k, (w, spp, mode) in enumerate([(128, 32, 1), (96, 48, 0), (160, 16, 1)]):  # 1.4 M samples
        jobs.append(dict(scene=sc, cam=swr.make_camera(cam["position"], cam["angle"], w, w, fov_deg=40), width=w,
                         height=w, spp=spp, depth=6, seed=100 + k, mode=mode))
    batch = swr.Batch()
    a = [o.clone() for o in batch.render(jobs, wave_size=1 << 16, use_graph=True)]
    b = [o.clone() for o in batch.render(jobs, wave_size=1 << 16, use_graph=False)]
    c = [o.clone() for o in batch.render(jobs, wave_size=1 << 16, use_graph=True)]  # graphs reused
    torch.cuda.synchronize()
    for x, y, z in zip(a, b, c):
        assert torch.equal(x, y) and torch.equal(x, z)
        assert float(x.max()) > 0
    batch.close()
