"""The configuration the benchmark times, checked against the oracle: the terrain scene (2,424,840
triangles in 4,164 objects) rendered with the reference's PathTracer semantics at depth 8 with
2^27 paths in flight (the whole image at once), per sample on image rows spread over the whole 1920x1080 image. Also a small
terrain at depth 8 with few and with many paths in flight, and batched jobs compared with the
oracle directly (not only with single-scene renders).

Reference: software_renderer/graphic/path_tracer.cpp:18-97 (renderPixel, traceSinglePath),
graphic/scene.cpp:22-56 (traceRay)."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# Radiance tolerance of the render tests: every float operation rounds like the reference's; only
# the double-precision sin/cos/acos of the device's libm and glibc may differ in the last bit.
RTOL, ATOL = 1e-4, 1e-7

# The benchmark's terrain image (bench.py, configuration c2): rank 0 renders with seed 1000.
BENCH_W, BENCH_H, BENCH_SPP, BENCH_DEPTH, BENCH_SEED, BENCH_WAVE = 1920, 1080, 64, 8, 1000, 1 << 27
BENCH_SCENE = dict(seed=2024, cells=1024, tile=16, spheres=64, sphere_subdiv=4, lights=4)


def _close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= RTOL * np.maximum(np.abs(b), 1e-6) + ATOL)


def _check_rows(samples, img, osc, cam, W, H, spp, depth, seed, rows):
    """samples: [H*W, spp, 4] host copy of the GPU's per-sample radiance; img: [H, W, 3]."""
    vi, pi, org = swr.camera_arrays(cam)
    ocam = O.camera(vi, pi, org)
    lit = 0
    for y in rows:
        ps, pp = O.render_reference(osc, ocam, W, H, spp, depth, seed, y * W, (y + 1) * W)
        got = samples[y * W:(y + 1) * W]
        # the same set of paths reaches a light, and every sample's radiance agrees
        assert np.array_equal(got[..., 3], ps[..., 3]), y
        assert _close(got[..., :3], ps[..., :3]), y
        assert _close(img[y], pp), y
        lit += int((ps[..., 3] > 0).sum())
    return lit


def test_terrain_bench_image_vs_oracle(tmp_path):
    """The benchmarked render itself: same scene files, camera, seed, depth and paths in flight as
    bench.py's default run; eight image rows (15,360 pixels x 64 samples) against the oracle."""
    kw = dict(BENCH_SCENE)
    s = scenes.terrain(kw.pop("seed"), str(tmp_path), **kw)
    sd = swr.load_scene(s["scene"], s["basepath"])
    assert sd.num_triangles == 2424840 and sd.ranks_exact
    sc = swr.Scene(sd)
    W, H, spp, depth, seed = BENCH_W, BENCH_H, BENCH_SPP, BENCH_DEPTH, BENCH_SEED
    cam = swr.load_camera(s["camera"], W, H)
    samples = torch.zeros((H * W, spp, 4), dtype=torch.float32, device="cuda")
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    sc.render(cam, W, H, spp, depth, seed=seed, wave_size=BENCH_WAVE, out=out, samples=samples)
    torch.cuda.synchronize()
    rows = [int(r) for r in np.linspace(H // 16, H - 1 - H // 16, 8)]
    idx = torch.cat([torch.arange(y * W, (y + 1) * W) for y in rows]).cuda()
    band = samples[idx].cpu().numpy()
    img = out.cpu().numpy()
    host = np.zeros((H * W, spp, 4), np.float32)
    for k, y in enumerate(rows):
        host[y * W:(y + 1) * W] = band[k * W:(k + 1) * W]
    del samples
    osc = O.OracleScene.from_scene_data(sd)
    lit = _check_rows(host, img, osc, cam, W, H, spp, depth, seed, rows)
    assert lit > 1000  # the rows include paths that reach the emissive quads
    # the whole image: finite, non-negative, and as bright as a resolve of the checked rows says
    assert np.all(np.isfinite(img)) and img.min() >= 0.0
    sc.close()


@pytest.mark.parametrize("wave", [4096, 1 << 27])
def test_small_terrain_depth8_vs_oracle(tmp_path, wave):
    """Depth 8 on a terrain with few paths in flight (many injections and compactions) and with a
    request for 2^27 (clamped to the image's samples): every pixel and sample against the oracle."""
    s = scenes.terrain(9, str(tmp_path), cells=64, tile=16, spheres=8, sphere_subdiv=2, lights=2)
    sd = swr.load_scene(s["scene"], s["basepath"])
    assert sd.ranks_exact
    sc = swr.Scene(sd)
    W, H, spp, depth, seed = 96, 64, 16, 8, 77
    cam = swr.load_camera(s["camera"], W, H)
    samples = np.zeros((H * W, spp, 4), np.float32)
    out = np.zeros((H, W, 3), np.float32)
    sc.render(cam, W, H, spp, depth, seed=seed, wave_size=wave, out=out, samples=samples)  # host buffers
    osc = O.OracleScene.from_scene_data(sd)
    lit = _check_rows(samples, out, osc, cam, W, H, spp, depth, seed, range(H))
    assert lit > 0
    sc.close()


def test_batch_jobs_vs_oracle():
    """Batched jobs of both modes against the oracle directly: reference-mode images against the
    oracle's per-pixel radiance, physical-mode images against the FP64 restatement on the same
    paths. The batch sums each pixel's samples in 64-bit fixed point, so agreement is to float
    rounding, not per sample."""
    rng = np.random.default_rng(8)
    specs = [(3000, 40, 30, 8, 0), (12000, 48, 36, 4, 1), (3000, 24, 18, 16, 1), (12000, 32, 24, 8, 0)]
    built = {}
    jobs = []
    for tris, w, h, spp, mode in specs:
        if tris not in built:
            sd, cam = scenes.random_scene(300 + tris, tris)
            built[tris] = (sd, swr.Scene(sd), cam)
        sd, sc, c = built[tris]
        jobs.append(dict(scene=sc, cam=swr.make_camera(c["position"], c["angle"], w, h, fov_deg=40), width=w,
                         height=h, spp=spp, depth=6, seed=int(rng.integers(1 << 30)), mode=mode,
                         rr_depth=3 if mode else 0, rr_survive=0.8 if mode else 1.0, data=sd))
    batch = swr.Batch()
    outs = batch.render(jobs, wave_size=1 << 13)
    torch.cuda.synchronize()
    for j, o in zip(jobs, outs):
        osc = O.OracleScene.from_scene_data(j["data"])
        vi, pi, org = swr.camera_arrays(j["cam"])
        got = o.cpu().numpy().reshape(-1, 3).astype(np.float64)
        if j["mode"] == 0:
            _, pp = O.render_reference(osc, O.camera(vi, pi, org), j["width"], j["height"], j["spp"], j["depth"],
                                       j["seed"])
            assert _close(got, pp), np.abs(got - pp).max()
        else:
            pp64, _ = O.render_physical64(osc, O.camera(vi, pi, org), j["width"], j["height"], j["spp"],
                                          j["depth"], j["seed"], rr_depth=3, rr_q=0.8)
            assert np.max(np.abs(got - pp64) / (np.abs(pp64) + 1e-3)) < 1e-4
        assert got.max() > 0
    batch.close()
