"""The RayTrace program's PathTracer and denoisers on the GPU (swr_rt_*, through the C ABI) against
the oracle's CPU restatement."""
import os
import subprocess

import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import rt, scenes
from helpers import GOLDEN_CASES, golden, golden_camera, golden_scene, rays_uniform
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# Radiance tolerance: every float operation rounds as in the oracle; only the double-precision
# sin/cos/acos of the device libm and glibc may differ in the last bit of a double, which can move
# a float result by one ulp and then propagate.
RTOL = 1e-4


def _close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= RTOL * np.maximum(np.abs(b), 1e-6) + 1e-7)


def _oracle_scene(g):
    sd = golden_scene(g)
    cam = golden_camera(g)
    vi, pi, org = swr.camera_arrays(cam)
    return sd, cam, O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_rt_hits_match_oracle(name):
    g = golden(name)
    sd, _, osc, _ = _oracle_scene(g)
    sc = swr.Scene(sd)
    ro, rd = rays_uniform(20000, sd.vpos.min(0) - 0.3, sd.vpos.max(0) + 0.3, seed=21)
    ro[:1000, :3] = g["ray_o"][:1000, :3]
    hits = rt.trace(sc, ro, rd)  # host buffers
    otri, ot = O.rt_trace(osc, ro, rd)
    assert np.array_equal(hits[:, 0], otri)
    m = otri != 0xFFFFFFFF
    assert np.array_equal(hits[m, 3], ot[m].view(np.uint32))
    assert np.array_equal(hits[m, 1], sd.tri_obj[otri[m]])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_rt_render_matches_oracle(name):
    g = golden(name)
    sd, cam, osc, ocam = _oracle_scene(g)
    sc = swr.Scene(sd)
    W, H, spp, vj = 32, 24, 13, 5
    rgb, rgba = rt.render(sc, cam, W, H, spp, vj)
    torch.cuda.synchronize()
    want_rgb, want_rgba = O.rt_render(osc, ocam, W, H, spp, vj)
    got = rgb.cpu().numpy().reshape(-1, 3)
    assert _close(got, want_rgb)
    assert np.mean(np.all(got.view(np.uint32) == want_rgb.view(np.uint32), axis=1)) > 0.99
    assert np.mean(np.all(rgba.cpu().numpy().reshape(-1, 4) == want_rgba, axis=1)) > 0.99
    assert np.any(want_rgb > 0)


@pytest.mark.parametrize("refill,shade_batch", [(1, 1), (8, 1), (32, 1), (4, 8), (2, 32)])
def test_gpu_rt_render_larger_image_and_refill(tmp_path, refill, shade_batch):
    """Many pixels per lane (persistent refill, batched shading), host output buffers, one output
    only."""
    s = scenes.cornell(8, str(tmp_path))
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    W, H, spp, vj = 96, 64, 9, 6
    cam = swr.load_camera(s["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    want_rgb, want_rgba = O.rt_render(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, spp, vj)
    rgba = np.zeros((H, W, 4), np.uint8)
    _, out = rt.render(sc, cam, W, H, spp, vj, rgba=rgba, want_rgb=False, refill=refill, shade_batch=shade_batch)
    assert out is rgba
    assert np.mean(np.all(rgba.reshape(-1, 4) == want_rgba, axis=1)) > 0.99
    rgb = np.zeros((H, W, 3), np.float32)
    rt.render(sc, cam, W, H, spp, vj, rgb=rgb, want_rgba=False, refill=refill, shade_batch=shade_batch)
    assert _close(rgb.reshape(-1, 3), want_rgb)


@pytest.mark.parametrize("W,H", [(1, 1), (7, 3), (33, 17), (640, 480)])
@pytest.mark.parametrize("k,sigma", [(1, 1.0), (3, 0.7), (5, 1.0), (9, 2.0), (19, 5.0)])
def test_gpu_gauss_denoiser_matches_oracle(W, H, k, sigma):
    img = np.random.default_rng(W * 7 + k).integers(0, 256, (H, W, 4), dtype=np.uint8)
    want = O.rt_denoise_gauss(img, k, sigma)
    dev = torch.from_numpy(img).cuda()
    got = rt.denoise_gauss(dev, k, sigma)
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), want)
    assert np.array_equal(rt.denoise_gauss(img, k, sigma), want)  # host buffers


@pytest.mark.parametrize("W,H", [(1, 1), (2, 5), (31, 9), (1920, 1080)])
def test_gpu_median_denoiser_matches_oracle(W, H):
    img = np.random.default_rng(W + H).integers(0, 256, (H, W, 4), dtype=np.uint8)
    want = O.rt_denoise_median(img)
    got = rt.denoise_median(torch.from_numpy(img).cuda())
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), want)
    assert np.array_equal(rt.denoise_median(img), want)


def test_gpu_rt_frame_with_denoiser_chain_matches_oracle_composition():
    g = golden("ref_cornell_box_with_blocks_and_ball")
    sd, cam, osc, ocam = _oracle_scene(g)
    sc = swr.Scene(sd)
    W, H = 48, 36
    params = dict(vision_jumps=5, spp=13, denoisers=[("GaussDenoiser", 5, 1.0), ("MedianDenoiser",),
                                                     ("GaussDenoiser", 3, 0.8)])
    _, img = O.rt_render(osc, ocam, W, H, 13, 5)
    img = img.reshape(H, W, 4)
    want = O.rt_denoise_median(O.rt_denoise_gauss(img, 5, 1.0))
    want = O.rt_denoise_gauss(want, 3, 0.8)
    got = rt.render_frame(sc, cam, W, H, params)
    torch.cuda.synchronize()
    got = got.cpu().numpy()
    # the frame itself matches the oracle on > 99 % of the pixels; the denoisers are exact on it
    frame = rt.render(sc, cam, W, H, 13, 5, want_rgb=False)[1].cpu().numpy()
    exact = O.rt_denoise_gauss(O.rt_denoise_median(O.rt_denoise_gauss(frame, 5, 1.0)), 3, 0.8)
    assert np.array_equal(got, exact)
    assert np.mean(np.all(got == want, axis=2)) > 0.97
    # no denoisers: the frame itself, written to a host buffer
    host = np.zeros((H, W, 4), np.uint8)
    rt.render_frame(sc, cam, W, H, dict(vision_jumps=5, spp=13), out=host)
    assert np.array_equal(host, frame)
    # the denoised frame into host memory, twice (the scene's buffer reused), then a larger frame
    # (the buffer grows) and the smaller one again
    for _ in range(2):
        host = np.zeros((H, W, 4), np.uint8)
        rt.render_frame(sc, cam, W, H, params, out=host)
        assert np.array_equal(host, got)
    big = rt.render_frame(sc, cam, 2 * W, 2 * H, params)
    big_host = np.zeros((2 * H, 2 * W, 4), np.uint8)
    rt.render_frame(sc, cam, 2 * W, 2 * H, params, out=big_host)
    torch.cuda.synchronize()
    assert np.array_equal(big_host, big.cpu().numpy())
    host = np.zeros((H, W, 4), np.uint8)
    rt.render_frame(sc, cam, W, H, params, out=host)
    assert np.array_equal(host, got)
    # swr_rt_render's host outputs go through the same buffer
    rgb_d, rgba_d = rt.render(sc, cam, W, H, 13, 5)
    rgb_h, rgba_h = np.zeros((H, W, 3), np.float32), np.zeros((H, W, 4), np.uint8)
    rt.render(sc, cam, W, H, 13, 5, rgb=rgb_h, rgba=rgba_h)
    torch.cuda.synchronize()
    assert np.array_equal(rgb_h, rgb_d.cpu().numpy()) and np.array_equal(rgba_h, rgba_d.cpu().numpy())


def test_gpu_rt_invalid_arguments():
    g = golden("ref_white_room")
    sd, cam, _, _ = _oracle_scene(g)
    sc = swr.Scene(sd)
    with pytest.raises(swr.SwrError):
        rt.render(sc, cam, 8, 8, 0, 5)  # visionRayPerPixelCount 0
    with pytest.raises(swr.SwrError):
        rt.render(sc, cam, 0, 8, 1, 5)
    with pytest.raises(swr.SwrError):
        rt.render(sc, cam, 8, 8, 1, 5, refill=33)
    img = torch.zeros((4, 4, 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(swr.SwrError):
        rt.denoise_gauss(img, 4, 1.0)  # even kernel size
    with pytest.raises(swr.SwrError):
        rt.denoise_median(img, out=img)  # in place
    with pytest.raises(swr.SwrError):
        rt.render_frame(sc, cam, 8, 8, dict(vision_jumps=5, spp=2, denoisers=[("GaussDenoiser", 2, 1.0)]))


def test_gpu_raytrace_cli(tmp_path):
    """The headless RayTrace drop-in: renderer file with a denoiser, scene, camera, result image."""
    s = scenes.cornell(4, str(tmp_path))
    W, H = 40, 30
    rfile = tmp_path / "path_tracer.renderer"
    rfile.write_text("PathTracer\n\tvisionJumpCount(5)\n\tvisionRayPerPixelCount(6)\nMedianDenoiser\n")
    binary = os.path.join(os.path.dirname(swr.__file__), "lib", "RayTrace")
    exe = os.path.join(s["basepath"], "RayTrace")
    if not os.path.exists(exe):
        os.symlink(binary, exe)
    out = tmp_path / "out.ppm"
    p = subprocess.run([exe, str(rfile), s["scene"], str(W), str(H), s["camera"], str(out), "3"],
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert p.stdout.count("Render Time:") == 3 and "Render finished!" in p.stdout
    data = out.read_bytes()
    header = b"P6\n%d\n%d\n255\n" % (W, H)
    assert data.startswith(header)
    got = np.frombuffer(data[len(header):], np.uint8).reshape(H, W, 3)
    sd = swr.load_scene(s["scene"], s["basepath"])
    cam = swr.load_camera(s["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    _, img = O.rt_render(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, 6, 5)
    want = O.rt_denoise_median(img.reshape(H, W, 4))[..., :3]
    assert np.mean(np.all(got == want, axis=2)) > 0.97


def test_gpu_rt_on_a_terrain_matches_oracle(tmp_path):
    """A deep tree (a 256^2-cell terrain in 256 tiles, spheres, lights): ray-query hits on random
    rays and a small frame against the oracle."""
    s = scenes.terrain(6, str(tmp_path), cells=256, tile=16, spheres=16, sphere_subdiv=3, lights=3)
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(20000, sd.vpos.min(0) - 0.05, sd.vpos.max(0) + 0.05, seed=8)
    hits = rt.trace(sc, torch.from_numpy(ro).cuda(), torch.from_numpy(rd).cuda()).cpu().numpy().view(np.uint32)
    otri, ot = O.rt_trace(osc, ro, rd)
    assert np.array_equal(hits[:, 0], otri)
    m = otri != 0xFFFFFFFF
    assert np.array_equal(hits[m, 3], ot[m].view(np.uint32)) and m.mean() > 0.2
    W, H, spp, vj = 48, 27, 4, 5
    cam = swr.load_camera(s["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    rgb, rgba = rt.render(sc, cam, W, H, spp, vj)
    torch.cuda.synchronize()
    want_rgb, want_rgba = O.rt_render(osc, O.camera(vi, pi, org), W, H, spp, vj)
    assert _close(rgb.cpu().numpy().reshape(-1, 3), want_rgb)
    assert np.mean(np.all(rgba.cpu().numpy().reshape(-1, 4) == want_rgba, axis=1)) > 0.99
