"""The RayTrace program's PathTracer and denoisers on the CPU: the oracle's restatement against
known answers and an independent float32 computation, the kernels' code (CPU twin) against the
oracle, the library's host helpers (renderer file, Gauss weights) against the reference's
formulas. The shaders themselves cannot run here (no graphics stack), so these pin the
restatement's own semantics."""
import math
import os

import numpy as np
import pytest

import master_thesis_b200 as swr
from master_thesis_b200 import rt, scenes
from master_thesis_b200.scenes import _entry, _layout, write_camera, write_obj
from helpers import GOLDEN_CASES, Twin, golden, golden_camera, golden_scene, rays_uniform
from oracle import oracle as O

PI_F = np.float32(3.1415926538)


def _planes_scene(root, planes, camera=((3.4, 0, 0), (1, 0))):
    """Quads in planes x = const (entries: x, normal sign, color, light strength or None,
    material keys), seen from a camera on the +x axis looking down -x."""
    base = _layout(root)
    write_obj(os.path.join(root, "res/obj/quad.obj"), *scenes.quad_mesh())
    s = ""
    for x, sign, color, light, extra in planes:
        kw = dict(color=color, scale=(1, 1000, 1000))
        if sign < 0:
            kw["rotation"] = (0, 1, 0, math.pi)
        if light is not None:
            kw["lightSource"] = light
        kw.update(extra)
        s += _entry("quad.obj", (x, 0, 0), **kw)
    path = os.path.join(root, "res/scene/planes.scene")
    with open(path, "w") as f:
        f.write(s)
    cam = os.path.join(root, "res/camera/planes.camera")
    write_camera(cam, *camera)
    return path, cam, base


def _oracle(scene_path, base, cam_path, W, H):
    sd = swr.load_scene(scene_path, base)
    cam = swr.load_camera(cam_path, W, H)
    vi, pi, org = swr.camera_arrays(cam)
    return sd, cam, O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org)


def test_rt_light_seen_directly_is_color_times_strength(tmp_path):
    sp, cp, base = _planes_scene(str(tmp_path), [(-1.0, 1, (0.5, 0.25, 1.0), 2.0, {})])
    _, _, osc, ocam = _oracle(sp, base, cp, 8, 6)
    rgb, rgba = O.rt_render(osc, ocam, 8, 6, 13, 5)
    assert np.all(rgb == np.float32([1.0, 0.5, 2.0]))
    # clamp, * 255, round half to even: 0.5 * 255 = 127.5 -> 128
    assert np.all(rgba == np.uint8([255, 128, 255, 0]))


def test_rt_back_face_retries_stop_after_four_traces(tmp_path):
    # five back-facing lights behind one another: traces 1-3 are retried, the fourth is kept
    planes = [(-1.0 - 0.5 * k, -1, (0.1 * (k + 1), 0.05, 0.02), 1.0, {}) for k in range(5)]
    sp, cp, base = _planes_scene(str(tmp_path), planes)
    _, _, osc, ocam = _oracle(sp, base, cp, 8, 6)
    rgb, _ = O.rt_render(osc, ocam, 8, 6, 4, 5)
    assert np.all(rgb == np.float32([0.4, 0.05, 0.02]))
    # fewer than four back faces and then nothing: a miss
    sp, cp, base = _planes_scene(str(tmp_path / "b"), planes[:2])
    _, _, osc, ocam = _oracle(sp, base, cp, 8, 6)
    rgb, rgba = O.rt_render(osc, ocam, 8, 6, 4, 5)
    assert np.all(rgb == 0) and np.all(rgba == 0)


def _lcg_draws(x, y, n):
    s = (625 + x * 7444 + y * 1045) % 21023
    out = []
    for _ in range(n):
        s = (6237 * s + 10697) % 21023
        out.append(np.float32(s) / np.float32(21023))
    return out


def test_rt_diffuse_bounce_matches_independent_float32_computation(tmp_path):
    """A diffuse wall facing the camera and a large light behind the camera facing the wall: every
    sample is one diffuse jump whose direction comes from the pixel's LCG draws; the sample counts
    when the jump reaches the light. Computed here draw by draw in float32."""
    cd = np.float32([0.8, 0.6, 0.4])
    cl = np.float32([0.9, 1.0, 0.7])
    strength = np.float32(1.5)
    planes = [(-1.0, 1, tuple(cd), None, {}), (3.5, -1, tuple(cl), float(strength), {"scale": (1, 1e6, 1e6)})]
    sp, cp, base = _planes_scene(str(tmp_path), planes)
    W, H, spp = 6, 4, 7
    _, _, osc, ocam = _oracle(sp, base, cp, W, H)
    rgb, _ = O.rt_render(osc, ocam, W, H, spp, 2)
    lc = cl * strength
    for y in range(H):
        for x in range(W):
            draws = _lcg_draws(x, y, 3 * spp)
            fin = np.zeros(3, np.float32)
            for s in range(spp):
                _, r1, r2 = draws[3 * s:3 * s + 3]
                theta = np.float32(np.float32(2.0) * PI_F) * r1
                u = np.float32(2.0) * r2 - np.float32(1.0)
                suu = np.sqrt(np.float32(1.0) - u * u)
                v = np.float32([suu * np.float32(math.cos(float(theta))), suu * np.float32(math.sin(float(theta))), u])
                if v[0] < 0:
                    v = -v
                if v[0] <= 0:
                    continue
                if 4.5 / float(v[0]) > 10000.0:  # beyond traceRay's tmax
                    continue
                col = (cd * v[0]).astype(np.float32) * lc
                fin = (fin + col).astype(np.float32)
            want = fin * np.float32(np.float32(2.0) * PI_F / np.float32(spp))
            got = rgb[y * W + x]
            assert np.allclose(got, want, rtol=1e-5, atol=1e-7), (x, y, got, want)


def test_rt_no_jumps_and_dark_scene_give_zero(tmp_path):
    sp, cp, base = _planes_scene(str(tmp_path), [(-1.0, 1, (0.8, 0.8, 0.8), None, {})])
    _, _, osc, ocam = _oracle(sp, base, cp, 6, 4)
    for vj in (0, 1, 5):
        rgb, rgba = O.rt_render(osc, ocam, 6, 4, 5, vj)
        assert np.all(rgb == 0) and np.all(rgba == 0)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_twin_rt_hits_match_oracle(name):
    g = golden(name)
    sd = golden_scene(g)
    tw = Twin(sd)
    osc = O.OracleScene.from_scene_data(sd)
    ro, rd = rays_uniform(4000, sd.vpos.min(0) - 0.3, sd.vpos.max(0) + 0.3, seed=5)
    # some origins on the surfaces themselves: the 0.001 lower bound decides
    ro[:500, :3] = g["ray_o"][:500, :3]
    tri, t = tw.rt_trace(ro, rd)
    otri, ot = O.rt_trace(osc, ro, rd)
    assert np.array_equal(tri, otri)
    assert np.array_equal(t[tri != 0xFFFFFFFF].view(np.uint32), ot[otri != 0xFFFFFFFF].view(np.uint32))


@pytest.mark.parametrize("name", ["ref_cornell_box_with_blocks_and_ball", "ref_white_room", "gen_cornell_3"])
def test_twin_rt_render_matches_oracle(name):
    g = golden(name)
    sd = golden_scene(g)
    tw = Twin(sd)
    cam = golden_camera(g)
    vi, pi, org = swr.camera_arrays(cam)
    osc = O.OracleScene.from_scene_data(sd)
    W, H, spp, vj = 16, 12, 13, 5
    got = tw.rt_render(cam, W, H, spp, vj)
    want, _ = O.rt_render(osc, O.camera(vi, pi, org), W, H, spp, vj)
    assert np.mean(np.all(got == want, axis=1)) > 0.99
    assert np.allclose(got, want, rtol=1e-4, atol=1e-6)
    assert np.any(want > 0)


@pytest.mark.parametrize("k,sigma", [(1, 1.0), (3, 0.5), (5, 1.0), (7, 2.5), (19, 4.0)])
def test_gauss_weights_follow_the_reference_formula(k, sigma):
    w = rt.gauss_weights(k, sigma)
    assert np.array_equal(w.view(np.uint32), O.rt_gauss_weights(k, sigma).view(np.uint32))
    # gauss_denoiser.cpp:31-46 in float: peak at i = k - 1, normalised by the float sum
    a = (np.arange(k, dtype=np.float32) - np.float32(k - 1)) ** 2
    r = np.exp((-a / (np.float32(2.0) * np.float32(sigma) * np.float32(sigma))).astype(np.float64)).astype(np.float32)
    s = np.float32(0.0)
    for x in r:
        s = np.float32(s + x)
    assert np.array_equal(w, r * (np.float32(1.0) / s))
    assert np.argmax(w) == k - 1


@pytest.mark.parametrize("k,sigma", [(0, 1.0), (2, 1.0), (21, 1.0), (5, 0.0), (5, -1.0)])
def test_gauss_weights_reject_sizes_the_shader_cannot_read(k, sigma):
    with pytest.raises(swr.SwrError):
        rt.gauss_weights(k, sigma)


def test_oracle_denoisers_known_answers():
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, (9, 11, 4), dtype=np.uint8)
    # a 1-tap Gauss kernel is the identity (byte / 255 * 1 * 1 stores back to the byte)
    assert np.array_equal(O.rt_denoise_gauss(img, 1, 1.0), img)
    # interior median = the per-channel median of the 3x3 block; outside texels count as 0
    P = np.pad(img, ((1, 1), (1, 1), (0, 0)))
    want = np.empty_like(img)
    for y in range(9):
        for x in range(11):
            want[y, x] = np.median(P[y:y + 3, x:x + 3].reshape(-1, 4), axis=0)
    assert np.array_equal(O.rt_denoise_median(img), want)
    # Gauss in float64 against the float32 restatement: within one unit of the last byte
    k, sigma = 5, 1.3
    g = O.rt_gauss_weights(k, sigma).astype(np.float64)
    off = k // 2
    f = img.astype(np.float64) / 255.0
    acc = np.zeros_like(f)
    for dx in range(-off, off + 1):
        for dy in range(-off, off + 1):
            sh = np.zeros_like(f)
            ys, xs = slice(max(0, -dy), 9 - max(0, dy)), slice(max(0, -dx), 11 - max(0, dx))
            yd, xd = slice(max(0, dy), 9 - max(0, -dy)), slice(max(0, dx), 11 - max(0, -dx))
            sh[ys, xs] = f[yd, xd]
            acc += sh * g[dx + off] * g[dy + off]
    want = np.clip(np.rint(np.clip(acc, 0, 1) * 255), 0, 255)
    assert np.max(np.abs(O.rt_denoise_gauss(img, k, sigma).astype(np.int64) - want)) <= 1


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)
    return str(path)


def test_rt_renderer_file(tmp_path):
    p = _write(tmp_path / "path_tracer.renderer",
               "PathTracer\n\tvisionJumpCount(5)\n\tvisionRayPerPixelCount(13)\n"
               "GaussDenoiser\n\tkernelSize(5)\n\tsigma(1.5)\nMedianDenoiser\n")
    r = rt.load_renderer(p)
    assert r == dict(vision_jumps=5, spp=13, denoisers=[("GaussDenoiser", 5, 1.5), ("MedianDenoiser",)])
    p = _write(tmp_path / "plain.renderer", "PathTracer\n\tvisionJumpCount(3)\n\tvisionRayPerPixelCount(2)\n")
    assert rt.load_renderer(p) == dict(vision_jumps=3, spp=2, denoisers=[])


def test_rt_renderer_file_errors(tmp_path):
    with pytest.raises(swr.SwrError, match="getRenderer not found"):
        rt.load_renderer(_write(tmp_path / "a.renderer", "Raymarcher\n\tvisionJumpCount(3)\n"))
    with pytest.raises(swr.SwrError) as e:
        rt.load_renderer(_write(tmp_path / "b.renderer", "Majercik2019\n"))
    assert e.value.code == 7
    with pytest.raises(swr.SwrError, match="getDenoiser not found"):
        rt.load_renderer(_write(tmp_path / "c.renderer",
                                "PathTracer\n\tvisionJumpCount(3)\n\tvisionRayPerPixelCount(2)\nBlur\n"))
    with pytest.raises(swr.SwrError, match="visionRayPerPixelCount"):
        rt.load_renderer(_write(tmp_path / "d.renderer", "PathTracer\n\tvisionJumpCount(3)\n\traysPerPixel(2)\n"))
    # the software renderer's reader keeps its own keys
    with pytest.raises(swr.SwrError):
        swr.load_renderer(_write(tmp_path / "e.renderer",
                                 "PathTracer\n\tvisionJumpCount(3)\n\tvisionRayPerPixelCount(2)\n"))
