"""GPU wavefront path tracer (swr_render, through the C ABI) against the reference's golden
radiance (Philox-shim runs of PathTracer::renderPixel) and the oracle."""
import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import scenes
from helpers import GOLDEN_CASES, golden, golden_camera, golden_scene, ref_pixel_from_samples
from oracle import oracle as O

pytestmark = pytest.mark.gpu

# Radiance tolerance: the kernels round every float operation like the reference; only the
# double-precision sin/cos/acos of the device libm and glibc may differ in the last bit of a
# double, which can move a float result by one ulp and then propagate.
RTOL = 1e-4


def _close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= RTOL * np.maximum(np.abs(b), 1e-6) + 1e-7)


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_gpu_reference_radiance_matches_golden(name):
    g = golden(name)
    sc = swr.Scene(golden_scene(g))
    W, H, spp, depth, seed = [int(x) for x in g["params"]]
    samples = torch.zeros((H * W, spp, 4), dtype=torch.float32, device="cuda")
    img = sc.render(golden_camera(g), W, H, spp, depth, seed=seed, samples=samples)
    torch.cuda.synchronize()
    ps = samples.cpu().numpy()
    want = g["per_sample"]
    assert np.array_equal(ps[..., 3], want[..., 3])  # same set of paths reach a light
    assert _close(ps[..., :3], want[..., :3])
    assert _close(img.cpu().numpy().reshape(-1, 3), g["per_pixel"])
    # bit-exactness is expected nearly everywhere
    assert np.mean(ps.view(np.uint32) == want.view(np.uint32)) > 0.999


@pytest.mark.parametrize("wave", [0, 4096])
def test_gpu_reference_render_larger_vs_oracle(tmp_path, wave):
    """More samples than one wave holds: injection, compaction and the in-order resolve."""
    s = scenes.cornell(8, str(tmp_path))
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    W, H, spp, depth = 40, 30, 16, 5
    cam = swr.load_camera(s["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    ps_o, pp_o = O.render_reference(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, spp, depth, 3)
    samples = np.zeros((H * W, spp, 4), np.float32)
    out = np.zeros((H, W, 3), np.float32)
    sc.render(cam, W, H, spp, depth, seed=3, wave_size=wave, out=out, samples=samples)  # host buffers
    assert np.array_equal(samples[..., 3], ps_o[..., 3])
    assert _close(samples[..., :3], ps_o[..., :3])
    assert _close(out.reshape(-1, 3), pp_o)


def test_gpu_physical_mode_matches_fp64(tmp_path):
    s = scenes.cornell(3, str(tmp_path))
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    W, H, spp = 32, 24, 64
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=True)
    vi, pi, org = swr.camera_arrays(cam)
    img = sc.render(cam, W, H, spp, 5, seed=9, mode=swr.MODE_PHYSICAL, rr_depth=3, rr_survive=0.8)
    torch.cuda.synchronize()
    pp64, var = O.render_physical64(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, spp, 5, 9,
                                    rr_depth=3, rr_q=0.8)
    m = img.cpu().numpy().reshape(-1, 3).astype(np.float64)
    # identical random numbers and hits: the estimates agree to float rounding
    assert np.max(np.abs(m - pp64) / (np.abs(pp64) + 1e-3)) < 1e-4


def test_gpu_render_invalid_args():
    g = golden("ref_white_room")
    sc = swr.Scene(golden_scene(g))
    with pytest.raises(swr.SwrError):
        sc.render(golden_camera(g), 8, 8, 1, 0)
    with pytest.raises(swr.SwrError):
        sc.render(golden_camera(g), 8, 8, 1, 40)


def test_gpu_converged_image_within_statistical_error_of_fp64(tmp_path):
    """A 256-spp GPU image against an independent 4096-spp FP64 host accumulation (other seed):
    per pixel and channel the difference must be consistent with the two estimates' standard
    errors (z-scores: mean square near 1, almost none beyond 4.5 sigma)."""
    s = scenes.cornell(5, str(tmp_path))
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    W, H, spp, hi = 24, 16, 256, 4096
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=True)
    vi, pi, org = swr.camera_arrays(cam)
    img = sc.render(cam, W, H, spp, 5, seed=1, mode=swr.MODE_PHYSICAL, rr_depth=3, rr_survive=0.8)
    torch.cuda.synchronize()
    m64, var64 = O.render_physical64(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, hi, 5, 2,
                                     rr_depth=3, rr_q=0.8)
    g = img.cpu().numpy().reshape(-1, 3).astype(np.float64)
    sigma2 = var64 * (hi / spp) + var64  # variance of the GPU mean + of the FP64 mean
    live = sigma2 > 0
    z = (g - m64)[live] / np.sqrt(sigma2[live])
    assert live.sum() > 0.5 * live.size
    assert 0.6 < float(np.mean(z ** 2)) < 1.5, float(np.mean(z ** 2))
    assert float(np.mean(np.abs(z) > 4.5)) < 2e-3
    assert np.all(np.abs(g - m64)[~live] < 1e-6)


def test_two_subwavefronts_equal_one_wavefront(tmp_path):
    """A chunk of 2^20 samples or more of a scene of 2^16 triangles or more runs as two concurrent
    sub-wavefronts on two streams; the image and every sample equal those of a single wavefront
    (SWR_RENDER_ONE_WAVEFRONT) and of the host-driven round loop (SWR_RENDER_HOST_LOOP)."""
    s = scenes.terrain(6, str(tmp_path), cells=192, tile=16, spheres=8, sphere_subdiv=2, lights=2)
    sd = swr.load_scene(s["scene"], s["basepath"])
    assert sd.num_triangles >= 1 << 16
    sc = swr.Scene(sd)
    W, H, spp, depth = 200, 150, 40, 6  # 1.2 M samples
    cam = swr.load_camera(s["camera"], W, H)
    import ctypes
    from master_thesis_b200 import _native as N
    outs = []
    for flags in (0, N.RENDER_ONE_WAVEFRONT, N.RENDER_HOST_LOOP):
        out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
        smp = torch.empty((H * W, spp, 4), dtype=torch.float32, device="cuda")
        o = N.RenderOpts(W, H, spp, depth, 5, 0, 0, 1.0, 1 << 16, 0, flags | N.RENDER_SAMPLES_OUT, 0, 0, 0)
        N.check(N.lib.swr_render(sc.handle, ctypes.byref(cam), ctypes.byref(o), out.data_ptr(), smp.data_ptr(),
                                 torch.cuda.current_stream().cuda_stream))
        torch.cuda.synchronize()
        outs.append((out.cpu().numpy(), smp.cpu().numpy()))
    for k in (1, 2):
        assert np.array_equal(outs[0][0], outs[k][0])
        assert np.array_equal(outs[0][1], outs[k][1])
    assert outs[0][0].max() > 0
    # and on a host output buffer, twice in a row (graphs and streams reused)
    for _ in range(2):
        host = np.zeros((H, W, 3), np.float32)
        sc.render(cam, W, H, spp, depth, seed=5, wave_size=1 << 16, out=host)
        assert np.array_equal(host, outs[0][0])
