"""The allocation-free render entry point (swr_render_noalloc) against the regular one.

swr_render_noalloc is for callers that cannot let a library allocate device memory during a call
(applications that own all device memory through their own pool, frame loops that cannot absorb
the device-wide synchronisation of cudaMalloc/cudaFree). Its scratch is a fixed file-scope device
array, so its results must equal swr_render's, call after call, while the device's free memory
does not move. This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import _native as N
from master_thesis_b200 import scenes

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-7  # the radiance tolerance of the other render tests


def _noalloc(sc, cam, o, out, samples=None):
    stream = torch.cuda.current_stream().cuda_stream
    return N.lib.swr_render_noalloc(sc.handle, ctypes.byref(cam), ctypes.byref(o), out.data_ptr(),
                                    None if samples is None else samples.data_ptr(), stream)


@pytest.mark.parametrize("mode", [swr.MODE_REFERENCE, swr.MODE_PHYSICAL])
def test_noalloc_render_matches_render_twice(tmp_path, mode):
    s = scenes.cornell(5, str(tmp_path))
    sc = swr.Scene(swr.load_scene(s["scene"], s["basepath"]))
    # 2.95M samples: more than one chunk of the fixed scratch (2^21 sample slots)
    W, H, spp, depth = 192, 160, 96, 5
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=(mode == swr.MODE_PHYSICAL))
    rr = (3, 0.8) if mode == swr.MODE_PHYSICAL else (0, 1.0)
    ref = sc.render(cam, W, H, spp, depth, seed=11, mode=mode, rr_depth=rr[0], rr_survive=rr[1]).cpu().numpy()
    o = N.RenderOpts(W, H, spp, depth, 11, mode, rr[0], rr[1], 0, 0, 0, 0, 0, 0)
    out = torch.full((H, W, 3), -1.0, dtype=torch.float32, device="cuda")
    N.check(_noalloc(sc, cam, o, out))  # first call on the device: symbol lookup + module load
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        out.fill_(-1.0)
        N.check(_noalloc(sc, cam, o, out))
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.allclose(got, ref, rtol=RTOL, atol=ATOL)
    assert torch.cuda.mem_get_info()[0] == free0
    sc.close()


def test_noalloc_samples_and_limits(tmp_path):
    s = scenes.cornell(6, str(tmp_path))
    sc = swr.Scene(swr.load_scene(s["scene"], s["basepath"]))
    W, H, spp, depth = 40, 30, 8, 5
    cam = swr.load_camera(s["camera"], W, H)
    want = torch.zeros((H * W, spp, 4), dtype=torch.float32, device="cuda")
    ref = sc.render(cam, W, H, spp, depth, seed=3, samples=want)
    o = N.RenderOpts(W, H, spp, depth, 3, 0, 0, 1.0, 0, 0, N.RENDER_SAMPLES_OUT, 0, 0, 0)
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    got = torch.zeros_like(want)
    N.check(_noalloc(sc, cam, o, out, got))
    torch.cuda.synchronize()
    assert torch.equal(got[..., 3], want[..., 3])
    assert np.allclose(got.cpu().numpy(), want.cpu().numpy(), rtol=RTOL, atol=ATOL)
    assert np.allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=RTOL, atol=ATOL)
    # requests beyond the fixed scratch are refused with a clear error
    big = N.RenderOpts(W, H, spp, depth, 3, 0, 0, 1.0, 65537, 0, 0, 0, 0, 0)
    assert _noalloc(sc, cam, big, out) == N.SWR_ERR_UNSUPPORTED
    assert b"65536" in N.lib.swr_last_error()
    many = N.RenderOpts(1, 1, (1 << 21) + 1, depth, 3, 0, 0, 1.0, 0, 0, 0, 0, 0, 0)
    assert _noalloc(sc, cam, many, out) == N.SWR_ERR_UNSUPPORTED
    # a host output buffer would need staging through a device allocation
    host = np.zeros((H, W, 3), np.float32)
    rc = N.lib.swr_render_noalloc(sc.handle, ctypes.byref(cam), ctypes.byref(o), host.ctypes.data, None,
                                  torch.cuda.current_stream().cuda_stream)
    assert rc == N.SWR_ERR_INVALID
    sc.close()


def test_noalloc_samples_vs_oracle(tmp_path):
    """The allocation-free render against the oracle directly, per sample, over more samples than
    one chunk of its fixed scratch holds (2^21), so the chunk loop is checked too."""
    from oracle import oracle as O
    s = scenes.cornell(7, str(tmp_path))
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    W, H, spp, depth, seed = 160, 120, 128, 5, 21
    cam = swr.load_camera(s["camera"], W, H)
    o = N.RenderOpts(W, H, spp, depth, seed, 0, 0, 1.0, 0, 0, N.RENDER_SAMPLES_OUT, 0, 0, 0)
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    got = torch.zeros((H * W, spp, 4), dtype=torch.float32, device="cuda")
    N.check(_noalloc(sc, cam, o, out, got))
    torch.cuda.synchronize()
    vi, pi, org = swr.camera_arrays(cam)
    ps, pp = O.render_reference(O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org), W, H, spp, depth, seed)
    g = got.cpu().numpy()
    assert np.array_equal(g[..., 3], ps[..., 3])
    assert np.allclose(g[..., :3], ps[..., :3], rtol=RTOL, atol=ATOL)
    assert np.allclose(out.cpu().numpy().reshape(-1, 3), pp, rtol=RTOL, atol=ATOL)
    assert ps[..., 3].sum() > 0
    sc.close()
