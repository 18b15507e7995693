"""Parts of one image (swr_render_opts pixel_begin/pixel_count and sample_begin/spp_total, through
the C ABI): pixel tiles must equal those pixels of a whole render bit for bit, sample ranges must
equal the oracle's samples of the same range, and parts over a partition must add up to the whole
image and its adjoint gradient. These are the units sharding.render_split / adjoint_split hand to
the GPUs of a multi-GPU job (one GPU here renders every rank's part in turn).

Reference: software_renderer/graphic/graphics_engine.cpp:49-56,73-74 (the image split over workers
by pixel), graphic/path_tracer.cpp:18-40 (a pixel's samples summed in order, times 2 pi / spp)."""
import ctypes

import numpy as np
import pytest
import torch

import master_thesis_b200 as swr
from master_thesis_b200 import _native as N
from master_thesis_b200 import scenes, sharding
from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL, ATOL = 1e-4, 1e-7  # radiance tolerance of the render tests
W, H, SPP, DEPTH, SEED = 64, 48, 12, 5, 19


@pytest.fixture(scope="module")
def cornell(tmp_path_factory):
    s = scenes.cornell(6, str(tmp_path_factory.mktemp("split")))
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    cam = swr.load_camera(s["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    return sd, sc, cam, O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org)


def _close(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= RTOL * np.maximum(np.abs(b), 1e-6) + ATOL)


@pytest.mark.parametrize("world", [1, 3, 7])
def test_pixel_tiles_equal_the_whole_image(cornell, world):
    sd, sc, cam, osc, ocam = cornell
    whole = sc.render(cam, W, H, SPP, DEPTH, seed=SEED).cpu().numpy().reshape(-1, 3)
    samples_whole = torch.zeros((H * W, SPP, 4), dtype=torch.float32, device="cuda")
    sc.render(cam, W, H, SPP, DEPTH, seed=SEED, samples=samples_whole)
    for r in range(world):
        lo, hi = sharding.shard(W * H, r, world)
        samples = torch.zeros((hi - lo, SPP, 4), dtype=torch.float32, device="cuda")
        tile = sc.render(cam, W, H, SPP, DEPTH, seed=SEED, pixel_begin=lo, pixel_count=hi - lo, samples=samples,
                         wave_size=4096)
        torch.cuda.synchronize()
        assert tile.shape == (hi - lo, 3)
        assert np.array_equal(tile.cpu().numpy(), whole[lo:hi])
        assert torch.equal(samples, samples_whole[lo:hi])


def test_pixel_tile_to_host_memory(cornell):
    sd, sc, cam, osc, ocam = cornell
    lo, n = 1000, 517
    out = np.zeros((n, 3), np.float32)
    sc.render(cam, W, H, SPP, DEPTH, seed=SEED, out=out, pixel_begin=lo, pixel_count=n)
    _, pp = O.render_reference(osc, ocam, W, H, SPP, DEPTH, SEED, lo, lo + n)
    assert _close(out, pp)


@pytest.mark.parametrize("mode", [swr.MODE_REFERENCE, swr.MODE_PHYSICAL])
def test_sample_ranges_match_oracle_and_sum_to_the_image(cornell, mode):
    sd, sc, cam, osc, ocam = cornell
    kw = dict(mode=mode, rr_depth=3, rr_survive=0.8) if mode else {}
    whole = sc.render(cam, W, H, SPP, DEPTH, seed=SEED, **kw).cpu().numpy().reshape(-1, 3).astype(np.float64)
    total = np.zeros_like(whole)
    for s0, s1 in [(0, 5), (5, 6), (6, 12)]:
        samples = torch.zeros((H * W, s1 - s0, 4), dtype=torch.float32, device="cuda")
        part = sc.render(cam, W, H, s1 - s0, DEPTH, seed=SEED, sample_begin=s0, spp_total=SPP,
                         samples=samples, **kw)
        torch.cuda.synchronize()
        part = part.cpu().numpy().reshape(-1, 3)
        if mode == swr.MODE_REFERENCE:
            ps, pp = O.render_reference(osc, ocam, W, H, SPP, DEPTH, SEED, samples=(s0, s1))
            got = samples.cpu().numpy()
            assert np.array_equal(got[..., 3], ps[..., 3])
            assert _close(got[..., :3], ps[..., :3])
            assert _close(part, pp)
        else:
            pp64, _ = O.render_physical64(osc, ocam, W, H, SPP, DEPTH, SEED, rr_depth=3, rr_q=0.8, samples=(s0, s1))
            assert np.max(np.abs(part - pp64) / (np.abs(pp64) + 1e-3)) < 1e-4
        total += part
    assert np.max(np.abs(total - whole) / (np.abs(whole) + 1e-3)) < 1e-5
    assert whole.max() > 0


def test_render_split_with_scene_parts_in_one_process(cornell):
    """sharding.render_split over this GPU's scene (no process group: one rank holds everything)."""
    sd, sc, cam, osc, ocam = cornell
    whole = sc.render(cam, W, H, SPP, DEPTH, seed=SEED)
    part = sharding.scene_part_renderer(sc, cam, W, H, SPP, DEPTH, seed=SEED)
    tiles = sharding.render_split(part, W, H, SPP, 0, 1, split="tiles", device="cuda")
    by_spp = sharding.render_split(part, W, H, SPP, 0, 1, split="spp", device="cuda")
    torch.cuda.synchronize()
    assert torch.equal(tiles, whole)
    assert torch.equal(by_spp, whole)


def test_adjoint_sample_ranges_sum_to_the_gradient(tmp_path):
    s = scenes.cornell_tessellated(2, str(tmp_path), wall_cells=6, box_cells=4)
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    w, h, spp = 32, 24, 10
    cam = swr.load_camera(s["camera"], w, h, use_fov_key=True)
    rng = np.random.default_rng(4)
    albedo = rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)
    sc.set_albedo(torch.from_numpy(albedo).cuda())
    dl = torch.from_numpy(rng.normal(size=(h, w, 3)).astype(np.float32)).cuda()
    ga1, ge1 = sc.render_adjoint(cam, w, h, spp, DEPTH, dl, seed=5, rr_depth=3, rr_survive=0.8)
    vi, pi, org = swr.camera_arrays(cam)
    osc = O.OracleScene.from_scene_data(sd, albedo=albedo)
    ga, ge = torch.zeros_like(ga1), torch.zeros_like(ge1)
    for s0, s1 in [(0, 3), (3, 10)]:
        pa, pe = sc.render_adjoint(cam, w, h, s1 - s0, DEPTH, dl, seed=5, rr_depth=3, rr_survive=0.8,
                                   sample_begin=s0, spp_total=spp)
        ra, re = O.adjoint_physical64(osc, O.camera(vi, pi, org), w, h, spp, DEPTH, 5, dl.cpu().numpy(), rr_depth=3,
                                      rr_q=0.8, samples=(s0, s1))
        pa64, pe64 = pa.cpu().numpy().astype(np.float64), pe.cpu().numpy().astype(np.float64)
        assert np.linalg.norm(pa64 - ra) <= 1e-4 * np.linalg.norm(ra)
        assert np.linalg.norm(pe64 - re) <= 1e-4 * np.linalg.norm(re)
        ga += pa
        ge += pe
    torch.cuda.synchronize()
    a, b = ga.cpu().numpy().astype(np.float64), ga1.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)
    a, b = ge.cpu().numpy().astype(np.float64), ge1.cpu().numpy().astype(np.float64)
    assert np.linalg.norm(a - b) <= 1e-5 * np.linalg.norm(b)


def test_bad_ranges_are_rejected(cornell):
    sd, sc, cam, osc, ocam = cornell
    with pytest.raises(swr.SwrError):
        sc.render(cam, W, H, 5, DEPTH, sample_begin=8, spp_total=12)  # 8 + 5 > 12
    with pytest.raises(swr.SwrError):
        sc.render(cam, W, H, SPP, DEPTH, pixel_begin=W * H - 10, pixel_count=11)
    with pytest.raises(swr.SwrError):
        sc.render(cam, W, H, SPP, DEPTH, pixel_begin=W * H, pixel_count=1)
    # whole images only: the bidirectional tracer, batches and the allocation-free render
    o = N.RenderOpts(W, H, SPP, 5, 1, 0, 0, 1.0, 0, 0, 0, 0, 0, 0, 0, 0, 16, 16)
    b = N.BdptOpts(5, 5, 0, 0)
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    assert N.lib.swr_render_bdpt(sc.handle, ctypes.byref(cam), ctypes.byref(o), ctypes.byref(b), out.data_ptr(),
                                 None, stream) == N.SWR_ERR_UNSUPPORTED
    assert N.lib.swr_render_noalloc(sc.handle, ctypes.byref(cam), ctypes.byref(o), out.data_ptr(), None,
                                    stream) == N.SWR_ERR_UNSUPPORTED
    batch = swr.Batch()
    arr = (N.BatchJob * 1)()
    arr[0].scene = sc.handle
    arr[0].cam = cam
    arr[0].opts = o
    arr[0].rgb_out = out.data_ptr()
    assert N.lib.swr_render_batch(batch._h, arr, 1, None, stream) == N.SWR_ERR_UNSUPPORTED
    batch.close()


def test_render_physical_split_one_rank_equals_render_physical(tmp_path):
    """The data-parallel autograd function with one rank holds the whole image and gradient."""
    from master_thesis_b200.diff import render_physical, render_physical_split
    s = scenes.cornell_tessellated(3, str(tmp_path), wall_cells=5, box_cells=3)
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    w, h, spp = 24, 16, 8
    cam = swr.load_camera(s["camera"], w, h, use_fov_key=True)
    rng = np.random.default_rng(6)
    alb = torch.from_numpy(rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)).cuda()
    em = torch.from_numpy((sd.materials["color"] * sd.materials["light_strength"][:, None]).astype(np.float32)).cuda()
    target = torch.from_numpy(rng.uniform(0, 0.3, (h, w, 3)).astype(np.float32)).cuda()
    grads = []
    for fn in (render_physical, render_physical_split):
        a = alb.clone().requires_grad_(True)
        e = em.clone().requires_grad_(True)
        img = fn(sc, cam, a, e, w, h, spp, DEPTH, seed=3, rr_depth=3, rr_survive=0.8)
        ((img - target) ** 2).sum().backward()
        grads.append((img.detach().cpu().numpy(), a.grad.cpu().numpy(), e.grad.cpu().numpy()))
    (i0, a0, e0), (i1, a1, e1) = grads
    assert np.array_equal(i0, i1)
    assert np.allclose(a1, a0, rtol=1e-5, atol=1e-7) and np.allclose(e1, e0, rtol=1e-5, atol=1e-7)
    assert np.abs(a0).max() > 0
