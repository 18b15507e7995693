"""The Vulkan application's PathTracer and its denoisers (the reference's RayTrace program),
restated as CUDA kernels over a built Scene: Python tooling over the swr_rt_* entry points of
include/swr.h.

Images: float radiance (height, width, 3) and rgba8 texels (height, width, 4) uint8. Device
buffers are torch cuda tensors; numpy arrays are host buffers that the library stages itself.
"""
import ctypes
import os

import numpy as np

from . import _native as N
from ._native import check, ptr
from .api import _stream_handle

GAUSS = N.DENOISER_GAUSS
MEDIAN = N.DENOISER_MEDIAN


def _empty(shape, dtype, like=None):
    if isinstance(like, np.ndarray):
        return np.empty(shape, dtype)
    import torch
    tdt = {np.float32: torch.float32, np.uint8: torch.uint8, np.uint32: torch.int32}[dtype]
    return torch.empty(shape, dtype=tdt, device="cuda" if like is None else like.device)


def trace(scene, ray_o, ray_d, out=None, stream=None):
    """traceRay's closest hit (t in [0.001, 10000], ties to the lower triangle id) per ray.
    ray_o/ray_d: (n, 4) float32. Returns (n, 4) uint32-viewed hits (tri, obj, +inf bits, t bits)."""
    n = ray_o.shape[0]
    if out is None:
        out = _empty((n, 4), np.uint32, ray_o)
    check(N.lib.swr_rt_trace_closest(scene.handle, ptr(ray_o), ptr(ray_d), n, ptr(out), _stream_handle(stream)))
    return out


def render(scene, cam, width, height, spp, vision_jumps, rgb=None, rgba=None, want_rgb=True, want_rgba=True,
           refill=0, shade_batch=0, blocks_per_sm=0, stream=None):
    """One PathTracer frame: (finalColor (height, width, 3) float32, rgba8 (height, width, 4)
    uint8); either output may be switched off (None is returned for it)."""
    if want_rgb and rgb is None:
        rgb = _empty((height, width, 3), np.float32, rgba)
    if want_rgba and rgba is None:
        rgba = _empty((height, width, 4), np.uint8, rgb)
    o = N.RtOpts(width, height, vision_jumps, spp, refill, shade_batch, blocks_per_sm)
    check(N.lib.swr_rt_render(scene.handle, ctypes.byref(cam), ctypes.byref(o), ptr(rgb) if want_rgb else None,
                              ptr(rgba) if want_rgba else None, _stream_handle(stream)))
    return (rgb if want_rgb else None), (rgba if want_rgba else None)


def gauss_weights(kernel_size, sigma):
    """GaussDenoiser's normalised weights (kernel_size odd, 1..19)."""
    out = (ctypes.c_float * 20)()
    check(N.lib.swr_rt_gauss_weights(kernel_size, sigma, out))
    return np.array(out[:kernel_size], np.float32)


def _image_out(img, out):
    if out is None:
        out = _empty(tuple(img.shape), np.uint8, img)
    return out


def denoise_gauss(img, kernel_size, sigma, out=None, stream=None):
    """GaussDenoiser pass over an rgba8 image (height, width, 4)."""
    h, w = img.shape[:2]
    out = _image_out(img, out)
    check(N.lib.swr_rt_denoise_gauss(ptr(img), ptr(out), w, h, kernel_size, sigma, _stream_handle(stream)))
    return out


def denoise_median(img, out=None, stream=None):
    """MedianDenoiser pass over an rgba8 image (height, width, 4); texels outside count as 0."""
    h, w = img.shape[:2]
    out = _image_out(img, out)
    check(N.lib.swr_rt_denoise_median(ptr(img), ptr(out), w, h, _stream_handle(stream)))
    return out


def load_renderer(renderer_path):
    """RayTrace renderer file: dict(vision_jumps, spp, denoisers=[("GaussDenoiser", kernel_size,
    sigma) | ("MedianDenoiser",), ...])."""
    r = N.RtRendererParams()
    check(N.lib.swr_rt_renderer_load(os.fsencode(renderer_path), ctypes.byref(r)))
    dn = []
    for k in range(r.num_denoisers):
        d = r.denoisers[k]
        dn.append(("GaussDenoiser", d.kernel_size, d.sigma) if d.kind == GAUSS else ("MedianDenoiser",))
    return dict(vision_jumps=r.vision_jumps, spp=r.spp, denoisers=dn)


def _denoiser_array(denoisers):
    arr = (N.RtDenoiser * max(1, len(denoisers)))()
    for k, d in enumerate(denoisers):
        if d[0] == "GaussDenoiser":
            arr[k] = N.RtDenoiser(GAUSS, d[1], d[2], 0)
        elif d[0] == "MedianDenoiser":
            arr[k] = N.RtDenoiser(MEDIAN, 0, 0.0, 0)
        else:
            raise ValueError("unknown denoiser %r" % (d[0],))
    return arr


def render_frame(scene, cam, width, height, params, out=None, refill=0, shade_batch=0, blocks_per_sm=0,
                 stream=None):
    """GraphicsEngine::render for the PathTracer: the frame, then the denoisers of `params`
    (a load_renderer() dict) in order. Returns the final rgba8 image (height, width, 4)."""
    if out is None:
        out = _empty((height, width, 4), np.uint8)
    o = N.RtOpts(width, height, params["vision_jumps"], params["spp"], refill, shade_batch, blocks_per_sm)
    dn = params.get("denoisers", [])
    check(N.lib.swr_rt_render_frame(scene.handle, ctypes.byref(cam), ctypes.byref(o), _denoiser_array(dn), len(dn),
                                    ptr(out), _stream_handle(stream)))
    return out
