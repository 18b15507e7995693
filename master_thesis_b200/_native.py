"""ctypes binding of the C ABI declared in include/swr.h (libswr.so, built in-tree).

The library is loaded from master_thesis_b200/lib/libswr.so. There is no fallback: if the
library is missing, importing the binding raises, so no code path can silently run without the
native kernels.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libswr.so")

SWR_OK = 0
SWR_ERR_IO = 1
SWR_ERR_PARSE = 2
SWR_ERR_ALLOC = 3
SWR_ERR_CUDA = 4
SWR_ERR_TIMEOUT = 5
SWR_ERR_INVALID = 6
SWR_ERR_UNSUPPORTED = 7
MODE_REFERENCE = 0
MODE_PHYSICAL = 1
RENDER_SAMPLES_OUT = 1
RENDER_PROFILE = 2
RENDER_COUNT = 4
RENDER_STATIC_FETCH = 8
RENDER_POSTPONE = 16
RENDER_ONE_WAVEFRONT = 32
RENDER_HOST_LOOP = 64


class SwrError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("swr error %d: %s" % (code, msg))
        self.code = code


class Material(ctypes.Structure):
    _fields_ = [("color", ctypes.c_float * 3), ("diffuse_t", ctypes.c_float),
                ("reflect_t", ctypes.c_float), ("transparent_t", ctypes.c_float),
                ("refraction_index", ctypes.c_float), ("light_source", ctypes.c_uint32),
                ("light_strength", ctypes.c_float)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("num_objects", ctypes.c_uint32), ("num_vertices", ctypes.c_uint32),
                ("num_triangles", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
                ("vertex_pos", ctypes.c_void_p), ("vertex_normal", ctypes.c_void_p),
                ("tri_vertices", ctypes.c_void_p), ("tri_object", ctypes.c_void_p),
                ("tri_rank", ctypes.c_void_p), ("object_first_vertex", ctypes.c_void_p),
                ("materials", ctypes.c_void_p), ("tri_albedo", ctypes.c_void_p)]


class BuildOpts(ctypes.Structure):
    _fields_ = [("sah_bins", ctypes.c_uint32), ("max_leaf", ctypes.c_uint32),
                ("threads", ctypes.c_uint32), ("leaf_cost_pct", ctypes.c_uint32),
                ("builder", ctypes.c_uint32), ("radius", ctypes.c_uint32), ("width", ctypes.c_uint32)]


BUILD_HOST = 0
BUILD_DEVICE = 1


class Camera(ctypes.Structure):
    _fields_ = [("view_inv", ctypes.c_float * 16), ("proj_inv", ctypes.c_float * 16),
                ("origin", ctypes.c_float * 3), ("reserved", ctypes.c_float)]


class RenderOpts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32),
                ("spp", ctypes.c_uint32), ("max_depth", ctypes.c_uint32),
                ("seed", ctypes.c_uint64), ("mode", ctypes.c_uint32),
                ("rr_depth", ctypes.c_uint32), ("rr_survive", ctypes.c_float),
                ("wave_size", ctypes.c_uint32), ("block_size", ctypes.c_uint32),
                ("flags", ctypes.c_uint32), ("refill", ctypes.c_uint32), ("trace_blocks", ctypes.c_uint32),
                ("shade_batch", ctypes.c_uint32), ("sample_begin", ctypes.c_uint32), ("spp_total", ctypes.c_uint32),
                ("pixel_begin", ctypes.c_uint32), ("pixel_count", ctypes.c_uint32)]


class RenderProfile(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ["rays", "bounce_rays", "node_visits", "tri_tests", "iterations",
                                               "launches", "trace_launches", "first_trace_rays", "h2d_bytes",
                                               "d2h_bytes"]] + \
               [(n, ctypes.c_double) for n in ["trace_ms", "shade_ms", "camera_ms", "resolve_ms"]]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class BatchJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("cam", Camera), ("opts", RenderOpts), ("rgb_out", ctypes.c_void_p)]


class BatchOpts(ctypes.Structure):
    _fields_ = [("wave_size", ctypes.c_uint32), ("refill", ctypes.c_uint32), ("flags", ctypes.c_uint32),
                ("shade_batch", ctypes.c_uint32)]


class BdptOpts(ctypes.Structure):
    _fields_ = [("light_jumps", ctypes.c_uint32), ("max_depth", ctypes.c_uint32), ("shade_batch", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32)]


class RendererParams(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("vision_jumps", ctypes.c_uint32), ("light_jumps", ctypes.c_uint32),
                ("max_depth", ctypes.c_uint32), ("spp", ctypes.c_uint32), ("reserved", ctypes.c_uint32 * 3)]


RENDERER_PATH_TRACER = 0
RENDERER_BIDIRECTIONAL = 1


class AdjointJob(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("cam", Camera), ("opts", RenderOpts), ("dl_dimage", ctypes.c_void_p),
                ("dl_dalbedo", ctypes.c_void_p), ("dl_demission", ctypes.c_void_p)]


BATCH_NO_GRAPH = 1


class ObjectTransform(ctypes.Structure):
    _fields_ = [("position", ctypes.c_float * 3), ("scale", ctypes.c_float * 3), ("rotation", ctypes.c_float * 4)]


class RtOpts(ctypes.Structure):
    _fields_ = [("width", ctypes.c_uint32), ("height", ctypes.c_uint32), ("vision_jumps", ctypes.c_uint32),
                ("spp", ctypes.c_uint32), ("refill", ctypes.c_uint32), ("shade_batch", ctypes.c_uint32),
                ("blocks_per_sm", ctypes.c_uint32), ("reserved", ctypes.c_uint32)]


DENOISER_GAUSS = 1
DENOISER_MEDIAN = 2
RT_MAX_DENOISERS = 8


class RtDenoiser(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_uint32), ("kernel_size", ctypes.c_uint32), ("sigma", ctypes.c_float),
                ("reserved", ctypes.c_uint32)]


class RtRendererParams(ctypes.Structure):
    _fields_ = [("vision_jumps", ctypes.c_uint32), ("spp", ctypes.c_uint32), ("num_denoisers", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("denoisers", RtDenoiser * RT_MAX_DENOISERS)]

P = ctypes.c_void_p
U32 = ctypes.c_uint32
U64 = ctypes.c_uint64
I = ctypes.c_int

# name -> (restype, argtypes); every function declared in include/swr.h
SIGNATURES = {
    "swr_last_error": (ctypes.c_char_p, []),
    "swr_abi_version": (I, []),
    "swr_sync": (I, [P]),
    "swr_host_scene_load": (I, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(P)]),
    "swr_host_scene_desc": (I, [P, ctypes.POINTER(SceneDesc)]),
    "swr_host_scene_ranks_exact": (I, [P]),
    "swr_host_scene_free": (None, [P]),
    "swr_camera_load": (I, [ctypes.c_char_p, U32, U32, U32, ctypes.POINTER(Camera)]),
    "swr_renderer_load": (I, [ctypes.c_char_p, ctypes.POINTER(U32), ctypes.POINTER(U32)]),
    "swr_camera_make": (I, [ctypes.POINTER(ctypes.c_float), ctypes.c_float, ctypes.c_float, ctypes.c_float, U32,
                            U32, ctypes.POINTER(Camera)]),
    "swr_scene_derive": (I, [ctypes.POINTER(SceneDesc), P, P, P, P, P]),
    "swr_scene_create": (I, [ctypes.POINTER(SceneDesc), ctypes.POINTER(BuildOpts), ctypes.POINTER(P)]),
    "swr_scene_destroy": (None, [P]),
    "swr_scene_stats": (I, [P, ctypes.POINTER(U64)]),
    "swr_trace_closest": (I, [P, P, P, U64, P, P]),
    "swr_trace_closest_stats": (I, [P, P, P, U64, P, P, P]),
    "swr_render": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), P, P, P]),
    "swr_render_profiled": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), P, P, P,
                                ctypes.POINTER(RenderProfile)]),
    "swr_render_noalloc": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), P, P, P]),
    "swr_batch_create": (I, [ctypes.POINTER(P)]),
    "swr_batch_destroy": (None, [P]),
    "swr_render_batch": (I, [P, ctypes.POINTER(BatchJob), U32, ctypes.POINTER(BatchOpts), P]),
    "swr_render_adjoint_batch": (I, [P, ctypes.POINTER(AdjointJob), U32, ctypes.POINTER(BatchOpts), P]),
    "swr_scene_set_albedo": (I, [P, P, P]),
    "swr_scene_set_emission": (I, [P, P, P]),
    "swr_render_adjoint": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), P, P, P, P]),
    "swr_render_adjoint_timed": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), P, P, P, P,
                                     ctypes.POINTER(ctypes.c_double)]),
    "swr_render_bdpt": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RenderOpts), ctypes.POINTER(BdptOpts), P, P, P]),
    "swr_renderer_load_params": (I, [ctypes.c_char_p, ctypes.POINTER(RendererParams)]),
    "swr_rotation_from_axis_angle": (I, [ctypes.POINTER(ctypes.c_float), ctypes.c_float,
                                         ctypes.POINTER(ctypes.c_float)]),
    "swr_host_scene_transforms": (I, [P, P]),
    "swr_scene_create_from_host": (I, [P, ctypes.POINTER(BuildOpts), ctypes.POINTER(P)]),
    "swr_scene_set_transforms": (I, [P, P, U32, P]),
    "swr_rt_trace_closest": (I, [P, P, P, U64, P, P]),
    "swr_rt_render": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RtOpts), P, P, P]),
    "swr_rt_gauss_weights": (I, [U32, ctypes.c_float, ctypes.POINTER(ctypes.c_float)]),
    "swr_rt_denoise_gauss": (I, [P, P, U32, U32, U32, ctypes.c_float, P]),
    "swr_rt_denoise_median": (I, [P, P, U32, U32, P]),
    "swr_rt_renderer_load": (I, [ctypes.c_char_p, ctypes.POINTER(RtRendererParams)]),
    "swr_rt_render_frame": (I, [P, ctypes.POINTER(Camera), ctypes.POINTER(RtOpts), ctypes.POINTER(RtDenoiser), U32,
                                P, P]),
    "swr_quantize_rgb8": (I, [P, U32, U32, P]),
    "swr_write_ppm": (I, [ctypes.c_char_p, P, U32, U32]),
    "swr_write_png": (I, [ctypes.c_char_p, P, U32, U32]),
}


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError("native library %s is missing: run `python -m master_thesis_b200.build`"
                          % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(rc):
    if rc != SWR_OK:
        raise SwrError(rc, lib.swr_last_error().decode(errors="replace"))
    return rc


def ptr(a):
    """Address of a numpy array or torch tensor (None -> NULL)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError("unsupported buffer type %r" % type(a))
