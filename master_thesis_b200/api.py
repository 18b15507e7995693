"""Python tooling over the C ABI: world-space scene data, the device scene handle, closest-hit
queries and renders. Device buffers are torch tensors; host buffers are numpy arrays (the
library stages host memory itself, which is the end-to-end path the reference's callers see).
"""
import ctypes
import os

import numpy as np

from . import _native as N
from ._native import check, ptr

MAT_DTYPE = np.dtype([("color", "<f4", (3,)), ("diffuse_t", "<f4"), ("reflect_t", "<f4"),
                      ("transparent_t", "<f4"), ("refraction_index", "<f4"),
                      ("light_source", "<u4"), ("light_strength", "<f4")])
assert MAT_DTYPE.itemsize == ctypes.sizeof(N.Material)


class SceneData:
    """World-space scene in the layout of swr_scene_desc (numpy, host memory)."""

    def __init__(self, vpos, vnrm, tri, tri_obj, obj_first_vertex, materials, tri_rank=None,
                 tri_albedo=None, ranks_exact=True):
        self.vpos = np.ascontiguousarray(vpos, dtype=np.float32).reshape(-1, 3)
        self.vnrm = np.ascontiguousarray(vnrm, dtype=np.float32).reshape(-1, 3)
        self.tri = np.ascontiguousarray(tri, dtype=np.uint32).reshape(-1, 3)
        self.tri_obj = np.ascontiguousarray(tri_obj, dtype=np.uint32).reshape(-1)
        self.obj_first_vertex = np.ascontiguousarray(obj_first_vertex, dtype=np.uint32).reshape(-1)
        self.materials = np.ascontiguousarray(materials, dtype=MAT_DTYPE).reshape(-1)
        self.tri_rank = None if tri_rank is None else np.ascontiguousarray(tri_rank, dtype=np.uint32).reshape(-1)
        self.tri_albedo = None if tri_albedo is None else np.ascontiguousarray(tri_albedo, dtype=np.float32).reshape(-1, 3)
        self.ranks_exact = ranks_exact

    @property
    def num_triangles(self):
        return self.tri.shape[0]

    @property
    def num_objects(self):
        return self.materials.shape[0]

    def desc(self):
        d = N.SceneDesc()
        d.num_objects = self.num_objects
        d.num_vertices = self.vpos.shape[0]
        d.num_triangles = self.num_triangles
        d.vertex_pos = ptr(self.vpos)
        d.vertex_normal = ptr(self.vnrm)
        d.tri_vertices = ptr(self.tri)
        d.tri_object = ptr(self.tri_obj)
        d.tri_rank = ptr(self.tri_rank)
        d.object_first_vertex = ptr(self.obj_first_vertex)
        d.materials = ptr(self.materials)
        d.tri_albedo = ptr(self.tri_albedo)
        return d

    def derive(self):
        """Edges, dot products, triangle and object boxes as the reference computes them."""
        nt, no = self.num_triangles, self.num_objects
        out = dict(e0=np.empty((nt, 3), np.float32), e1=np.empty((nt, 3), np.float32),
                   den=np.empty((nt, 4), np.float32), tri_box=np.empty((nt, 6), np.float32),
                   obj_box=np.empty((no, 6), np.float32))
        d = self.desc()
        check(N.lib.swr_scene_derive(ctypes.byref(d), ptr(out["e0"]), ptr(out["e1"]),
                                     ptr(out["den"]), ptr(out["tri_box"]), ptr(out["obj_box"])))
        return out


def load_scene(scene_path, basepath):
    """Scene file -> SceneData through the library's MeshManager-equivalent loader."""
    h = ctypes.c_void_p()
    check(N.lib.swr_host_scene_load(os.fsencode(scene_path), os.fsencode(basepath), ctypes.byref(h)))
    try:
        return _scene_data(h)
    finally:
        N.lib.swr_host_scene_free(h)


def _scene_data(h):
    """SceneData copied out of a loaded host scene."""
    d = N.SceneDesc()
    check(N.lib.swr_host_scene_desc(h, ctypes.byref(d)))
    nv, nt, no = d.num_vertices, d.num_triangles, d.num_objects

    def arr(p, n, dt):
        return np.ctypeslib.as_array((dt * n).from_address(p)).copy()

    vpos = arr(d.vertex_pos, nv * 3, ctypes.c_float)
    vnrm = arr(d.vertex_normal, nv * 3, ctypes.c_float)
    tri = arr(d.tri_vertices, nt * 3, ctypes.c_uint32)
    tobj = arr(d.tri_object, nt, ctypes.c_uint32)
    rank = arr(d.tri_rank, nt, ctypes.c_uint32)
    ofv = arr(d.object_first_vertex, no + 1, ctypes.c_uint32)
    mats = np.frombuffer(ctypes.string_at(d.materials, no * MAT_DTYPE.itemsize), dtype=MAT_DTYPE).copy()
    exact = bool(N.lib.swr_host_scene_ranks_exact(h))
    return SceneData(vpos, vnrm, tri, tobj, ofv, mats, tri_rank=rank, ranks_exact=exact)


def rotation_from_axis_angle(axis, angle):
    """The quaternion (s, x, y, z) a scene file's rotation(x, y, z, angle) gives."""
    a = (ctypes.c_float * 3)(*[float(x) for x in axis])
    out = (ctypes.c_float * 4)()
    check(N.lib.swr_rotation_from_axis_angle(a, float(angle), out))
    return np.array(out[:], np.float32)


def load_camera(camera_path, width, height, use_fov_key=False):
    c = N.Camera()
    check(N.lib.swr_camera_load(os.fsencode(camera_path), width, height, 1 if use_fov_key else 0,
                                ctypes.byref(c)))
    return c


def make_camera(position, angle, width, height, fov_deg=0.0):
    """Camera from values, as a .camera file with position(...) angle(theta, phi) [fov(deg)]."""
    c = N.Camera()
    p = (ctypes.c_float * 3)(*[float(x) for x in position])
    check(N.lib.swr_camera_make(p, float(angle[0]), float(angle[1]), float(fov_deg), width, height, ctypes.byref(c)))
    return c


def camera_arrays(cam):
    return (np.array(cam.view_inv, np.float32).reshape(4, 4),
            np.array(cam.proj_inv, np.float32).reshape(4, 4),
            np.array(cam.origin, np.float32))


def load_renderer(renderer_path):
    depth, spp = ctypes.c_uint32(), ctypes.c_uint32()
    check(N.lib.swr_renderer_load(os.fsencode(renderer_path), ctypes.byref(depth), ctypes.byref(spp)))
    return depth.value, spp.value


def load_renderer_params(renderer_path):
    """Renderer file of either reference renderer: dict(kind "PathTracer" or
    "BidirectionalPathTracer", vision_jumps, light_jumps, max_depth, spp)."""
    r = N.RendererParams()
    check(N.lib.swr_renderer_load_params(os.fsencode(renderer_path), ctypes.byref(r)))
    return dict(kind="PathTracer" if r.kind == N.RENDERER_PATH_TRACER else "BidirectionalPathTracer",
                vision_jumps=r.vision_jumps, light_jumps=r.light_jumps, max_depth=r.max_depth, spp=r.spp)


def _stream_handle(stream):
    if stream is None:
        try:
            import torch
            if torch.cuda.is_available():
                return torch.cuda.current_stream().cuda_stream
        except ImportError:
            pass
        return None
    return getattr(stream, "cuda_stream", stream)


class Scene:
    """Device scene (wide BVH + triangle records) built from SceneData."""

    def __init__(self, data, sah_bins=0, max_leaf=0, threads=0, leaf_cost_pct=0, builder="host", radius=0,
                 width=0):
        """builder: "host" (binned SAH on the host) or "device" (clustering + collapse on the GPU);
        width: children per wide node (2..8, 0 = 8)."""
        self.data = data
        d = data.desc()
        b = {"host": N.BUILD_HOST, "device": N.BUILD_DEVICE}[builder]
        o = N.BuildOpts(sah_bins, max_leaf, threads, leaf_cost_pct, b, radius, width)
        self._h = ctypes.c_void_p()
        check(N.lib.swr_scene_create(ctypes.byref(d), ctypes.byref(o), ctypes.byref(self._h)))

    @classmethod
    def from_file(cls, scene_path, basepath, sah_bins=0, max_leaf=0, threads=0, leaf_cost_pct=0, builder="host",
                  radius=0, width=0):
        """Scene loaded from a scene file, keeping the object-space meshes on the device so that
        set_transforms() can move its objects."""
        h = ctypes.c_void_p()
        check(N.lib.swr_host_scene_load(os.fsencode(scene_path), os.fsencode(basepath), ctypes.byref(h)))
        self = cls.__new__(cls)
        try:
            self.data = _scene_data(h)
            no = self.data.num_objects
            xf = np.zeros((no, 10), np.float32)
            check(N.lib.swr_host_scene_transforms(h, ptr(xf)))
            b = {"host": N.BUILD_HOST, "device": N.BUILD_DEVICE}[builder]
            o = N.BuildOpts(sah_bins, max_leaf, threads, leaf_cost_pct, b, radius, width)
            self._h = ctypes.c_void_p()
            check(N.lib.swr_scene_create_from_host(h, ctypes.byref(o), ctypes.byref(self._h)))
            self._xf = xf
        finally:
            N.lib.swr_host_scene_free(h)
        return self

    def transforms(self):
        """Current object placements [num_objects, 10]: position xyz, scale xyz, rotation quaternion
        (s, x, y, z); a scene made from SceneData has none."""
        return None if getattr(self, "_xf", None) is None else self._xf.copy()

    def set_transforms(self, xf, stream=None):
        """Moves the objects of a scene made by from_file: xf [num_objects, 10] as transforms()."""
        xf = np.ascontiguousarray(xf, dtype=np.float32).reshape(-1, 10)
        check(N.lib.swr_scene_set_transforms(self._h, ptr(xf), xf.shape[0], _stream_handle(stream)))
        self._xf = xf.copy()

    def close(self):
        if getattr(self, "_h", None):
            N.lib.swr_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def stats(self):
        out = (ctypes.c_uint64 * 8)()
        check(N.lib.swr_scene_stats(self._h, out))
        keys = ["nodes", "depth", "node_bytes", "tri_bytes", "triangles", "objects", "node_size", "tri_size"]
        return dict(zip(keys, list(out)))

    def trace(self, ray_o, ray_d, out=None, counts=None, stream=None):
        """Closest hit per ray. ray_o/ray_d: (n,4) float32 (numpy = host, torch cuda = device).
        Returns (n,4) uint32-viewed hits (tri, obj, dist2 bits, t bits) of the same kind."""
        n = ray_o.shape[0]
        if out is None:
            if isinstance(ray_o, np.ndarray):
                out = np.empty((n, 4), np.uint32)
            else:
                import torch
                out = torch.empty((n, 4), dtype=torch.int32, device=ray_o.device)
        s = _stream_handle(stream)
        if counts is not None:
            check(N.lib.swr_trace_closest_stats(self._h, ptr(ray_o), ptr(ray_d), n, ptr(out), ptr(counts), s))
        else:
            check(N.lib.swr_trace_closest(self._h, ptr(ray_o), ptr(ray_d), n, ptr(out), s))
        return out

    def render(self, cam, width, height, spp, depth, seed=0, mode=N.MODE_REFERENCE, rr_depth=0,
               rr_survive=1.0, wave_size=0, block_size=0, out=None, samples=None, stream=None,
               profile=False, count=False, return_profile=False, static_fetch=False, refill=0,
               trace_blocks=0, sample_begin=0, spp_total=0, pixel_begin=0, pixel_count=0, host_loop=False):
        """Renders an image (height, width, 3) float32 into `out` (torch cuda tensor or numpy array;
        a numpy array makes the library stage the result through the device).

        host_loop: the host launches every shade/trace round (SWR_RENDER_HOST_LOOP) instead of a
        CUDA graph whose loop ends on the device, so that a profiler can capture single launches.

        Part of an image: samples [sample_begin, sample_begin + spp) of an image of spp_total
        samples per pixel (scaled by that image's 1/spp_total, so parts over a partition of the
        samples sum to the image), and/or pixels [pixel_begin, pixel_begin + pixel_count) in
        row-major order (out then holds (pixel_count, 3) floats, bit-identical to those pixels of
        the whole image)."""
        flags = (N.RENDER_SAMPLES_OUT if samples is not None else 0) | (N.RENDER_PROFILE if profile else 0) | \
            (N.RENDER_COUNT if count else 0) | (N.RENDER_STATIC_FETCH if static_fetch else 0) | \
            (N.RENDER_HOST_LOOP if host_loop else 0)
        o = N.RenderOpts(width, height, spp, depth, seed, mode, rr_depth, rr_survive, wave_size, block_size, flags,
                         refill, trace_blocks, 0, sample_begin, spp_total, pixel_begin, pixel_count)
        if out is None:
            import torch
            shape = (pixel_count or width * height - pixel_begin, 3) if (pixel_begin or pixel_count) else \
                (height, width, 3)
            out = torch.empty(shape, dtype=torch.float32, device="cuda")
        s = _stream_handle(stream)
        prof = N.RenderProfile()
        check(N.lib.swr_render_profiled(self._h, ctypes.byref(cam), ctypes.byref(o), ptr(out), ptr(samples),
                                        s, ctypes.byref(prof)))
        return (out, prof.as_dict()) if return_profile else out


def _scene_set_albedo(self, albedo, stream=None):
    """Per-triangle diffuse albedo [num_triangles, 3] (by triangle id) for the physical mode."""
    check(N.lib.swr_scene_set_albedo(self._h, ptr(albedo), _stream_handle(stream)))


def _scene_set_emission(self, emission, stream=None):
    """Per-object emitted radiance [num_objects, 3] (only light-source objects emit)."""
    check(N.lib.swr_scene_set_emission(self._h, ptr(emission), _stream_handle(stream)))


def _scene_render_adjoint(self, cam, width, height, spp, depth, dl_dimage, seed=0, rr_depth=0, rr_survive=1.0,
                          refill=0, stream=None, return_ms=False, shade_batch=0, sample_begin=0, spp_total=0):
    """Gradients (albedo [num_triangles,3], emission [num_objects,3]) of sum(dl_dimage * image) for
    the physical-mode image rendered with the same arguments (path replay). Device tensors. With a
    sample range (sample_begin, spp_total) the gradient covers those samples only, weighted by the
    whole image's 1/spp_total, so gradients over a partition of the samples sum to the image's."""
    import torch
    dl = dl_dimage.contiguous()
    ga = torch.empty((self.data.num_triangles, 3), dtype=torch.float32, device=dl.device)
    ge = torch.empty((self.data.num_objects, 3), dtype=torch.float32, device=dl.device)
    o = N.RenderOpts(width, height, spp, depth, seed, N.MODE_PHYSICAL, rr_depth, rr_survive, 0, 0, 0, refill, 0,
                     shade_batch, sample_begin, spp_total, 0, 0)
    ms = ctypes.c_double(0.0)
    check(N.lib.swr_render_adjoint_timed(self._h, ctypes.byref(cam), ctypes.byref(o), ptr(dl), ptr(ga), ptr(ge),
                                         _stream_handle(stream), ctypes.byref(ms) if return_ms else None))
    return (ga, ge, ms.value) if return_ms else (ga, ge)


def _scene_render_bdpt(self, cam, width, height, spp, vision_jumps, light_jumps, max_depth, seed=0, out=None,
                       samples=None, refill=0, shade_batch=0, blocks_per_sm=0, chunk=0, stream=None):
    """BidirectionalPathTracer image (height, width, 3) into `out` (torch cuda tensor or numpy
    array); `samples` (optional, (height*width, spp, 4)) receives the per-sample contributions."""
    flags = N.RENDER_SAMPLES_OUT if samples is not None else 0
    o = N.RenderOpts(width, height, spp, vision_jumps, seed, N.MODE_REFERENCE, 0, 1.0, chunk, 0, flags, refill, 0, 0)
    b = N.BdptOpts(light_jumps, max_depth, shade_batch, blocks_per_sm)
    if out is None:
        import torch
        out = torch.empty((height, width, 3), dtype=torch.float32, device="cuda")
    check(N.lib.swr_render_bdpt(self._h, ctypes.byref(cam), ctypes.byref(o), ctypes.byref(b), ptr(out), ptr(samples),
                                _stream_handle(stream)))
    return out


Scene.render_bdpt = _scene_render_bdpt
Scene.set_albedo = _scene_set_albedo
Scene.set_emission = _scene_set_emission
Scene.render_adjoint = _scene_render_adjoint


class Batch:
    """Batch context (shared wavefront buffers + captured CUDA graph), reused across calls."""

    def __init__(self):
        self._h = ctypes.c_void_p()
        check(N.lib.swr_batch_create(ctypes.byref(self._h)))

    def close(self):
        if getattr(self, "_h", None):
            N.lib.swr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, jobs, wave_size=0, refill=0, use_graph=True, stream=None):
        """jobs: list of dicts with scene, cam, width, height, spp, depth and optional seed, mode,
        rr_depth, rr_survive, out (torch cuda tensor [h, w, 3]). Returns the output tensors."""
        import torch
        arr = (N.BatchJob * len(jobs))()
        outs = []
        for k, j in enumerate(jobs):
            out = j.get("out")
            if out is None:
                out = torch.empty((j["height"], j["width"], 3), dtype=torch.float32, device="cuda")
            outs.append(out)
            arr[k].scene = j["scene"].handle
            arr[k].cam = j["cam"]
            arr[k].opts = N.RenderOpts(j["width"], j["height"], j["spp"], j["depth"], j.get("seed", 0),
                                       j.get("mode", N.MODE_REFERENCE), j.get("rr_depth", 0),
                                       j.get("rr_survive", 1.0), 0, 0, 0, 0, 0, 0)
            arr[k].rgb_out = out.data_ptr()
        o = N.BatchOpts(wave_size, refill, 0 if use_graph else N.BATCH_NO_GRAPH, 0)
        check(N.lib.swr_render_batch(self._h, arr, len(jobs), ctypes.byref(o), _stream_handle(stream)))
        return outs

    def render_adjoint(self, jobs, refill=0, stream=None, shade_batch=0):
        """Path-replay adjoint of many physical-mode jobs in one launch. jobs: dicts as for render
        plus dl_dimage (cuda tensor [h, w, 3]) and optionally grad_albedo / grad_emission (cuda
        tensors [num_triangles, 3] / [num_objects, 3]; jobs of one scene may share them and then
        add into them). Returns [(grad_albedo, grad_emission)] per job."""
        import torch
        arr = (N.AdjointJob * len(jobs))()
        keep, grads = [], []
        for k, j in enumerate(jobs):
            dl = j["dl_dimage"].contiguous()
            sd = j["scene"].data
            ga = j.get("grad_albedo")
            if ga is None:
                ga = torch.empty((sd.num_triangles, 3), dtype=torch.float32, device=dl.device)
            ge = j.get("grad_emission")
            if ge is None:
                ge = torch.empty((sd.num_objects, 3), dtype=torch.float32, device=dl.device)
            keep.append(dl)
            grads.append((ga, ge))
            arr[k].scene = j["scene"].handle
            arr[k].cam = j["cam"]
            arr[k].opts = N.RenderOpts(j["width"], j["height"], j["spp"], j["depth"], j.get("seed", 0), N.MODE_PHYSICAL,
                                       j.get("rr_depth", 0), j.get("rr_survive", 1.0), 0, 0, 0, 0, 0, 0)
            arr[k].dl_dimage = dl.data_ptr()
            arr[k].dl_dalbedo = ga.data_ptr()
            arr[k].dl_demission = ge.data_ptr()
        o = N.BatchOpts(0, refill, 0, shade_batch)
        check(N.lib.swr_render_adjoint_batch(self._h, arr, len(jobs), ctypes.byref(o), _stream_handle(stream)))
        return grads


def quantize_rgb8(img):
    img = np.ascontiguousarray(img, dtype=np.float32)
    h, w = img.shape[:2]
    out = np.empty((h, w, 3), np.uint8)
    check(N.lib.swr_quantize_rgb8(ptr(img), w, h, ptr(out)))
    return out


def write_ppm(path, rgb8):
    rgb8 = np.ascontiguousarray(rgb8, dtype=np.uint8)
    h, w = rgb8.shape[:2]
    check(N.lib.swr_write_ppm(os.fsencode(path), ptr(rgb8), w, h))


def write_png(path, rgb8):
    rgb8 = np.ascontiguousarray(rgb8, dtype=np.uint8)
    h, w = rgb8.shape[:2]
    check(N.lib.swr_write_png(os.fsencode(path), ptr(rgb8), w, h))
