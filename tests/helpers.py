"""Shared test helpers: seeded ray sets, the CPU twin of the kernels (test-only library), scene
fixtures."""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TWIN_SRC = os.path.join(ROOT, "tests", "native", "twin.cpp")
TWIN_SO = os.path.join(ROOT, "tests", "_build", "libswr_twin.so")
HOST_SRC = ["surface.cpp", "ref_bvh.cpp", "wide_bvh.cpp", "derive.cpp", "capi_host.cpp", "scene_pack.cpp"]


def rays_uniform(n, lo, hi, seed):
    """Origins uniform in the box [lo, hi], directions uniform on the sphere; (n,4) float32 each."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(lo, np.float64), np.asarray(hi, np.float64)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    ro = np.zeros((n, 4), np.float32)
    rd = np.zeros((n, 4), np.float32)
    ro[:, :3] = o
    rd[:, :3] = d
    return ro, rd


def build_twin():
    deps = [TWIN_SRC] + [os.path.join(ROOT, "master_thesis_b200/csrc/host", s) for s in HOST_SRC]
    for d, _, fs in os.walk(os.path.join(ROOT, "master_thesis_b200/csrc")):
        deps += [os.path.join(d, f) for f in fs if f.endswith((".h", ".cuh"))]
    if os.path.exists(TWIN_SO) and all(os.path.getmtime(TWIN_SO) >= os.path.getmtime(d) for d in deps):
        return TWIN_SO
    os.makedirs(os.path.dirname(TWIN_SO), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-I/usr/local/cuda/include",
           "-o", TWIN_SO, TWIN_SRC] + [os.path.join(ROOT, "master_thesis_b200/csrc/host", s) for s in HOST_SRC] + \
        ["-lpthread"]
    subprocess.run(cmd, check=True)
    return TWIN_SO


class Twin:
    """CPU build of the kernels' traversal and shading code over the packed scene records."""
    _lib = None

    def __init__(self, scene_data, sah_bins=0, max_leaf=0, width=0):
        if Twin._lib is None:
            L = ctypes.CDLL(build_twin())
            P = ctypes.c_void_p
            L.twin_create.restype = P
            L.twin_create.argtypes = [P, P]
            L.twin_destroy.argtypes = [P]
            L.twin_depth.argtypes = [P]
            L.twin_depth.restype = ctypes.c_uint32
            L.twin_nodes.argtypes = [P]
            L.twin_nodes.restype = ctypes.c_uint32
            L.twin_node_words.argtypes = [P, P]
            L.twin_node_words.restype = ctypes.c_uint32
            L.twin_trace.argtypes = [P, P, P, ctypes.c_uint64, P, P, P, P, ctypes.c_int]
            L.twin_render.argtypes = [P, P] + [ctypes.c_uint32] * 4 + [ctypes.c_uint64, ctypes.c_uint32,
                                                                        ctypes.c_uint32, ctypes.c_float,
                                                                        ctypes.c_uint32, ctypes.c_uint32, P]
            L.twin_rt_trace.argtypes = [P, P, P, ctypes.c_uint64, P, P]
            L.twin_rt_render.argtypes = [P, P] + [ctypes.c_uint32] * 6 + [P]
            Twin._lib = L
        from master_thesis_b200 import _native as N
        self._d = scene_data.desc()
        self._o = N.BuildOpts(sah_bins, max_leaf, 0, 0, 0, 0, width)
        self._h = Twin._lib.twin_create(ctypes.byref(self._d), ctypes.byref(self._o))
        if not self._h:
            Twin._lib.swr_last_error.restype = ctypes.c_char_p  # the twin keeps its own error
            raise RuntimeError("twin_create failed: " + Twin._lib.swr_last_error().decode())

    def __del__(self):
        if getattr(self, "_h", None):
            Twin._lib.twin_destroy(self._h)

    @property
    def depth(self):
        return Twin._lib.twin_depth(self._h)

    @property
    def num_nodes(self):
        return Twin._lib.twin_nodes(self._h)

    def node_words(self):
        """The compressed wide-BVH records, 20 words per node."""
        out = np.empty(Twin._lib.twin_node_words(self._h, None), np.uint32)
        Twin._lib.twin_node_words(self._h, out.ctypes.data)
        return out

    def trace(self, ro, rd, counts=False, postpone=False):
        n = ro.shape[0]
        tri = np.empty(n, np.uint32)
        d2 = np.empty(n, np.float32)
        t = np.empty(n, np.float32)
        c = np.empty((n, 2), np.uint32) if counts else None
        Twin._lib.twin_trace(self._h, ro.ctypes.data, rd.ctypes.data, n, tri.ctypes.data, d2.ctypes.data,
                             t.ctypes.data, None if c is None else c.ctypes.data, 1 if postpone else 0)
        return (tri, d2, t, c) if counts else (tri, d2, t)

    def render(self, cam, W, H, spp, depth, seed, mode=0, rr_depth=0, rr_q=1.0, p0=0, p1=None):
        p1 = W * H if p1 is None else p1
        out = np.empty((p1 - p0, spp, 4), np.float32)
        Twin._lib.twin_render(self._h, ctypes.byref(cam), W, H, spp, depth, seed, mode, rr_depth, rr_q,
                              p0, p1, out.ctypes.data)
        return out


    def rt_trace(self, ro, rd):
        n = ro.shape[0]
        tri = np.empty(n, np.uint32)
        t = np.empty(n, np.float32)
        Twin._lib.twin_rt_trace(self._h, ro.ctypes.data, rd.ctypes.data, n, tri.ctypes.data, t.ctypes.data)
        return tri, t

    def rt_render(self, cam, W, H, spp, vision_jumps, p0=0, p1=None):
        p1 = W * H if p1 is None else p1
        out = np.empty((p1 - p0, 3), np.float32)
        Twin._lib.twin_rt_render(self._h, ctypes.byref(cam), W, H, vision_jumps, spp, p0, p1, out.ctypes.data)
        return out


def ref_pixel_from_samples(ps, spp):
    """The reference's per-pixel value from per-sample slots: float sum in sample order of the lit
    samples, times 2*pi*(1/spp) taken in double (path_tracer.cpp:28-37)."""
    n = ps.shape[0]
    acc = np.zeros((n, 3), np.float32)
    for s in range(spp):
        lit = ps[:, s, 3] != 0
        acc[lit] = (acc[lit] + ps[lit, s, :3]).astype(np.float32)
    sc = 2.0 * np.pi * float(np.float32(1.0) / np.float32(spp))
    return (acc.astype(np.float64) * sc).astype(np.float32)


GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["ref_cornell_box_with_blocks", "ref_cornell_box_with_ball", "ref_cornell_box_with_blocks_and_ball",
                "ref_cornell_box_5", "ref_white_room", "gen_cornell_3"]


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_scene(g):
    """SceneData built from a golden fixture's reference world data."""
    from master_thesis_b200 import MAT_DTYPE, SceneData
    no = g["mat_color"].shape[0]
    mats = np.zeros(no, MAT_DTYPE)
    mats["color"] = g["mat_color"]
    mats["diffuse_t"] = g["mat_thresholds"][:, 0]
    mats["reflect_t"] = g["mat_thresholds"][:, 1]
    mats["transparent_t"] = g["mat_thresholds"][:, 2]
    mats["refraction_index"] = g["mat_eta"]
    mats["light_source"] = g["mat_light"]
    mats["light_strength"] = g["mat_strength"]
    return SceneData(g["vpos"], g["vnrm"], g["tri"], g["tri_obj"], g["obj_first_vertex"], mats,
                     tri_rank=g["tri_rank"])


def golden_camera(g):
    from master_thesis_b200 import _native as N
    c = N.Camera()
    c.view_inv[:] = g["cam_view_inv"].reshape(-1).tolist()
    c.proj_inv[:] = g["cam_proj_inv"].reshape(-1).tolist()
    c.origin[:] = g["cam_origin"].reshape(-1).tolist()
    return c


def grid_mesh_scene(root, cells=160):
    """One OBJ mesh: a flat grid of cells x cells squares (2 * cells^2 triangles) in the y = 0
    plane with dyadic coordinates (x, z = (i - cells/2) / 64), so that rays straight down onto its
    edges and vertices hit several triangles at exactly the same squared distance (ties). Plus an
    emissive quad above it. Returns (scene path, basepath)."""
    from master_thesis_b200 import scenes
    base = scenes._layout(root)
    g = cells + 1
    c = (np.arange(g, dtype=np.float64) - cells / 2) / 64.0
    zz, xx = np.meshgrid(c, c, indexing="ij")
    pos = np.stack([xx, np.zeros_like(xx), zz], -1).reshape(-1, 3)
    nrm = np.tile([0.0, 1.0, 0.0], (g * g, 1))
    faces = []
    for r in range(cells):
        for q in range(cells):
            a = r * g + q
            faces += [(a, a + g, a + 1), (a + 1, a + g, a + g + 1)]
    scenes.write_obj(os.path.join(root, "res/obj/grid.obj"), pos, nrm, faces)
    scenes.write_obj(os.path.join(root, "res/obj/quad.obj"), *scenes.quad_mesh())
    path = os.path.join(root, "res/scene/grid.scene")
    with open(path, "w") as f:
        f.write(scenes._entry("grid.obj", (0, 0, 0), color=(0.7, 0.7, 0.7)))
        f.write(scenes._entry("quad.obj", (0, 1.5, 0), scale=(0.3, 0.3, 0.3), rotation=(0, 0, 1, -np.pi / 2),
                              color=(1, 1, 1), lightSource=10.0))
    return path, base


def rays_down_onto_grid_lines(n, cells, seed):
    """Rays straight down from y = 1 onto points of the grid's edges (a coordinate on a grid line)
    and vertices (both), all inside the grid."""
    rng = np.random.default_rng(seed)
    half = cells // 2
    i = rng.integers(-half + 1, half, (n, 2)).astype(np.float64) / 64.0
    f = rng.integers(0, 64, (n, 2)).astype(np.float64) / 4096.0  # dyadic offsets inside a cell
    kind = rng.integers(0, 3, n)  # 0: on an x line, 1: on a z line, 2: on a vertex
    x = i[:, 0] + np.where(kind == 1, f[:, 0], 0.0)
    z = i[:, 1] + np.where(kind == 0, f[:, 1], 0.0)
    ro = np.zeros((n, 4), np.float32)
    rd = np.zeros((n, 4), np.float32)
    ro[:, 0], ro[:, 1], ro[:, 2] = x, 1.0, z
    rd[:, 1] = -1.0
    return ro, rd
