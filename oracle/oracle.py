"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the oracle's C restatement (libswr_oracle.so).

The oracle takes world-space scene arrays (from a reference-harness dump, or from any scene
source whose arrays were checked against one) and answers closest-hit and radiance queries with
the reference's rules, independently of the product library."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libswr_oracle.so")


def _lib():
    if not os.path.exists(LIB):
        import subprocess
        subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    lib.swo_trace.argtypes = [P, P, P, ctypes.c_uint64, P, P, P, ctypes.c_int]
    lib.swo_render_reference.argtypes = [P, P] + [ctypes.c_uint32] * 4 + [ctypes.c_uint64] + \
        [ctypes.c_uint32] * 2 + [P, P, ctypes.c_int]
    lib.swo_render_physical64.argtypes = [P, P] + [ctypes.c_uint32] * 4 + [ctypes.c_uint64, ctypes.c_uint32,
                                                                           ctypes.c_double] + \
        [ctypes.c_uint32] * 2 + [P, P, ctypes.c_int]
    lib.swo_adjoint_physical64.argtypes = [P, P] + [ctypes.c_uint32] * 4 + [ctypes.c_uint64, ctypes.c_uint32,
                                                                            ctypes.c_double, P, P, P, ctypes.c_int]
    U = ctypes.c_uint32
    lib.swo_render_reference_part.argtypes = [P, P] + [U] * 6 + [ctypes.c_uint64] + [U] * 2 + [P, P, ctypes.c_int]
    lib.swo_render_physical64_part.argtypes = [P, P] + [U] * 6 + [ctypes.c_uint64, U, ctypes.c_double] + \
        [U] * 2 + [P, P, ctypes.c_int]
    lib.swo_adjoint_physical64_part.argtypes = [P, P] + [U] * 6 + [ctypes.c_uint64, U, ctypes.c_double, P, P, P,
                                                                     ctypes.c_int]
    lib.swo_render_bdpt.argtypes = [P, P] + [ctypes.c_uint32] * 6 + [ctypes.c_uint64] + [ctypes.c_uint32] * 2 + \
        [P, P, ctypes.c_int]
    lib.swo_render_bdpt.restype = ctypes.c_int
    lib.swo_rt_render.argtypes = [P, P] + [ctypes.c_uint32] * 6 + [P, P, ctypes.c_int]
    lib.swo_rt_trace.argtypes = [P, P, P, ctypes.c_uint64, P, P, ctypes.c_int]
    lib.swo_rt_gauss_weights.argtypes = [ctypes.c_uint32, ctypes.c_float, P]
    lib.swo_rt_gauss_weights.restype = ctypes.c_int
    lib.swo_rt_denoise_gauss.argtypes = [P, P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, P]
    lib.swo_rt_denoise_median.argtypes = [P, P, ctypes.c_uint32, ctypes.c_uint32]
    return lib


_L = None


def lib():
    global _L
    if _L is None:
        _L = _lib()
    return _L


class _Scene(ctypes.Structure):
    _fields_ = [("ntri", ctypes.c_uint32), ("nobj", ctypes.c_uint32)] + \
        [(n, ctypes.c_void_p) for n in ["v0", "e0", "e1", "den", "tri_box", "obj_box", "tri_obj",
                                        "obj_first", "visit", "nrm", "mats", "albedo", "emission", "vtx"]]


class _Camera(ctypes.Structure):
    _fields_ = [("vi", ctypes.c_float * 16), ("pi", ctypes.c_float * 16), ("org", ctypes.c_float * 3)]


def _p(a):
    return None if a is None else a.ctypes.data


def _threads():
    return max(1, os.cpu_count() or 1)


class OracleScene:
    """Arrays: v0/e0/e1 [n,3], den [n,4], tri_box [n,6], obj_box [m,6], tri_obj [n],
    rank [n] (visit order position), nrm [n,9] corner normals, mats [m,9]
    (color rgb, dT, rT, tT, eta, light, strength), optional albedo [n,3], emission [m,3],
    vtx [n,9] corner positions (needed by the bidirectional tracer's light sampling)."""

    def __init__(self, v0, e0, e1, den, tri_box, obj_box, tri_obj, rank, nrm, mats, albedo=None,
                 emission=None, vtx=None):
        f = lambda a, c: np.ascontiguousarray(a, dtype=np.float32).reshape(-1, c)
        self.v0, self.e0, self.e1 = f(v0, 3), f(e0, 3), f(e1, 3)
        self.den, self.tri_box, self.obj_box = f(den, 4), f(tri_box, 6), f(obj_box, 6)
        self.nrm, self.mats = f(nrm, 9), f(mats, 9)
        self.albedo = None if albedo is None else f(albedo, 3)
        self.emission = None if emission is None else f(emission, 3)
        self.vtx = None if vtx is None else f(vtx, 9)
        self.tri_obj = np.ascontiguousarray(tri_obj, dtype=np.uint32).reshape(-1)
        rank = np.asarray(rank, dtype=np.int64).reshape(-1)
        self.visit = np.ascontiguousarray(np.argsort(rank, kind="stable"), dtype=np.uint32)
        nobj = self.obj_box.shape[0]
        counts = np.bincount(self.tri_obj, minlength=nobj)
        self.obj_first = np.zeros(nobj + 1, np.uint32)
        self.obj_first[1:] = np.cumsum(counts)
        self._s = _Scene(self.v0.shape[0], nobj, *[_p(a) for a in (
            self.v0, self.e0, self.e1, self.den, self.tri_box, self.obj_box, self.tri_obj,
            self.obj_first, self.visit, self.nrm, self.mats, self.albedo, self.emission, self.vtx)])

    @staticmethod
    def from_scene_data(sd, albedo=None, emission=None):
        """From a master_thesis_b200.SceneData (its derived arrays come from the library's
        reference-exact derivation, which the tests check against the reference harness)."""
        dv = sd.derive()
        tri = sd.tri.astype(np.int64)
        nrm = sd.vnrm[tri].reshape(-1, 9)
        m = sd.materials
        mats = np.concatenate([m["color"], m["diffuse_t"][:, None], m["reflect_t"][:, None],
                               m["transparent_t"][:, None], m["refraction_index"][:, None],
                               m["light_source"][:, None].astype(np.float32),
                               m["light_strength"][:, None]], axis=1)
        rank = sd.tri_rank if sd.tri_rank is not None else np.arange(sd.num_triangles)
        return OracleScene(sd.vpos[tri[:, 0]], dv["e0"], dv["e1"], dv["den"], dv["tri_box"],
                           dv["obj_box"], sd.tri_obj, rank, nrm, mats,
                           albedo=albedo if albedo is not None else sd.tri_albedo, emission=emission,
                           vtx=sd.vpos[tri].reshape(-1, 9))

    @staticmethod
    def from_dump(R):
        """From a reference-harness dump (oracle/ref_harness dump)."""
        nt = R["tri_obj"].shape[0]
        ofs, nts = R["obj_first_tri"], R["obj_num_tris"]
        rank = np.zeros(nt, np.int64)
        tord = np.split(R["tri_order"].astype(np.int64), np.cumsum(nts)[:-1])
        base = 0
        for o in R["scene_order"]:
            rank[ofs[o] + tord[o]] = base + np.arange(nts[o])
            base += int(nts[o])
        tri = R["tri"].reshape(-1, 3).astype(np.int64)
        nrm = R["vnrm"].reshape(-1, 3)[tri].reshape(-1, 9)
        om = R["obj_mat"].reshape(-1, 8)  # color3 dT rT tT eta strength
        mats = np.concatenate([om[:, :7], R["obj_light"][:, None].astype(np.float32), om[:, 7:8]], axis=1)
        return OracleScene(R["tri_v0"], R["tri_e0"], R["tri_e1"], R["tri_den"], R["tri_box"],
                           R["obj_box"], R["tri_obj"], rank, nrm, mats,
                           vtx=R["vpos"].reshape(-1, 3)[tri].reshape(-1, 9))

    def trace(self, ro, rd, threads=None):
        ro = np.ascontiguousarray(ro, dtype=np.float32).reshape(-1, 4)
        rd = np.ascontiguousarray(rd, dtype=np.float32).reshape(-1, 4)
        n = ro.shape[0]
        tri = np.empty(n, np.uint32)
        d2 = np.empty(n, np.float32)
        t = np.empty(n, np.float32)
        lib().swo_trace(ctypes.byref(self._s), _p(ro), _p(rd), n, _p(tri), _p(d2), _p(t),
                        threads or _threads())
        return tri, d2, t


def camera(vi, pi, org):
    c = _Camera()
    c.vi[:] = np.asarray(vi, np.float32).reshape(-1).tolist()
    c.pi[:] = np.asarray(pi, np.float32).reshape(-1).tolist()
    c.org[:] = np.asarray(org, np.float32).reshape(-1).tolist()
    return c


def render_reference(sc, cam, W, H, spp, depth, seed, p0=0, p1=None, threads=None, samples=None):
    """Per-sample (r g b flag) [n, k, 4] and per-pixel [n, 3] radiance of pixels [p0, p1); with
    samples=(s0, s1) only those samples of each pixel (k = s1 - s0), per-pixel values scaled by the
    whole image's 2 pi / spp."""
    p1 = W * H if p1 is None else p1
    s0, s1 = (0, spp) if samples is None else samples
    n = p1 - p0
    ps = np.empty((n, s1 - s0, 4), np.float32)
    pp = np.empty((n, 3), np.float32)
    lib().swo_render_reference_part(ctypes.byref(sc._s), ctypes.byref(cam), W, H, spp, s0, s1, depth, seed, p0, p1,
                                    _p(ps), _p(pp), threads or _threads())
    return ps, pp


def render_bdpt(sc, cam, W, H, spp, vision_jumps, light_jumps, max_depth, seed, p0=0, p1=None, threads=None):
    """BidirectionalPathTracer: per-sample contributions [n, spp, 4] (before the 2 pi / spp scale)
    and per-pixel radiance [n, 3]."""
    p1 = W * H if p1 is None else p1
    n = p1 - p0
    ps = np.empty((n, spp, 4), np.float32)
    pp = np.empty((n, 3), np.float32)
    rc = lib().swo_render_bdpt(ctypes.byref(sc._s), ctypes.byref(cam), W, H, spp, vision_jumps, light_jumps,
                               max_depth, seed, p0, p1, _p(ps), _p(pp), threads or _threads())
    if rc != 0:
        raise ValueError("oracle BDPT: %s" % ("no light source" if rc == -2 else "bad arguments"))
    return ps, pp


def render_physical64(sc, cam, W, H, spp, depth, seed, rr_depth=0, rr_q=1.0, p0=0, p1=None, threads=None,
                      samples=None):
    """Physical-mode estimate per pixel in double (and the variance of the mean); with
    samples=(s0, s1) only those samples, weighted by the whole image's 1/spp (variance unused)."""
    p1 = W * H if p1 is None else p1
    s0, s1 = (0, spp) if samples is None else samples
    n = p1 - p0
    pp = np.empty((n, 3), np.float64)
    var = np.empty((n, 3), np.float64)
    lib().swo_render_physical64_part(ctypes.byref(sc._s), ctypes.byref(cam), W, H, spp, s0, s1, depth, seed,
                                     rr_depth, float(np.float32(rr_q)), p0, p1, _p(pp), _p(var),
                                     threads or _threads())
    return pp, var


def adjoint_physical64(sc, cam, W, H, spp, depth, seed, dl_dimg, rr_depth=0, rr_q=1.0, threads=None,
                       samples=None):
    """Gradient of sum(dl_dimg * image) w.r.t. albedo and emission in double; with samples=(s0, s1)
    only those samples' share (weights 1/spp of the whole image)."""
    dl = np.ascontiguousarray(dl_dimg, dtype=np.float32).reshape(-1, 3)
    s0, s1 = (0, spp) if samples is None else samples
    ga = np.empty((sc.v0.shape[0], 3), np.float64)
    ge = np.empty((sc.obj_box.shape[0], 3), np.float64)
    lib().swo_adjoint_physical64_part(ctypes.byref(sc._s), ctypes.byref(cam), W, H, spp, s0, s1, depth, seed,
                                      rr_depth, float(np.float32(rr_q)), _p(dl), _p(ga), _p(ge),
                                      threads or _threads())
    return ga, ge


def rt_render(sc, cam, W, H, spp, vision_jumps, p0=0, p1=None, threads=None):
    """The RayTrace program's PathTracer for pixels [p0, p1): finalColor [n, 3] and the stored
    rgba8 texels [n, 4]."""
    p1 = W * H if p1 is None else p1
    n = p1 - p0
    rgb = np.empty((n, 3), np.float32)
    rgba = np.empty((n, 4), np.uint8)
    lib().swo_rt_render(ctypes.byref(sc._s), ctypes.byref(cam), W, H, vision_jumps, spp, p0, p1, _p(rgb), _p(rgba),
                        threads or _threads())
    return rgb, rgba


def rt_trace(sc, ro, rd, threads=None):
    """traceRay's closest hit per ray: (triangle id or 0xFFFFFFFF, t)."""
    ro = np.ascontiguousarray(ro, dtype=np.float32).reshape(-1, 4)
    rd = np.ascontiguousarray(rd, dtype=np.float32).reshape(-1, 4)
    n = ro.shape[0]
    tri = np.empty(n, np.uint32)
    t = np.empty(n, np.float32)
    lib().swo_rt_trace(ctypes.byref(sc._s), _p(ro), _p(rd), n, _p(tri), _p(t), threads or _threads())
    return tri, t


def rt_gauss_weights(kernel_size, sigma):
    out = np.zeros(20, np.float32)
    if lib().swo_rt_gauss_weights(kernel_size, float(np.float32(sigma)), _p(out)) != 0:
        raise ValueError("GaussDenoiser kernel size must be odd and in 1..19")
    return out[:kernel_size]


def rt_denoise_gauss(img, kernel_size, sigma):
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape[:2]
    g = np.zeros(20, np.float32)
    g[:kernel_size] = rt_gauss_weights(kernel_size, sigma)
    out = np.empty_like(img)
    lib().swo_rt_denoise_gauss(_p(img), _p(out), w, h, kernel_size, _p(g))
    return out


def rt_denoise_median(img):
    img = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = img.shape[:2]
    out = np.empty_like(img)
    lib().swo_rt_denoise_median(_p(img), _p(out), w, h)
    return out
