"""Seeded synthetic scenes written in the reference's file formats.

Each generator writes OBJ meshes, a .scene file and a .camera file under a root directory laid
out like the reference tree (root/res/obj, root/res/scene, root/res/camera) and returns the paths
plus the basepath to pass to the loaders (root/bin/, so that basepath + "../res/obj/" resolves as
in the reference). The same files therefore load in the reference's SoftwareRenderer and here.

Scenes (shapes and sizes of the benchmark configurations):
  cornell(seed)  closed box of 5 quad walls (10 tris), 2 boxes rotated about y by seeded angles in
                 [0, 30 deg] (24 tris), a ceiling light quad (2 tris, lightSource(15), color 1);
                 Lambertian albedo per wall uniform in [0.1, 0.9]^3; camera fov(40).
  terrain(seed)  N x N heightfield cells (2 tris each; heights from seeded 6-octave fBm in
                 [0, 0.2]) split into OBJ tiles, icospheres of subdivision 4 with log-uniform radii
                 in [0.01, 0.1] and albedo in [0.1, 0.9]^3, and emissive quads.
"""
import functools
import math
import os

import numpy as np


def _fmt(x):
    return "%.9g" % float(np.float32(x))


def write_obj(path, pos, nrm, faces):
    """faces: (k, 3) zero-based vertex indices; every corner uses its vertex's normal."""
    pos = np.asarray(pos, np.float32)
    nrm = np.asarray(nrm, np.float32)
    lines = ["# generated"]
    lines += ["v %s %s %s" % (_fmt(p[0]), _fmt(p[1]), _fmt(p[2])) for p in pos]
    lines += ["vn %s %s %s" % (_fmt(n[0]), _fmt(n[1]), _fmt(n[2])) for n in nrm]
    f = np.asarray(faces, np.int64) + 1
    lines += ["f %d//%d %d//%d %d//%d" % (a, a, b, b, c, c) for a, b, c in f]
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def quad_mesh():
    """Unit square in the plane x = 0, y and z in [-1, 1], normal +x (two triangles)."""
    pos = [(0, -1, -1), (0, 1, -1), (0, 1, 1), (0, -1, 1)]
    nrm = [(1, 0, 0)] * 4
    faces = [(0, 1, 2), (0, 2, 3)]
    return pos, nrm, faces


def cube_mesh():
    """Cube [-1, 1]^3 with flat outward normals (24 vertices, 12 triangles)."""
    pos, nrm, faces = [], [], []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            n = [0.0, 0.0, 0.0]
            n[axis] = sgn
            u, v = [(axis + 1) % 3, (axis + 2) % 3]
            base = len(pos)
            for a, b in ((-1, -1), (1, -1), (1, 1), (-1, 1)):
                p = [0.0, 0.0, 0.0]
                p[axis] = sgn
                p[u] = a
                p[v] = b
                pos.append(tuple(p))
                nrm.append(tuple(n))
            if sgn > 0:
                faces += [(base, base + 1, base + 2), (base, base + 2, base + 3)]
            else:
                faces += [(base, base + 2, base + 1), (base, base + 3, base + 2)]
    return pos, nrm, faces


def icosphere_mesh(subdiv):
    pos, nrm, faces = _icosphere(subdiv)
    return pos.copy(), nrm.copy(), list(faces)


@functools.lru_cache(maxsize=None)
def _icosphere(subdiv):
    t = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t),
             (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(v, np.float64) / np.linalg.norm(v) for v in verts]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(subdiv):
        cache = {}
        nf = []

        def mid(a, b):
            k = (min(a, b), max(a, b))
            if k not in cache:
                m = verts[a] + verts[b]
                verts.append(m / np.linalg.norm(m))
                cache[k] = len(verts) - 1
            return cache[k]
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    pos = np.array(verts, np.float32)
    return pos, pos.copy(), tuple(faces)


def _layout(root):
    for d in ("res/obj", "res/scene", "res/camera", "bin"):
        os.makedirs(os.path.join(root, d), exist_ok=True)
    return os.path.join(root, "bin") + "/"


def _entry(name, position, **kw):
    s = "%s\n\tposition(%s, %s, %s)\n" % (name, _fmt(position[0]), _fmt(position[1]), _fmt(position[2]))
    for k, v in kw.items():
        s += "\t%s(%s)\n" % (k, ", ".join(_fmt(x) for x in np.atleast_1d(v)))
    return s + "\n"


def write_camera(path, position, angle, fov=None):
    s = "Camera\n\tposition(%s, %s, %s)\n\tangle(%s, %s)\n" % tuple(_fmt(x) for x in (*position, *angle))
    if fov is not None:
        s += "\tfov(%s)\n" % _fmt(fov)
    with open(path, "w") as f:
        f.write(s)


def cornell(seed, root):
    """Cornell-style scene (36 triangles). Returns dict(scene, camera, basepath)."""
    rng = np.random.default_rng(seed)
    base = _layout(root)
    write_obj(os.path.join(root, "res/obj/quad.obj"), *quad_mesh())
    write_obj(os.path.join(root, "res/obj/cube.obj"), *cube_mesh())
    hp = math.pi / 2
    walls = [((-1, 0, 0), None), ((0, -1, 0), (0, 0, 1, hp)), ((0, 1, 0), (0, 0, 1, -hp)),
             ((0, 0, -1), (0, 1, 0, -hp)), ((0, 0, 1), (0, 1, 0, hp))]
    s = ""
    for pos, rot in walls:
        kw = dict(color=rng.uniform(0.1, 0.9, 3))
        if rot is not None:
            kw["rotation"] = rot
        s += _entry("quad.obj", pos, **kw)
    s += _entry("quad.obj", (0, 0.99, 0), scale=(0.25, 0.25, 0.25), rotation=(0, 0, 1, -hp),
                color=(1, 1, 1), lightSource=15.0)
    for pos, sc in (((0.4, -0.7, -0.4), (0.3, 0.3, 0.3)), ((-0.4, -0.4, 0.4), (0.3, 0.6, 0.3))):
        ang = math.radians(rng.uniform(0.0, 30.0))
        s += _entry("cube.obj", pos, scale=sc, rotation=(0, 1, 0, ang), color=rng.uniform(0.1, 0.9, 3))
    scene = os.path.join(root, "res/scene/cornell_%d.scene" % seed)
    with open(scene, "w") as f:
        f.write(s)
    cam = os.path.join(root, "res/camera/cornell.camera")
    write_camera(cam, (3.4, 0, 0), (1, 0), fov=40)
    return dict(scene=scene, camera=cam, basepath=base)


def grid_quad_mesh(n):
    """The unit square of quad_mesh (plane x = 0, y and z in [-1, 1], normal +x) as an n x n grid of
    cells, two triangles each."""
    t = np.linspace(-1.0, 1.0, n + 1)
    zz, yy = np.meshgrid(t, t, indexing="ij")
    pos = np.stack([np.zeros_like(yy), yy, zz], -1).reshape(-1, 3)
    nrm = np.tile([1.0, 0.0, 0.0], (pos.shape[0], 1))
    faces = []
    for i in range(n):
        for j in range(n):
            a = i * (n + 1) + j
            faces += [(a, a + 1, a + n + 2), (a, a + n + 2, a + n + 1)]
    return pos, nrm, faces


def grid_cube_mesh(m):
    """Cube [-1, 1]^3 with every face an m x m grid (flat outward normals)."""
    pos, nrm, faces = [], [], []
    t = np.linspace(-1.0, 1.0, m + 1)
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            u, v = (axis + 1) % 3, (axis + 2) % 3
            base = len(pos)
            for i in range(m + 1):
                for j in range(m + 1):
                    p = [0.0, 0.0, 0.0]
                    p[axis] = sgn
                    p[u] = t[i]
                    p[v] = t[j]
                    n = [0.0, 0.0, 0.0]
                    n[axis] = sgn
                    pos.append(p)
                    nrm.append(n)
            for i in range(m):
                for j in range(m):
                    a = base + i * (m + 1) + j
                    b, c, d = a + m + 1, a + m + 2, a + 1
                    faces += [(a, b, c), (a, c, d)] if sgn > 0 else [(a, c, b), (a, d, c)]
    return pos, nrm, faces


def cornell_tessellated(seed, root, wall_cells=48, box_cells=33):
    """Cornell-style scene with tessellated walls and boxes (about 49k triangles with the defaults)
    and two emissive ceiling quads; for the differentiable configuration. Returns dict(scene,
    camera, basepath, triangles)."""
    rng = np.random.default_rng(seed)
    base = _layout(root)
    write_obj(os.path.join(root, "res/obj/wall.obj"), *grid_quad_mesh(wall_cells))
    write_obj(os.path.join(root, "res/obj/box.obj"), *grid_cube_mesh(box_cells))
    write_obj(os.path.join(root, "res/obj/quad.obj"), *quad_mesh())
    hp = math.pi / 2
    walls = [((-1, 0, 0), None), ((0, -1, 0), (0, 0, 1, hp)), ((0, 1, 0), (0, 0, 1, -hp)),
             ((0, 0, -1), (0, 1, 0, -hp)), ((0, 0, 1), (0, 1, 0, hp))]
    s = ""
    for pos, rot in walls:
        kw = dict(color=(0.7, 0.7, 0.7))
        if rot is not None:
            kw["rotation"] = rot
        s += _entry("wall.obj", pos, **kw)
    for z in (-0.35, 0.35):
        s += _entry("quad.obj", (0.1, 0.99, z), scale=(0.15, 0.15, 0.15), rotation=(0, 0, 1, -hp),
                    color=(1, 1, 1), lightSource=8.0)
    for pos, sc in (((0.4, -0.7, -0.4), (0.3, 0.3, 0.3)), ((-0.4, -0.4, 0.4), (0.3, 0.6, 0.3))):
        ang = math.radians(rng.uniform(0.0, 30.0))
        s += _entry("box.obj", pos, scale=sc, rotation=(0, 1, 0, ang), color=(0.7, 0.7, 0.7))
    scene = os.path.join(root, "res/scene/cornell_tess_%d.scene" % seed)
    with open(scene, "w") as f:
        f.write(s)
    cam = os.path.join(root, "res/camera/cornell.camera")
    write_camera(cam, (3.4, 0, 0), (1, 0), fov=40)
    ntri = 5 * 2 * wall_cells ** 2 + 2 * 12 * box_cells ** 2 + 4
    return dict(scene=scene, camera=cam, basepath=base, triangles=ntri)


def _vertex_normals(pos, faces):
    p = np.asarray(pos, np.float64)
    f = np.asarray(faces, np.int64)
    fn = np.cross(p[f[:, 1]] - p[f[:, 0]], p[f[:, 2]] - p[f[:, 0]])
    n = np.zeros_like(p)
    for k in range(3):
        np.add.at(n, f[:, k], fn)
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    return n


def random_scene(seed, target_tris):
    """World-space scene of about target_tris triangles built in memory: a ground quad, an emissive
    quad above, and seeded displaced icospheres and stacks of boxes. Returns (SceneData, camera
    dict(position, angle)) for the batched configuration."""
    from .api import MAT_DTYPE, SceneData
    rng = np.random.default_rng(seed)
    objs = []  # (pos, nrm, faces, albedo, light_strength)
    g = 4.0
    objs.append((np.array([(-g, 0, -g), (g, 0, -g), (g, 0, g), (-g, 0, g)], np.float64),
                 np.tile([0.0, 1.0, 0.0], (4, 1)), [(0, 2, 1), (0, 3, 2)], rng.uniform(0.3, 0.8, 3), 0.0))
    objs.append((np.array([(-0.6, 2.5, -0.6), (0.6, 2.5, -0.6), (0.6, 2.5, 0.6), (-0.6, 2.5, 0.6)], np.float64),
                 np.tile([0.0, -1.0, 0.0], (4, 1)), [(0, 1, 2), (0, 2, 3)], np.ones(3), 12.0))
    remaining = max(0, int(target_tris) - 4)
    while remaining >= 80:
        s = 1
        while 20 * 4 ** (s + 1) <= remaining and s < 7:
            s += 1
        p, _, f = icosphere_mesh(s)
        p = p.astype(np.float64)
        # displacement: a few seeded sinusoids of the direction
        k = rng.normal(size=(4, 3)) * 3.0
        ph = rng.uniform(0, 2 * np.pi, 4)
        disp = 1.0 + 0.15 * np.sum(np.sin(p @ k.T + ph), axis=1) / 4.0
        r = rng.uniform(0.15, 0.6)
        c = np.array([rng.uniform(-2.5, 2.5), 0.0, rng.uniform(-2.5, 2.5)])
        c[1] = r * 1.2
        pos = p * (disp * r)[:, None] + c
        objs.append((pos, _vertex_normals(pos, f), f, rng.uniform(0.1, 0.9, 3), 0.0))
        remaining -= len(f)
    cp, cn, cf = cube_mesh()
    cp, cn = np.asarray(cp, np.float64), np.asarray(cn, np.float64)
    while remaining >= 12:
        n_box = min(remaining // 12, int(rng.integers(2, 8)))
        base = np.array([rng.uniform(-3, 3), 0.0, rng.uniform(-3, 3)])
        y = 0.0
        for _ in range(n_box):
            hs = rng.uniform(0.05, 0.25, 3)
            ang = rng.uniform(0, np.pi)
            rot = np.array([[np.cos(ang), 0, np.sin(ang)], [0, 1, 0], [-np.sin(ang), 0, np.cos(ang)]])
            pos = (cp * hs) @ rot.T + base + np.array([0, y + hs[1], 0])
            objs.append((pos, cn @ rot.T, cf, rng.uniform(0.1, 0.9, 3), 0.0))
            y += 2 * hs[1]
            remaining -= 12
    vpos, vnrm, tri, tobj, ofv = [], [], [], [], [0]
    mats = np.zeros(len(objs), MAT_DTYPE)
    nv = 0
    for o, (p, n, f, alb, le) in enumerate(objs):
        vpos.append(np.asarray(p, np.float32))
        vnrm.append(np.asarray(n, np.float32))
        tri.append(np.asarray(f, np.int64) + nv)
        tobj.append(np.full(len(f), o, np.uint32))
        nv += len(p)
        ofv.append(nv)
        mats[o]["color"] = alb
        mats[o]["diffuse_t"] = mats[o]["reflect_t"] = mats[o]["transparent_t"] = 1.0
        mats[o]["refraction_index"] = 1.0
        mats[o]["light_source"] = 1 if le > 0 else 0
        mats[o]["light_strength"] = le
    sd = SceneData(np.concatenate(vpos), np.concatenate(vnrm), np.concatenate(tri), np.concatenate(tobj),
                   np.array(ofv, np.uint32), mats)
    az = rng.uniform(-np.pi, np.pi)
    el = rng.uniform(np.radians(20), np.radians(40))
    dist = 6.5
    pos = np.array([dist * np.cos(el) * np.cos(az), dist * np.sin(el), dist * np.cos(el) * np.sin(az)])
    d = -pos / np.linalg.norm(pos)
    theta, phi = np.arctan2(d[2], d[0]), np.arccos(d[1])
    cam = dict(position=pos.tolist(), angle=(float(theta / np.pi), float((np.pi / 2 - phi) / (np.pi / 2))))
    return sd, cam


def fbm_heights(n, seed, octaves=6, hmax=0.2):
    """(n+1, n+1) heights in [0, hmax] from seeded value-noise fBm."""
    rng = np.random.default_rng(seed)
    h = np.zeros((n + 1, n + 1), np.float64)
    x = np.linspace(0.0, 1.0, n + 1)
    amp = 1.0
    for o in range(octaves):
        cells = 4 * (2 ** o)
        lat = rng.uniform(-1.0, 1.0, (cells + 2, cells + 2))
        gx = x * cells
        i0 = np.floor(gx).astype(np.int64)
        f = gx - i0
        f = f * f * (3 - 2 * f)
        a = lat[i0][:, i0]
        b = lat[i0 + 1][:, i0]
        c = lat[i0][:, i0 + 1]
        d = lat[i0 + 1][:, i0 + 1]
        fy, fx = f[:, None], f[None, :]
        h += amp * ((a * (1 - fy) + b * fy) * (1 - fx) + (c * (1 - fy) + d * fy) * fx)
        amp *= 0.5
    h = (h - h.min()) / max(h.max() - h.min(), 1e-12)
    return (h * hmax).astype(np.float32)


def terrain(seed, root, cells=1024, tile=16, spheres=64, sphere_subdiv=4, lights=4):
    """Terrain scene: cells x cells heightfield over [-1, 1]^2 (xz) in tiles of tile x tile cells,
    icospheres and emissive quads. Returns dict(scene, camera, basepath, triangles)."""
    rng = np.random.default_rng(seed)
    base = _layout(root)
    hgt = fbm_heights(cells, seed)
    coords = np.linspace(-1.0, 1.0, cells + 1).astype(np.float32)
    # per-vertex normals of the heightfield (central differences)
    dzdx = np.gradient(hgt.astype(np.float64), coords.astype(np.float64), axis=1)
    dzdy = np.gradient(hgt.astype(np.float64), coords.astype(np.float64), axis=0)
    nrm_all = np.stack([-dzdx, np.ones_like(dzdx), -dzdy], axis=-1)
    nrm_all /= np.linalg.norm(nrm_all, axis=-1, keepdims=True)
    s_parts = []
    ntiles = cells // tile
    g = tile + 1
    fi = []
    for r in range(tile):
        for c in range(tile):
            a = r * g + c
            fi += [(a, a + g, a + 1), (a + 1, a + g, a + g + 1)]
    fi = np.array(fi, np.int64)
    for ty in range(ntiles):
        for tx in range(ntiles):
            r0, c0 = ty * tile, tx * tile
            zz, xx = np.meshgrid(coords[r0:r0 + g], coords[c0:c0 + g], indexing="ij")
            pos = np.stack([xx, hgt[r0:r0 + g, c0:c0 + g], zz], -1).reshape(-1, 3)
            nrm = nrm_all[r0:r0 + g, c0:c0 + g].reshape(-1, 3)
            name = "t_%d_%d.obj" % (ty, tx)
            write_obj(os.path.join(root, "res/obj", name), pos, nrm, fi)
            s_parts.append(_entry(name, (0, 0, 0), color=(0.6, 0.55, 0.45)))
    sp, sn, sf = icosphere_mesh(sphere_subdiv)
    write_obj(os.path.join(root, "res/obj/sphere.obj"), sp, sn, sf)
    for _ in range(spheres):
        r = float(np.exp(rng.uniform(np.log(0.01), np.log(0.1))))
        x, z = rng.uniform(-0.9, 0.9, 2)
        ix = int(round((x + 1) / 2 * cells))
        iz = int(round((z + 1) / 2 * cells))
        y = float(hgt[min(iz, cells), min(ix, cells)]) + r
        s_parts.append(_entry("sphere.obj", (x, y, z), scale=(r, r, r), color=rng.uniform(0.1, 0.9, 3)))
    write_obj(os.path.join(root, "res/obj/quad.obj"), *quad_mesh())
    for k in range(lights):
        x, z = rng.uniform(-0.6, 0.6, 2)
        s_parts.append(_entry("quad.obj", (x, 0.8, z), scale=(0.1, 0.1, 0.1),
                              rotation=(0, 0, 1, -math.pi / 2), color=(1, 1, 1), lightSource=15.0))
    scene = os.path.join(root, "res/scene/terrain_%d.scene" % seed)
    with open(scene, "w") as f:
        f.write("".join(s_parts))
    cam = os.path.join(root, "res/camera/terrain.camera")
    # from above and in front of the terrain, looking down at it
    write_camera(cam, (0.0, 1.3, 2.2), (-0.5, -0.35))
    ntri = ntiles * ntiles * fi.shape[0] + spheres * len(sf) + 2 * lights
    return dict(scene=scene, camera=cam, basepath=base, triangles=ntri)


def uniform_rays(n, lo, hi, seed, device="cuda"):
    """Closest-hit microbenchmark rays as two (n, 4) float32 tensors: origins uniform in the box
    [lo, hi], directions uniform on the unit sphere (z = 2u - 1, phi = 2 pi v, the mapping of the
    reference's random direction, random.cpp:16-29). Seeded torch generator on `device`."""
    import torch
    g = torch.Generator(device=device)
    g.manual_seed(int(seed))
    u = torch.rand((n, 5), generator=g, device=device, dtype=torch.float32)
    lo_t = torch.as_tensor(np.asarray(lo, np.float32), device=device)
    hi_t = torch.as_tensor(np.asarray(hi, np.float32), device=device)
    o = torch.zeros((n, 4), dtype=torch.float32, device=device)
    o[:, :3] = lo_t + (hi_t - lo_t) * u[:, :3]
    z = 2.0 * u[:, 3] - 1.0
    r = torch.sqrt(torch.clamp(1.0 - z * z, min=0.0))
    phi = (2.0 * math.pi) * u[:, 4]
    d = torch.zeros((n, 4), dtype=torch.float32, device=device)
    d[:, 0] = r * torch.cos(phi)
    d[:, 1] = r * torch.sin(phi)
    d[:, 2] = z
    return o, d
