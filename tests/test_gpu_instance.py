"""Moving objects on the GPU (swr_scene_create_from_host + swr_scene_set_transforms): after new
placements, a scene must answer exactly like a scene loaded from a file with those placements
(hits, tie ranks, renders), with its BVH refit instead of rebuilt."""
import math
import os

import numpy as np
import pytest

import master_thesis_b200 as swr
from master_thesis_b200 import rt, scenes
from master_thesis_b200.scenes import _entry, _layout, write_camera, write_obj
from helpers import rays_uniform

pytestmark = pytest.mark.gpu


def _objects(rng):
    """Cornell-like walls, boxes, spheres and a light: (mesh, color, light strength)."""
    objs = [("quad.obj", (0.8, 0.8, 0.8), None) for _ in range(5)]
    objs += [("cube.obj", tuple(rng.uniform(0.2, 0.9, 3)), None) for _ in range(3)]
    objs += [("sphere.obj", tuple(rng.uniform(0.2, 0.9, 3)), None) for _ in range(3)]
    objs += [("quad.obj", (1.0, 1.0, 1.0), 12.0)]
    return objs


def _placements(rng, n, spread):
    pos = rng.uniform(-spread, spread, (n, 3)).astype(np.float32)
    scl = rng.uniform(0.15, 0.6, (n, 3)).astype(np.float32)
    axis = rng.normal(size=(n, 3)).astype(np.float32)
    ang = rng.uniform(-math.pi, math.pi, n).astype(np.float32)
    return pos, scl, axis, ang


def _write_scene(root, name, objs, pos, scl, axis, ang):
    s = ""
    for k, (mesh, color, light) in enumerate(objs):
        kw = dict(scale=scl[k], rotation=(axis[k][0], axis[k][1], axis[k][2], ang[k]), color=color)
        if light is not None:
            kw["lightSource"] = light
        s += _entry(mesh, pos[k], **kw)
    path = os.path.join(root, "res/scene/%s.scene" % name)
    with open(path, "w") as f:
        f.write(s)
    return path


def _setup(tmp_path, seed=3):
    root = str(tmp_path)
    base = _layout(root)
    write_obj(os.path.join(root, "res/obj/quad.obj"), *scenes.quad_mesh())
    write_obj(os.path.join(root, "res/obj/cube.obj"), *scenes.cube_mesh())
    write_obj(os.path.join(root, "res/obj/sphere.obj"), *scenes.icosphere_mesh(2))
    cam = os.path.join(root, "res/camera/c.camera")
    write_camera(cam, (3.4, 0, 0), (1, 0), fov=50)
    rng = np.random.default_rng(seed)
    objs = _objects(rng)
    return root, base, cam, objs, rng


def _xf(pos, scl, axis, ang):
    q = np.stack([swr.rotation_from_axis_angle(axis[k], ang[k]) for k in range(len(pos))])
    return np.concatenate([pos, scl, q], axis=1).astype(np.float32)


def _hits(sc, ro, rd):
    return sc.trace(ro, rd).view(np.uint32)


@pytest.mark.parametrize("builder", ["host", "device"])
def test_moved_scene_answers_like_a_loaded_scene(tmp_path, builder):
    root, base, cam_path, objs, rng = _setup(tmp_path)
    p0 = _placements(rng, len(objs), 1.0)
    p1 = _placements(rng, len(objs), 1.0)
    moving = swr.Scene.from_file(_write_scene(root, "a", objs, *p0), base, builder=builder)
    loaded0 = swr.Scene(swr.load_scene(_write_scene(root, "a0", objs, *p0), base))
    assert np.array_equal(moving.transforms(), _xf(*p0))
    ro, rd = rays_uniform(30000, (-1.6, -1.6, -1.6), (1.6, 1.6, 1.6), seed=9)
    assert np.array_equal(_hits(moving, ro, rd), _hits(loaded0, ro, rd))
    moving.set_transforms(_xf(*p1))
    loaded1 = swr.Scene(swr.load_scene(_write_scene(root, "a1", objs, *p1), base))
    h_moving, h_loaded = _hits(moving, ro, rd), _hits(loaded1, ro, rd)
    assert np.array_equal(h_moving, h_loaded)  # triangle id, object, dist2 and t, ties included
    assert np.mean(h_loaded[:, 0] != 0xFFFFFFFF) > 0.1
    # renders: the reference path tracer (per-sample radiance), the RayTrace frame
    W, H = 40, 30
    cam = swr.load_camera(cam_path, W, H, use_fov_key=True)
    for sc in (moving, loaded1):
        sc._img = sc.render(cam, W, H, 8, 5, seed=4).cpu().numpy()
        sc._rt = rt.render(sc, cam, W, H, 5, 5, want_rgb=False)[1].cpu().numpy()
    assert np.array_equal(moving._img, loaded1._img)
    assert np.array_equal(moving._rt, loaded1._rt)
    # the bidirectional tracer samples the moved light's triangles
    b1 = moving.render_bdpt(cam, W, H, 4, 5, 5, 5, seed=2).cpu().numpy()
    b2 = loaded1.render_bdpt(cam, W, H, 4, 5, 5, 5, seed=2).cpu().numpy()
    assert np.array_equal(b1, b2)
    # moving back restores the first placements exactly
    moving.set_transforms(_xf(*p0))
    assert np.array_equal(_hits(moving, ro, rd), _hits(loaded0, ro, rd))


def test_many_small_moves_keep_hits_exact(tmp_path):
    """A sequence of small moves (an animation) through the refit, checked at the end and
    against a loaded scene at every third frame."""
    root, base, cam_path, objs, rng = _setup(tmp_path, seed=5)
    pos, scl, axis, ang = _placements(rng, len(objs), 1.0)
    moving = swr.Scene.from_file(_write_scene(root, "m", objs, pos, scl, axis, ang), base)
    ro, rd = rays_uniform(20000, (-1.6, -1.6, -1.6), (1.6, 1.6, 1.6), seed=2)
    vel = rng.normal(scale=0.05, size=pos.shape).astype(np.float32)
    for frame in range(9):
        pos = (pos + vel).astype(np.float32)
        ang = (ang + np.float32(0.1)).astype(np.float32)
        moving.set_transforms(_xf(pos, scl, axis, ang))
        if frame % 3 == 2:
            ref = swr.Scene(swr.load_scene(_write_scene(root, "m%d" % frame, objs, pos, scl, axis, ang), base))
            assert np.array_equal(_hits(moving, ro, rd), _hits(ref, ro, rd)), frame


def test_moving_objects_on_a_terrain(tmp_path):
    s = scenes.terrain(4, str(tmp_path), cells=128, tile=16, spheres=12, sphere_subdiv=2, lights=2)
    moving = swr.Scene.from_file(s["scene"], s["basepath"], builder="device")
    xf = moving.transforms()
    rng = np.random.default_rng(1)
    sd = moving.data
    nobj = sd.num_objects
    # lift every object (tiles, spheres, lights) by a different small amount
    xf2 = xf.copy()
    xf2[:, 1] += rng.uniform(0.0, 0.05, nobj).astype(np.float32)
    moving.set_transforms(xf2)
    ro, rd = rays_uniform(50000, sd.vpos.min(0) - 0.1, sd.vpos.max(0) + 0.1, seed=3)
    # reference: the same scene data with the lifted placements, through the host loader
    text = open(s["scene"]).read()
    lines = text.split("\n")
    k = -1
    out = []
    for line in lines:
        if line and not line.startswith("\t"):
            k += 1
        if line.startswith("\tposition("):
            p = xf2[k, :3]
            line = "\tposition(%s, %s, %s)" % tuple(scenes._fmt(x) for x in p)
        out.append(line)
    path2 = os.path.join(os.path.dirname(s["scene"]), "lifted.scene")
    with open(path2, "w") as f:
        f.write("\n".join(out))
    ref = swr.Scene(swr.load_scene(path2, s["basepath"]))
    assert np.array_equal(_hits(moving, ro, rd), _hits(ref, ro, rd))


def test_set_transforms_rejects_bad_requests(tmp_path):
    root, base, cam_path, objs, rng = _setup(tmp_path)
    p0 = _placements(rng, len(objs), 1.0)
    path = _write_scene(root, "e", objs, *p0)
    plain = swr.Scene(swr.load_scene(path, base))
    with pytest.raises(swr.SwrError):
        plain.set_transforms(_xf(*p0))  # not made from a host scene
    moving = swr.Scene.from_file(path, base)
    with pytest.raises(swr.SwrError):
        moving.set_transforms(_xf(*p0)[:-1])  # one transform per object
    bad = _xf(*p0)
    bad[2, 0] = np.nan
    with pytest.raises(swr.SwrError):
        moving.set_transforms(bad)
    # finite placements whose products overflow: refused after the fact; valid ones then restore
    # exact answers
    huge = _xf(*p0)
    huge[3, 0:6] = np.float32(3e38)  # position and scale: some vertex coordinate exceeds 3.4e38
    with pytest.raises(swr.SwrError):
        moving.set_transforms(huge)
    moving.set_transforms(_xf(*p0))
    ro, rd = rays_uniform(5000, (-1.6, -1.6, -1.6), (1.6, 1.6, 1.6), seed=4)
    assert np.array_equal(_hits(moving, ro, rd), _hits(plain, ro, rd))


def test_set_transforms_rejects_normals_that_overflow(tmp_path):
    """A finite placement whose world positions stay finite while some world normals overflow: a
    sphere of radius 1e-3 scaled by 3e38 in x and y and turned by a non-unit quaternion (|q|^2 =
    1.414, 45 degrees about z), so the matrix rows hold +-3e38 and a normal near (1, 1, 0)/sqrt(2)
    sums two of them past the float range. The object boxes are finite; the call must still fail,
    and valid placements afterwards restore exact answers."""
    root, base, cam_path, objs, rng = _setup(tmp_path)
    pos, nrm, faces = scenes.icosphere_mesh(2)
    write_obj(os.path.join(root, "res/obj/tiny.obj"), pos * np.float32(1e-3), nrm, faces)
    objs = objs + [("tiny.obj", (0.5, 0.5, 0.5), None)]
    p0 = _placements(rng, len(objs), 1.0)
    path = _write_scene(root, "n", objs, *p0)
    plain = swr.Scene(swr.load_scene(path, base))
    moving = swr.Scene.from_file(path, base)
    bad = _xf(*p0)
    k = math.sqrt(1.414)
    h = math.radians(22.5)
    bad[-1] = np.array([0.0, 0.0, 0.0, 3e38, 3e38, 1.0, k * math.cos(h), 0.0, 0.0, k * math.sin(h)], np.float32)
    with pytest.raises(swr.SwrError, match="normals"):
        moving.set_transforms(bad)
    moving.set_transforms(_xf(*p0))
    ro, rd = rays_uniform(5000, (-1.6, -1.6, -1.6), (1.6, 1.6, 1.6), seed=6)
    assert np.array_equal(_hits(moving, ro, rd), _hits(plain, ro, rd))
