"""The two builds of the reference's closest-centre BVH order (bounding_volume_hierachy.cpp:9-75):
the flat build and the kd-tree build must make the same merge at every step, ties included.
The flat build itself is checked against the reference's own builder in test_surface.py."""
import ctypes

import numpy as np
import pytest

from helpers import build_twin


def _merges(boxes, mode):
    L = ctypes.CDLL(build_twin())
    L.twin_ref_merges.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    L.twin_ref_merges.restype = None
    b = np.ascontiguousarray(boxes, np.float32)
    n = b.shape[0]
    left = np.full(2 * n - 1, -7, np.int32)
    right = np.full(2 * n - 1, -7, np.int32)
    L.twin_ref_merges(b.ctypes.data, n, mode, left.ctypes.data, right.ctypes.data)
    return left, right


def _boxes(centres, half):
    c = np.asarray(centres, np.float32)
    h = np.broadcast_to(np.asarray(half, np.float32), c.shape)
    return np.concatenate([c - h, c + h], 1)


def _cases():
    rng = np.random.default_rng(11)
    yield "uniform", _boxes(rng.uniform(-1, 1, (1500, 3)), rng.uniform(0, 0.05, (1500, 3)))
    # a terrain-like lattice: equal spacing, so equal distances everywhere
    g = np.stack(np.meshgrid(np.arange(40), np.arange(40), indexing="ij"), -1).reshape(-1, 2).astype(np.float32)
    lat = np.stack([g[:, 0] / 32, rng.integers(0, 3, g.shape[0]) / 64, g[:, 1] / 32], 1)
    yield "lattice", _boxes(lat, 1 / 64)
    yield "flat lattice", _boxes(np.stack([g[:, 0], np.zeros(len(g)), g[:, 1]], 1), 0.5)
    # many exactly equal centres
    dup = rng.uniform(-1, 1, (300, 3))
    dup[::2] = dup[0]
    dup[1::7] = dup[3]
    yield "duplicates", _boxes(dup, 0.01)
    # points on a line with geometric spacing (long merge chains)
    line = np.zeros((400, 3), np.float32)
    line[:, 0] = np.cumsum(1.01 ** np.arange(400))
    yield "geometric line", _boxes(line, 0.0)
    # tight clusters far apart, and mixed scales
    cl = np.concatenate([rng.normal(c, 1e-4, (200, 3)) for c in ([0, 0, 0], [5e3, 0, 0], [0, -7e3, 2e3])])
    yield "clusters", _boxes(cl, rng.uniform(0, 1e-4, (600, 3)))
    mix = np.concatenate([rng.uniform(-1e6, 1e6, (100, 3)), rng.uniform(-1e-6, 1e-6, (100, 3)), rng.uniform(-1, 1, (100, 3))])
    yield "mixed scales", _boxes(mix, 0.0)
    # squared distances in the subnormal range, many of them rounding to equal values or to 0
    yield "subnormal distances", _boxes(rng.uniform(-1, 1, (300, 3)) * 3e-20, 0.0)
    # integer grid in 3D: huge numbers of exact ties
    g3 = np.stack(np.meshgrid(*[np.arange(9)] * 3, indexing="ij"), -1).reshape(-1, 3)
    yield "cube lattice", _boxes(g3, 0.25)
    # boxes of very different sizes (centres of unequal boxes)
    lo = rng.uniform(-1, 1, (500, 3))
    yield "uneven boxes", np.concatenate([lo, lo + rng.exponential(0.2, (500, 3))], 1)


@pytest.mark.parametrize("name,boxes", list(_cases()), ids=[c[0] for c in _cases()])
def test_indexed_build_merges_like_flat(name, boxes):
    fl = _merges(boxes, 1)
    ix = _merges(boxes, 2)
    assert np.array_equal(fl[0], ix[0]) and np.array_equal(fl[1], ix[1]), name
    auto = _merges(boxes, 0)
    assert np.array_equal(auto[0], fl[0]) and np.array_equal(auto[1], fl[1])
    n = boxes.shape[0]
    # every node is merged exactly once, and a parent comes after its children
    kids = np.concatenate([fl[0][n:], fl[1][n:]])
    assert np.array_equal(np.sort(kids), np.arange(2 * n - 2))
    assert np.all(fl[0][n:] < np.arange(n, 2 * n - 1)) and np.all(fl[0][n:] < fl[1][n:])


def test_indexed_build_with_threaded_first_queries():
    rng = np.random.default_rng(4)
    g = np.stack(np.meshgrid(np.arange(64), np.arange(64), indexing="ij"), -1).reshape(-1, 2).astype(np.float32)
    terrain = np.stack([g[:, 0] / 32, rng.integers(0, 4, len(g)) / 128, g[:, 1] / 32], 1)
    spheres = rng.uniform(0, 2, (64, 3)) * [1, 0.4, 1]
    b = _boxes(np.concatenate([terrain, spheres]), 1 / 64)
    fl, ix = _merges(b, 1), _merges(b, 3)
    assert np.array_equal(fl[0], ix[0]) and np.array_equal(fl[1], ix[1])


@pytest.mark.parametrize("n", [2, 3, 5, 17, 63, 64, 65, 130])
def test_indexed_build_small_inputs(n):
    rng = np.random.default_rng(n)
    for spread in (1.0, 1e-3):
        c = np.round(rng.uniform(-1, 1, (n, 3)) * 4) / 4 * spread  # coarse values: ties
        b = _boxes(c, 0.01 * spread)
        fl, ix = _merges(b, 1), _merges(b, 2)
        assert np.array_equal(fl[0], ix[0]) and np.array_equal(fl[1], ix[1])


def test_inputs_outside_the_indexed_range_take_the_flat_build():
    rng = np.random.default_rng(3)
    c = rng.uniform(-1, 1, (200, 3)).astype(np.float32)
    c[5] = [3e19, 0, 0]  # squared distances overflow: the flat build handles them
    c[9] = [np.nan, 0, 0]
    b = _boxes(c, 0.01)
    fl, ix = _merges(b, 1), _merges(b, 2)
    assert np.array_equal(fl[0], ix[0]) and np.array_equal(fl[1], ix[1])
