"""The C ABI library loads without a GPU and exports every function include/swr.h declares; the
Python binding declares exactly those functions; argument validation needs no GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import master_thesis_b200 as swr
from master_thesis_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "swr.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(swr_[a-z0-9_]+)\s*\(", src)))


def test_header_symbols_exported():
    names = _declared()
    assert len(names) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(N.LIB_PATH)
    for n in names:
        getattr(lib, n)


def test_binding_covers_header():
    assert sorted(N.SIGNATURES) == _declared()


def test_abi_version_and_errors():
    assert N.lib.swr_abi_version() == 3
    d = N.SceneDesc()
    h = ctypes.c_void_p()
    rc = N.lib.swr_scene_create(ctypes.byref(d), None, ctypes.byref(h))
    assert rc == N.SWR_ERR_INVALID and not h.value
    assert b"empty scene" in N.lib.swr_last_error()
    assert N.lib.swr_scene_create(None, None, ctypes.byref(h)) == N.SWR_ERR_INVALID


def test_descriptor_validation():
    mats = np.zeros(1, swr.MAT_DTYPE)
    mats["refraction_index"] = 1.0
    v = np.zeros((3, 3), np.float32)
    v[1, 0] = v[2, 1] = 1
    sd = swr.SceneData(v, v, [[0, 1, 2]], [0], [0, 3], mats)
    out = sd.derive()
    assert np.array_equal(out["e0"], [[1, 0, 0]])
    bad = swr.SceneData(v, v, [[0, 1, 5]], [0], [0, 3], mats)
    with pytest.raises(swr.SwrError) as e:
        bad.derive()
    assert e.value.code == N.SWR_ERR_INVALID
    bad2 = swr.SceneData(v, v, [[0, 1, 2]], [0], [0, 2], mats)
    with pytest.raises(swr.SwrError):
        bad2.derive()
