"""TEST INFRASTRUCTURE ONLY. Reader for the tagged binary files written by oracle/ref_harness
and helpers that run the compiled reference harness (oracle/_ref/) to produce them."""
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
HARNESS = os.path.join(REF_DIR, "ref_harness")
REF_BENCH = os.path.join(REF_DIR, "ref_bench")
REF_BENCH_SHIM = os.path.join(REF_DIR, "ref_bench_shim")
REF_CLI = os.path.join(REF_DIR, "SoftwareRenderer")

_KINDS = {"f": np.float32, "u": np.uint32}


def reference_root():
    """The reference checkout the harness is built from: SWR_REFERENCE, else oracle/Makefile's REF."""
    ref = os.environ.get("SWR_REFERENCE")
    if ref:
        return ref
    p = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True, text=True)
    return p.stdout.strip()


def reference_available():
    """True when the reference sources and the compiled harness are both present."""
    return os.path.isdir(os.path.join(reference_root(), "software_renderer")) and os.path.exists(HARNESS)


def read(path):
    with open(path, "rb") as f:
        buf = f.read()
    if buf[:8] != b"SWRB0001":
        raise ValueError("not a harness dump: %s" % path)
    out = {}
    off = 8
    while off < len(buf):
        hdr = buf[off:off + 48]
        name = hdr[:32].split(b"\0", 1)[0].decode()
        kind = chr(hdr[32])
        count = int(np.frombuffer(hdr[40:48], np.uint64)[0])
        dt = _KINDS[kind]
        nbytes = count * np.dtype(dt).itemsize
        out[name] = np.frombuffer(buf[off + 48:off + 48 + nbytes], dtype=dt).copy()
        off += 48 + nbytes
    return out


def available():
    return os.path.exists(HARNESS)


def run(*args, timeout=600):
    p = subprocess.run([HARNESS] + [str(a) for a in args], capture_output=True, text=True,
                       timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError("ref_harness %s failed (%d): %s" % (args[0], p.returncode, p.stderr))


def dump(basepath, scene, camera, width, height, out):
    run("dump", basepath, scene, camera, width, height, out)
    return read(out)


def trace(basepath, scene, rays6, out):
    rays6 = np.ascontiguousarray(rays6, dtype=np.float32).reshape(-1, 6)
    rpath = out + ".rays"
    rays6.tofile(rpath)
    run("trace", basepath, scene, rpath, out)
    return read(out)


def render(basepath, scene, camera, width, height, spp, depth, seed, p0, p1, out):
    run("render", basepath, scene, camera, width, height, spp, depth, seed, p0, p1, out)
    return read(out)


def render_bdpt(basepath, scene, camera, width, height, spp, vision, light, max_depth, seed, p0, p1, out):
    run("render_bdpt", basepath, scene, camera, width, height, spp, vision, light, max_depth, seed, p0, p1, out)
    return read(out)


def tree(boxes6, out):
    boxes6 = np.ascontiguousarray(boxes6, dtype=np.float32).reshape(-1, 6)
    bpath = out + ".boxes"
    boxes6.tofile(bpath)
    run("tree", bpath, out)
    return read(out)["tree"]
