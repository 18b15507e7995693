"""Builds the native library in-tree: master_thesis_b200/lib/libswr.so and the command-line
drop-ins SoftwareRenderer and RayTrace (headless), for sm_100a. Host C++ is compiled without floating-point contraction
because the world-space geometry and camera math must round exactly like the reference's build.

Usage: python -m master_thesis_b200.build [--verbose]
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(HERE, "lib")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
HOST_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-Wno-unused-function",
              "-I/usr/local/cuda/include"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
                     "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"]

HOST_SRC = ["host/surface.cpp", "host/ref_bvh.cpp", "host/wide_bvh.cpp", "host/derive.cpp",
            "host/capi_host.cpp", "host/scene_pack.cpp"]
CUDA_SRC = ["cuda/scene.cu", "cuda/render.cu", "cuda/batch.cu", "cuda/build.cu", "cuda/rt.cu", "cuda/instance.cu"]
CLI_SRC = {"SoftwareRenderer": "cli/swr_main.cpp", "RayTrace": "cli/rt_main.cpp"}


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("command failed: %s\n%s\n%s" % (" ".join(cmd), p.stdout, p.stderr))
    if verbose and (p.stdout or p.stderr):
        print(p.stdout + p.stderr, flush=True)
    return p.stdout + p.stderr


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _headers():
    hs = [os.path.join(ROOT, "include", "swr.h")]
    for d, _, fs in os.walk(CSRC):
        hs += [os.path.join(d, f) for f in fs if f.endswith((".h", ".cuh"))]
    return hs


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = _headers()
    jobs = []
    objs = []
    for s in HOST_SRC:
        src = os.path.join(CSRC, s)
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, [src] + headers):
            jobs.append([CXX] + HOST_FLAGS + ["-c", src, "-o", o])
    for s in CUDA_SRC:
        src = os.path.join(CSRC, s)
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, [src] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVCC_FLAGS + extra + ["-c", src, "-o", o])
    logs = []
    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        for out in ex.map(lambda c: _run(c, verbose), jobs):
            logs.append(out)
    so = os.path.join(LIB, "libswr.so")
    if _stale(so, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", so] + objs + ["-lpthread"], verbose)
    for name, rel in CLI_SRC.items():
        cli = os.path.join(LIB, name)
        cli_src = os.path.join(CSRC, rel)
        if _stale(cli, [cli_src, so] + headers):
            _run([CXX, "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include",
                  cli_src, "-o", cli, "-L" + LIB, "-lswr", "-L/usr/local/cuda/lib64", "-lcudart",
                  "-Wl,-rpath,$ORIGIN:" + LIB + ":/usr/local/cuda/lib64"], verbose)
    return so, "\n".join(logs)


def build_oracle(verbose=False):
    """Compiles the oracle's C restatement and, when the reference sources are present, the
    reference harness binaries (test infrastructure)."""
    oracle = os.path.join(ROOT, "oracle")
    _run(["make", "-s", "-C", oracle, "oracle"], verbose)
    # the reference checkout: SWR_REFERENCE, else the Makefile's default (absent on GPU machines)
    ref = _run(["make", "-s", "-C", oracle, "print-ref"], False).strip()
    if os.path.isdir(os.path.join(ref, "software_renderer")):
        _run(["make", "-s", "-j8", "-C", oracle, "ref"], verbose)


if __name__ == "__main__":
    v = "--verbose" in sys.argv
    so, logs = build(verbose=v, ptxas_info="--ptxas" in sys.argv)
    if "--ptxas" in sys.argv:
        print(logs)
    print(so)
