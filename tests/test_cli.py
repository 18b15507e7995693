"""SoftwareRenderer command-line drop-in (software_renderer/main.cpp:28-87): argument handling on
the CPU; on the GPU, the written P6 file must equal the library's own render of the same files,
quantised as the reference does."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from master_thesis_b200 import scenes

CLI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "master_thesis_b200", "lib",
                   "SoftwareRenderer")


def test_cli_wrong_argument_count():
    p = subprocess.run([CLI, "a", "b"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 255
    assert "wrong paramter count" in p.stdout and "Usage: SoftwareRenderer renderer scene" in p.stdout


def _setup(tmp_path, spp=8, depth=5):
    s = scenes.cornell(3, str(tmp_path))
    exe = os.path.join(s["basepath"], "SoftwareRenderer")  # meshes resolve from <exe dir>/../res/obj
    shutil.copy(CLI, exe)
    rpath = tmp_path / "PathTracer.renderer"
    rpath.write_text("PathTracer\n\tvisionJumpCount(%d)\n\traysPerPixel(%d)\n" % (depth, spp))
    return s, exe, str(rpath)


def test_cli_rejects_unknown_renderer(tmp_path):
    s, exe, _ = _setup(tmp_path)
    bad = tmp_path / "B.renderer"
    bad.write_text("PhotonMapper\n\tvisionJumpCount(5)\n\traysPerPixel(4)\n")
    p = subprocess.run([exe, str(bad), s["scene"], "8", "8", "2", s["camera"], str(tmp_path / "o.ppm")],
                       capture_output=True, text=True, timeout=120, env=dict(os.environ, CUDA_VISIBLE_DEVICES=""))
    assert p.returncode != 0
    assert "getRenderer not found" in p.stderr and "PhotonMapper" in p.stderr
    assert not (tmp_path / "o.ppm").exists()


@pytest.mark.gpu
def test_cli_image_equals_library_render(tmp_path):
    import master_thesis_b200 as swr
    W, H, spp, depth = 64, 48, 8, 5
    s, exe, rpath = _setup(tmp_path, spp, depth)
    out = tmp_path / "out.ppm"
    p = subprocess.run([exe, rpath, s["scene"], str(W), str(H), "4", s["camera"], str(out)],
                       capture_output=True, text=True, timeout=300, env=dict(os.environ, SWR_SEED="5"))
    assert p.returncode == 0, p.stdout + p.stderr
    data = out.read_bytes()
    header = b"P6\n%d\n%d\n255\n" % (W, H)
    assert data.startswith(header) and len(data) == len(header) + W * H * 3
    sd = swr.load_scene(s["scene"], s["basepath"])
    cam = swr.load_camera(s["camera"], W, H)
    img = swr.Scene(sd).render(cam, W, H, spp, depth, seed=5, mode=swr.MODE_REFERENCE)
    ref = swr.quantize_rgb8(img.cpu().numpy())
    got = np.frombuffer(data[len(header):], np.uint8).reshape(H, W, 3)
    assert np.array_equal(got, ref)
    assert ref.max() > 0


@pytest.mark.gpu
def test_cli_bidirectional_equals_library_render(tmp_path):
    import master_thesis_b200 as swr
    W, H = 48, 32
    s, exe, _ = _setup(tmp_path)
    rpath = tmp_path / "BDPT.renderer"
    rpath.write_text("BidirectionalPathTracer\n\tvisionJumpCount(5)\n\tlightJumpCount(4)\n\tmaxDepth(5)\n"
                     "\traysPerPixel(6)\n")
    out = tmp_path / "bd.ppm"
    p = subprocess.run([exe, str(rpath), s["scene"], str(W), str(H), "4", s["camera"], str(out)],
                       capture_output=True, text=True, timeout=300, env=dict(os.environ, SWR_SEED="9"))
    assert p.returncode == 0, p.stdout + p.stderr
    sd = swr.load_scene(s["scene"], s["basepath"])
    cam = swr.load_camera(s["camera"], W, H)
    img = swr.Scene(sd).render_bdpt(cam, W, H, 6, 5, 4, 5, seed=9)
    header = b"P6\n%d\n%d\n255\n" % (W, H)
    got = np.frombuffer(out.read_bytes()[len(header):], np.uint8).reshape(H, W, 3)
    ref = swr.quantize_rgb8(img.cpu().numpy())
    assert np.array_equal(got, ref) and ref.max() > 0


RT_CLI = os.path.join(os.path.dirname(CLI), "RayTrace")


def test_raytrace_cli_argument_handling(tmp_path):
    """The headless RayTrace drop-in (src/main.cpp:100-133 of the Vulkan program): argument count
    check, the windowed form without a camera file refused, renderer names checked before any
    device work."""
    p = subprocess.run([RT_CLI, "a", "b"], capture_output=True, text=True, timeout=60)
    assert p.returncode == 255
    assert "wrong paramter count" in p.stdout and "Usage: RayTrace renderer scene" in p.stdout
    s = scenes.cornell(3, str(tmp_path))
    exe = os.path.join(s["basepath"], "RayTrace")
    shutil.copy(RT_CLI, exe)
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    p = subprocess.run([exe, "r.renderer", s["scene"], "8", "8"], capture_output=True, text=True, timeout=60, env=env)
    assert p.returncode == 255 and "needs one" in p.stdout
    for text, msg in [("Majercik2022\n", "does not restate"), ("Raymarcher\n", "getRenderer not found"),
                      ("PathTracer\n\tvisionJumpCount(5)\n\tvisionRayPerPixelCount(2)\nBlur\n", "getDenoiser not found")]:
        r = tmp_path / "x.renderer"
        r.write_text(text)
        out = tmp_path / "o.ppm"
        p = subprocess.run([exe, str(r), s["scene"], "8", "8", s["camera"], str(out), "1"], capture_output=True,
                           text=True, timeout=120, env=env)
        assert p.returncode != 0 and msg in p.stderr, p.stderr
        assert not out.exists()
