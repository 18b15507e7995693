"""B200-native re-implementation of vikkre/master_thesis's SoftwareRenderer path tracer.

The compute path is the native library (master_thesis_b200/lib/libswr.so: C++ host surface +
sm_100a CUDA kernels behind the C ABI in include/swr.h); this package is the Python tooling on
top of it. The native library is loaded on first use of any public name and its absence raises
ImportError there: nothing falls back to another implementation. (Importing the build module,
master_thesis_b200.build, does not load it, so a stale or missing library can be rebuilt.)
"""
import importlib

_EXPORTS = {
    "MODE_PHYSICAL": "._native", "MODE_REFERENCE": "._native", "SwrError": "._native",
    "Scene": ".api", "SceneData": ".api", "Batch": ".api", "MAT_DTYPE": ".api", "camera_arrays": ".api",
    "load_camera": ".api", "make_camera": ".api", "load_renderer": ".api", "load_renderer_params": ".api",
    "load_scene": ".api", "quantize_rgb8": ".api", "rotation_from_axis_angle": ".api",
    "write_ppm": ".api", "write_png": ".api",
}

__all__ = sorted(_EXPORTS)


def __getattr__(name):
    mod = _EXPORTS.get(name)
    if mod is None:
        raise AttributeError("module 'master_thesis_b200' has no attribute %r" % name)
    value = getattr(importlib.import_module(mod, __name__), name)
    globals()[name] = value
    return value
