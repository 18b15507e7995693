"""B200-native re-implementation of vikkre/master_thesis's SoftwareRenderer path tracer.

The compute path is the native library (master_thesis_b200/lib/libswr.so: C++ host surface +
sm_100a CUDA kernels behind the C ABI in include/swr.h); this package is the Python tooling on
top of it. Importing it loads the native library and fails if it has not been built.
"""
from ._native import (MODE_PHYSICAL, MODE_REFERENCE, SwrError)  # noqa: F401
from .api import (Scene, SceneData, MAT_DTYPE, camera_arrays, load_camera, load_renderer,  # noqa: F401
                  load_scene, quantize_rgb8, write_ppm)
