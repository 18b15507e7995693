"""The benchmark's terrain configuration and the GPU parity test of that same image must describe
one workload: scene parameters, image size, samples, depth, seed and paths in flight."""
import bench
import test_gpu_terrain_render as T


def test_terrain_parity_test_renders_the_benchmarked_configuration():
    c = bench.CONFIGS["c2"]
    assert (c["W"], c["H"], c["spp"], c["depth"]) == (T.BENCH_W, T.BENCH_H, T.BENCH_SPP, T.BENCH_DEPTH)
    assert c["wave_size"] == T.BENCH_WAVE
    assert dict(seed=c["seed"], cells=c["cells"], tile=c["tile"], spheres=c["spheres"], sphere_subdiv=c["subdiv"],
                lights=c["lights"]) == T.BENCH_SCENE
    # rank 0 of bench.py renders its image with seed 1000 + rank
    assert T.BENCH_SEED == 1000
