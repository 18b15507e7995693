"""Benchmark of the path tracer on the terrain workload (the plain method at scale):
1024x1024-cell heightfield terrain (2,097,152 triangles, seeded 6-octave fBm heights in [0, 0.2])
in 64x64 OBJ tiles, 64 icospheres of subdivision 4 (radii log-uniform 0.01-0.1), 4 emissive quads;
1920x1080 pixels, 64 samples per pixel, depth 8, reference semantics (so the reference's CPU path
renders the identical files with the identical estimator).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c2|c1]

One step = one full image (all pixels x spp samples). `value` is Msamples/s with the scene
resident in device memory; `e2e` renders through the C ABI into a pinned host buffer (the
library's device->host copy of the image inside the timed region). With N>1 every rank renders
its own image of the same scene with its own seed (independent units, weak scaling); no
collective is on the data path. The reference arm (--impl reference) times the reference's own
CPU implementation (oracle/_ref/ref_bench: the unmodified SoftwareRenderer sources) on this
machine's cores for a bounded sample of the same workload.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: scene parameters, image, spp, depth
    # wave_size: paths in flight, 2^27 measured best for this image by the autotuner (2^24..2^27
    # with refill 4-12 and shading blocks 256/512): the whole image's 132.7 M samples are in flight
    # at once. The library's default of 2^23 bounds a scene's queue memory at 1.2 GB; 2^27 takes
    # 19.3 GB
    "c2": dict(kind="terrain", cells=1024, tile=16, spheres=64, subdiv=4, lights=4, W=1920, H=1080, spp=64,
               depth=8, seed=2024, microbench_rays=1 << 24, wave_size=1 << 27),
    "c1": dict(kind="cornell", W=256, H=256, spp=16, depth=5, seed=1),
    # the Cornell scene through the bidirectional tracer with the reference's own BDPT renderer
    # settings (res/renderer/SoftwareRendererBidirectionalPathTracer.renderer: 5/5/5)
    "c1b": dict(kind="cornell", renderer="bdpt", W=256, H=256, spp=16, depth=5, light_jumps=5, max_depth=5, seed=1),
    # the terrain scene at a reduced image size, for profiler captures of single kernel launches
    "c2s": dict(kind="terrain", cells=1024, tile=16, spheres=64, subdiv=4, lights=4, W=480, H=270, spp=16,
                depth=8, seed=2024, microbench_rays=1 << 22),
    # batched: 256 scenes, 1k-500k triangles (log-uniform), image sides {64..1024}, spp {4,16,64}, depth 6
    "c3": dict(kind="batch", scenes=256, depth=6, seed=7, sides=[64, 128, 256, 512, 1024], spps=[4, 16, 64],
               tris=[1e3, 5e5]),
    # the same batch restricted to small jobs (64x64..128x128, 4-16 spp, 1k-50k triangles): launch-bound per scene
    "c3s": dict(kind="batch", scenes=256, depth=6, seed=7, sides=[64, 128], spps=[4, 16], tris=[1e3, 5e4]),
    # the RayTrace program's PathTracer (Vulkan shaders restated in CUDA) with its own renderer file
    # settings (res/renderer/path_tracer.renderer: visionJumpCount 5, visionRayPerPixelCount 13) on
    # the Cornell scene at 1920x1080, and on the terrain scene
    # (launch shape: refill / shading batch / blocks per SM measured best per scene)
    "c6": dict(kind="cornell", renderer="rt", W=1920, H=1080, spp=13, depth=5, seed=1, refill=4, shade_batch=16,
               blocks_per_sm=6),
    # the same at 480x270, for profiler captures of single kernel launches
    "c6s": dict(kind="cornell", renderer="rt", W=480, H=270, spp=13, depth=5, seed=1),
    "c6t": dict(kind="terrain", renderer="rt", cells=1024, tile=16, spheres=64, subdiv=4, lights=4, W=1920, H=1080,
                spp=13, depth=5, seed=2024, refill=2, shade_batch=8, blocks_per_sm=0),
    # moving objects: the terrain scene with its 64 spheres on a seeded random walk, one refit
    # (swr_scene_set_transforms) and one 1920x1080 x 16 spp render per frame
    "c7": dict(kind="animate", cells=1024, tile=16, spheres=64, subdiv=4, lights=4, W=1920, H=1080, spp=16,
               depth=8, seed=2024, step=0.01),
    # the same scene with a 480x270 x 4 spp image, for profiler captures of the update and
    # device-builder kernels (about 2 GB on the device)
    "c7s": dict(kind="animate", cells=1024, tile=16, spheres=64, subdiv=4, lights=4, W=480, H=270, spp=4,
                depth=8, seed=2024, step=0.01),
    # differentiable: tessellated Cornell (~49k triangles), 512x512, 32 spp primal + 32 spp adjoint, depth 6
    "c4": dict(kind="diff", W=512, H=512, spp=32, depth=6, seed=11),
    # batched inverse rendering: 64 scenes (5k-200k triangles, 128^2-512^2), 16 spp primal/adjoint, depth 5,
    # per-triangle albedo from a seeded random start by 200 Adam steps (lr 1e-2)
    "c5": dict(kind="inverse", scenes=64, tris=[5e3, 2e5], sides=[128, 256, 512], spp=16, depth=5, adam_steps=200,
               lr=1e-2, target_spp=64, seed=13),
}
METRIC = "Msamples/s (camera paths per second)"


def make_scene(cfg, root):
    from master_thesis_b200 import scenes
    if cfg["kind"] == "terrain":
        return scenes.terrain(cfg["seed"], root, cells=cfg["cells"], tile=cfg["tile"], spheres=cfg["spheres"],
                              sphere_subdiv=cfg["subdiv"], lights=cfg["lights"])
    return scenes.cornell(cfg["seed"], root)


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples taken while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()
        # nvidia-smi's start-up (driver and NVML initialisation) stalls this process's CUDA calls
        # for up to ~0.1 s: wait for its first sample so the start-up falls before the timed region
        t0 = time.time()
        while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
            time.sleep(0.01)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        loaded = [x for x in sm if x > 0.5 * max(sm)] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per traced ray of the bounce traversal kernel, from the committed summary of one
    ncu capture of a full-queue launch on the terrain scene (profiles/k_trace_terrain.json)."""
    p = os.path.join(ROOT, "profiles", "k_trace_terrain.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def cpu_reference(cfg, files, threads, target_s, impl_bin, timed=1, warm=0):
    """Times the reference's own PathTracer or BidirectionalPathTracer (unmodified sources) on a
    bounded pixel sample (every k-th pixel of the image), sized by an untimed probe inside the same
    process so that one pass takes about target_s; `warm` untimed and `timed` timed passes over
    that sample follow one scene load."""
    W, H, spp, depth = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"]
    extra = ["fast"] if cfg["kind"] == "terrain" else []
    if cfg.get("renderer") == "bdpt":
        extra += ["bdpt", str(cfg["light_jumps"]), str(cfg["max_depth"])]
    extra += ["passes", str(timed), str(warm), "target", str(target_s)]
    out = subprocess.run([impl_bin, files["basepath"], files["scene"], files["camera"], str(W), str(H), str(spp),
                          str(depth), str(threads), str(W * H)] + extra, capture_output=True, text=True,
                         timeout=3600)
    if out.returncode != 0:
        raise RuntimeError("ref_bench failed: " + out.stderr[-2000:])
    return json.loads(out.stdout.strip().splitlines()[-1])


def scene_objects(scene_path):
    """Number of objects a scene file lists (entries start at column 0, keys are indented)."""
    with open(scene_path) as f:
        return sum(1 for line in f if line.strip() and not line[0].isspace())


def bench_config(cfg, files, world, workload, split="images"):
    """The `config` object of the JSON line; both arms print the identical dict."""
    W, H = cfg["W"], cfg["H"]
    par = {"images": "independent images per GPU", "spp": "one image split by sample range over GPUs "
           "(all_reduce of the image)", "tiles": "one image split by pixel tile over GPUs (all_gather)"}[split]
    c = {"workload": workload, "objects": scene_objects(files["scene"]), "pixels": W * H, "spp": cfg["spp"],
         "depth": cfg["depth"], "l2": "flushed between steps (256 MB write)",
         "parallelism": par if world > 1 else "single GPU"}
    if "triangles" in files:
        c["triangles"] = int(files["triangles"])
    if cfg.get("renderer") == "bdpt":
        c.update(vision_jumps=cfg["depth"], light_jumps=cfg["light_jumps"], max_depth=cfg["max_depth"])
    elif cfg.get("renderer") != "rt":
        c["wave_size"] = cfg.get("wave_size", 0) or (1 << 23)
    return c


def traversal_microbench(scene, sd, n, steps, flush, stream):
    """Closest-hit queries only (swr_trace_closest on device buffers): n rays with origins uniform
    in the scene's bounding box and directions uniform on the sphere. Hit ids of these rays are
    checked against the oracle by tests/test_gpu_trace.py."""
    import torch
    from master_thesis_b200 import scenes
    ro, rd = scenes.uniform_rays(n, sd.vpos.min(0), sd.vpos.max(0), seed=16)
    hits = torch.empty((n, 4), dtype=torch.int32, device="cuda")
    counts = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    scene.trace(ro, rd, out=hits, counts=counts, stream=stream)  # node/triangle counts (untimed)
    torch.cuda.synchronize()
    nodes = float(counts[:, 0].double().mean())
    tris = float(counts[:, 1].double().mean())
    miss = float((hits[:, 0] == -1).double().mean())
    for _ in range(3):
        scene.trace(ro, rd, out=hits, stream=stream)
    ms = []
    for _ in range(max(steps, 1)):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        scene.trace(ro, rd, out=hits, stream=stream)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    t = sum(ms) / len(ms)
    per_ray = 32 + 16 + 80 * nodes + 48 * tris
    peak, peak_kind = measured_peaks()
    achieved = n * per_ray / (t / 1e3) / 1e9
    return {"rays": n, "mrays_per_s": n / (t / 1e3) / 1e6, "ms_per_launch": t, "miss_fraction": miss,
            "node_visits_per_ray": nodes, "tri_tests_per_ray": tris,
            "roofline": {"bound": "hbm", "kernel": "k_trace_closest", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "algorithmic_bytes_per_ray": per_ray}}


def _events_ms(fn, steps, flush):
    import torch
    total = 0.0
    for _ in range(steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total / steps


def batch_vs_per_scene(args, cfg, tune):
    """One batch of cfg's scenes: the batched wavefront against one single-scene render call per
    scene, both timed with CUDA events (L2 flushed between steps); returns a dict."""
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import autotune, scenes
    rng = np.random.default_rng(cfg["seed"])
    jobs, datas, t0 = [], [], time.time()
    tris = 0
    for k in range(cfg["scenes"]):
        n = int(np.exp(rng.uniform(np.log(cfg["tris"][0]), np.log(cfg["tris"][1]))))
        side = int(rng.choice(cfg["sides"]))
        spp = int(rng.choice(cfg["spps"]))
        sd, cam = scenes.random_scene(cfg["seed"] * 100003 + k, n)
        datas.append(sd)
        tris += sd.num_triangles
        jobs.append(dict(cam=swr.make_camera(cam["position"], cam["angle"], side, side, fov_deg=40),
                         width=side, height=side, spp=spp, depth=cfg["depth"], seed=k, mode=swr.MODE_PHYSICAL))
    # with --tune, the tree options (BVH width, leaf size) of every scene are picked on the batch
    build_opts = autotune.tune_batch_build(datas, jobs) if tune else {}
    jobs = [dict(j, scene=swr.Scene(sd, **build_opts)) for j, sd in zip(jobs, datas)]
    setup_s = time.time() - t0
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    outs = [torch.empty((j["height"], j["width"], 3), dtype=torch.float32, device="cuda") for j in jobs]
    jobs = [dict(j, out=o) for j, o in zip(jobs, outs)]
    batch = swr.Batch()
    launch = autotune.tune_batch(batch, jobs) if tune else {}
    tuned = {"build": build_opts, "launch": launch} if tune else {}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    if args.no_graph:  # the rounds launched from the host (kernels visible to a profiler one by one)
        launch = dict(launch, use_graph=False)
    for _ in range(max(args.warmup, 3)):
        batch.render(jobs, **launch)
    b_ms = _events_ms(lambda: batch.render(jobs, **launch), args.steps, flush)
    batched = [o.clone() for o in outs]

    def per_scene():
        for j in jobs:
            j["scene"].render(j["cam"], j["width"], j["height"], j["spp"], j["depth"], seed=j["seed"], mode=j["mode"],
                              out=j["out"])
    per_scene()
    s_ms = _events_ms(per_scene, args.steps, flush)
    diff = max(float((a - b).abs().max() / b.abs().max().clamp_min(1e-12)) for a, b in zip(batched, outs))
    batch.close()
    for j in jobs:
        j["scene"].close()
    return {"workload": "%d scenes, %d triangles, %d samples, depth %d, physical mode" %
                        (len(jobs), tris, samples, cfg["depth"]),
            "msamples_per_s": samples / (b_ms / 1e3) / 1e6, "ms_per_step": b_ms, "tuned": tuned,
            "per_scene_launches": {"msamples_per_s": samples / (s_ms / 1e3) / 1e6, "ms_per_step": s_ms},
            "speedup_vs_per_scene": s_ms / b_ms, "max_rel_image_diff_vs_per_scene": diff, "setup_s": setup_s}


def run_batch(args, cfg):
    """C3: all scenes in one batched wavefront vs one single-scene render call per scene; the line
    also carries the same comparison on the batch restricted to small jobs (configuration c3s)."""
    main = batch_vs_per_scene(args, cfg, args.tune)
    small = batch_vs_per_scene(args, CONFIGS["c3s"], args.tune) if cfg is not CONFIGS["c3s"] else None
    print(json.dumps({
        "metric": "Msamples/s (batched, %d scenes)" % cfg["scenes"], "value": main["msamples_per_s"],
        "unit": "Msamples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": main["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded in-memory scenes)",
        "config": {"workload": main["workload"], "tuned": main["tuned"]},
        "per_scene_launches": {"value": main["per_scene_launches"]["msamples_per_s"],
                               "ms_per_step": main["per_scene_launches"]["ms_per_step"]},
        "speedup_vs_per_scene": main["speedup_vs_per_scene"],
        "max_rel_image_diff_vs_per_scene": main["max_rel_image_diff_vs_per_scene"], "setup_s": main["setup_s"],
        "small_job_batch": small}))


def run_bdpt(args, cfg, files, workload):
    """Bidirectional tracer: K timed images (L2 flushed before each) and the same through a host
    output buffer; the reference's own BidirectionalPathTracer timed on the host cores beside it."""
    import torch
    import master_thesis_b200 as swr
    W, H, spp, vj, lj, md = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"], cfg["light_jumps"], cfg["max_depth"]
    sd = swr.load_scene(files["scene"], files["basepath"])
    sc = swr.Scene(sd)
    cam = swr.load_camera(files["camera"], W, H)
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    render = lambda o, seed: sc.render_bdpt(cam, W, H, spp, vj, lj, md, seed=seed, out=o, stream=stream)
    for k in range(max(args.warmup, 3)):
        render(out, k)
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms = []
    for k in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        render(out, 100 + k)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    host = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True).numpy()
    for k in range(max(args.warmup, 3)):
        render(host, 300 + k)
    torch.cuda.synchronize()
    e2e = []
    for k in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        render(host, 200 + k)
        e1.record(stream)
        e1.synchronize()
        e2e.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    samples = W * H * spp
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import refdump
        if os.path.exists(refdump.REF_BENCH):
            r = cpu_reference(cfg, files, os.cpu_count() or 1, args.cpu_budget, refdump.REF_BENCH)
            cpu = {"value": r["msamples_per_s"], "unit": "Msamples/s", "cores": os.cpu_count() or 1,
                   "kind": "reference", "sample": "%d of %d pixels (every k-th), %d spp" % (r["pixels"], W * H, spp)}
    t = sum(ms) / len(ms)
    print(json.dumps({
        "metric": "Msamples/s (bidirectional path tracer)", "value": samples / (t / 1e3) / 1e6, "unit": "Msamples/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene files)",
        "config": bench_config(cfg, files, 1, workload),
        "e2e": {"value": samples / (sum(e2e) / len(e2e) / 1e3) / 1e6, "unit": "Msamples/s", "h2d_bytes_per_step": 96,
                "d2h_bytes_per_step": W * H * 12},
        "clocks": clk, "cpu_baseline": cpu}))


def rt_cpu_port(cfg, files, threads, target_s, timed=1, warm=0):
    """The oracle's CPU restatement of the RayTrace PathTracer timed on whole image rows through the
    image centre (all host threads): an untimed probe row sizes the sample so that one pass takes
    about target_s, then `warm` untimed and `timed` timed passes over it."""
    import master_thesis_b200 as swr
    from oracle import oracle as O
    W, H, spp, vj = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"]
    sd = swr.load_scene(files["scene"], files["basepath"])
    cam = swr.load_camera(files["camera"], W, H)
    vi, pi, org = swr.camera_arrays(cam)
    osc, ocam = O.OracleScene.from_scene_data(sd), O.camera(vi, pi, org)
    mid = (H // 2) * W
    t0 = time.time()
    O.rt_render(osc, ocam, W, H, spp, vj, mid, mid + W, threads=threads)
    rate = W / max(time.time() - t0, 1e-6)
    rows = int(max(1, min(H, target_s * rate / W)))
    p0 = max(0, (H - rows) // 2) * W
    for _ in range(warm):
        O.rt_render(osc, ocam, W, H, spp, vj, p0, p0 + rows * W, threads=threads)
    pass_s = []
    for _ in range(timed):
        t0 = time.time()
        O.rt_render(osc, ocam, W, H, spp, vj, p0, p0 + rows * W, threads=threads)
        pass_s.append(time.time() - t0)
    dt = sum(pass_s)
    return {"msamples_per_s": rows * W * spp * timed / dt / 1e6, "pixels": rows * W, "rows": rows, "seconds": dt,
            "pass_s": pass_s, "timed_passes": timed, "warmup_passes": warm}


def reference_line(args, cfg, files, workload, metric, r, kind, sample):
    """The reference arm's JSON line: one step = one pass over the bounded pixel sample, timed on
    the host cores; steps/warmup are the passes actually run."""
    W, H, spp = cfg["W"], cfg["H"], cfg["spp"]
    v = r["msamples_per_s"]
    nproc = os.cpu_count() or 1
    pass_ms = [1e3 * x for x in r["pass_s"]]
    return {
        "impl": "reference", "metric": metric, "value": v, "unit": "Msamples/s", "n_gpus": args.gpus,
        "steps": r["timed_passes"], "warmup": r["warmup_passes"], "ms_per_step": sum(pass_ms) / len(pass_ms),
        "step": "one pass over the sampled pixels (%d of %d, %d spp each)" % (r["pixels"], W * H, spp),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene files)",
        "config": bench_config(cfg, files, args.gpus, workload, args.split if args.gpus > 1 else "images"),
        "sample_pixels": r["pixels"],
        "full_image_ms_estimate": W * H * spp / (v * 1e6) * 1e3,
        "cpu_baseline": {"value": v, "unit": "Msamples/s", "cores": nproc, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": "Msamples/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def reference_pass_target(args):
    """Seconds per reference pass: about a minute of CPU rendering for the whole run."""
    return min(10.0, max(0.2, 60.0 / max(1, args.steps + args.warmup)))


def run_rt(args, cfg, files, workload):
    """RayTrace PathTracer frames (the LCG is seeded by the pixel, so every frame is the same
    image): K timed frames with L2 flushed before each, the same through a pinned host output
    buffer (swr_rt_render_frame, device->host copy inside), and the two denoisers on the frame."""
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import rt
    W, H, spp, vj = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"]
    t0 = time.time()
    sd = swr.load_scene(files["scene"], files["basepath"])
    t1 = time.time()
    sc = swr.Scene(sd)
    torch.cuda.synchronize()
    t2 = time.time()
    cam = swr.load_camera(files["camera"], W, H)
    rgba = torch.empty((H, W, 4), dtype=torch.uint8, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    params = dict(vision_jumps=vj, spp=spp, denoisers=[])
    shape = dict(refill=cfg.get("refill", 0), shade_batch=cfg.get("shade_batch", 0),
                 blocks_per_sm=cfg.get("blocks_per_sm", 0))
    frame = lambda out: rt.render_frame(sc, cam, W, H, params, out=out, stream=stream, **shape)
    for _ in range(max(args.warmup, 3)):
        frame(rgba)
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    ms = _events_ms(lambda: frame(rgba), args.steps, flush)
    host = torch.empty((H, W, 4), dtype=torch.uint8, pin_memory=True).numpy()
    for _ in range(max(args.warmup, 3)):
        frame(host)
    e2e = _events_ms(lambda: frame(host), args.steps, flush)
    den = torch.empty_like(rgba)
    for _ in range(max(args.warmup, 3)):
        rt.denoise_gauss(rgba, 5, 1.0, out=den, stream=stream)
        rt.denoise_median(rgba, out=den, stream=stream)
    g_ms = _events_ms(lambda: rt.denoise_gauss(rgba, 5, 1.0, out=den, stream=stream), args.steps, flush)
    m_ms = _events_ms(lambda: rt.denoise_median(rgba, out=den, stream=stream), args.steps, flush)
    clk = clocks.stop()
    samples = W * H * spp
    cpu = None
    if not args.no_cpu_baseline:
        nproc = os.cpu_count() or 1
        r = rt_cpu_port(cfg, files, nproc, args.cpu_budget)
        cpu = {"value": r["msamples_per_s"], "unit": "Msamples/s", "cores": nproc, "kind": "port",
               "sample": "%d image rows through the centre (%d of %d pixels), %d spp, the oracle's C restatement "
                         "on %d threads" % (r["rows"], r["pixels"], W * H, spp, nproc)}
    peak, peak_kind = measured_peaks()
    img_bytes = W * H * 8  # one rgba8 image read and one written
    print(json.dumps({
        "metric": "Msamples/s (RayTrace PathTracer frame)", "value": samples / (ms / 1e3) / 1e6,
        "unit": "Msamples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene files)",
        "config": bench_config(cfg, files, 1, workload), "launch": shape,
        "e2e": {"value": samples / (e2e / 1e3) / 1e6, "unit": "Msamples/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": W * H * 4},
        "gpu_launches": 1 * args.steps,
        "roofline": None,
        "roofline_note": "k_rt_path: the scene's nodes and triangles stay in L1/L2 (no HBM bound); see the "
                         "denoisers for the memory-bound kernels",
        "denoisers": {"gauss_5_ms": g_ms, "median_ms": m_ms,
                      "gauss_5_frac_of_hbm": img_bytes / (g_ms / 1e3) / 1e9 / peak,
                      "median_frac_of_hbm": img_bytes / (m_ms / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
        "clocks": clk, "cpu_baseline": cpu,
        "setup_s": {"load": t1 - t0, "build_upload": t2 - t1}}))


def run_animate(args, cfg):
    """Moving objects: per frame, new placements for the spheres (a seeded random walk), the GPU
    transform + BVH refit, and a render; against the same frames with the BVH rebuilt on the
    device from the moved scene's data each frame."""
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    tmp = args.scene_dir or tempfile.mkdtemp(prefix="swr_bench_c7_")
    s = scenes.terrain(cfg["seed"], tmp, cells=cfg["cells"], tile=cfg["tile"], spheres=cfg["spheres"],
                       sphere_subdiv=cfg["subdiv"], lights=cfg["lights"])
    t0 = time.time()
    sc = swr.Scene.from_file(s["scene"], s["basepath"], builder="device")
    torch.cuda.synchronize()
    t1 = time.time()
    W, H, spp, depth = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"]
    cam = swr.load_camera(s["camera"], W, H)
    xf0 = sc.transforms()
    tiles = (cfg["cells"] // cfg["tile"]) ** 2
    movers = np.arange(tiles, tiles + cfg["spheres"])
    rng = np.random.default_rng(cfg["seed"])
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    frames = []
    xf = xf0.copy()
    for _ in range(max(args.warmup, 3) + args.steps):
        xf[movers, :3] += rng.normal(scale=cfg["step"], size=(len(movers), 3)).astype(np.float32)
        frames.append(xf.copy())
    for f in frames[:max(args.warmup, 3)]:
        sc.set_transforms(f, stream=stream)
        sc.render(cam, W, H, spp, depth, seed=1, out=out, stream=stream)
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    refit_ms, render_ms = [], []
    for f in frames[max(args.warmup, 3):]:
        flush.fill_(1.0)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        sc.set_transforms(f, stream=stream)
        e1.record(stream)
        sc.render(cam, W, H, spp, depth, seed=1, out=out, stream=stream)
        e2.record(stream)
        e2.synchronize()
        refit_ms.append(e0.elapsed_time(e1))
        render_ms.append(e1.elapsed_time(e2))
    clk = clocks.stop()
    # the last frame's placements with a BVH built from scratch (device builder), for the tree
    # quality after the moves and the rebuild time a refit replaces
    sd = sc.data
    moved = sc.transforms()
    path = os.path.join(tmp, "moved.scene")
    text = open(s["scene"]).read().split("\n")
    k, lines = -1, []
    for line in text:
        if line and not line.startswith("\t"):
            k += 1
        if line.startswith("\tposition("):
            line = "\tposition(%s, %s, %s)" % tuple(scenes._fmt(x) for x in moved[k, :3])
        lines.append(line)
    with open(path, "w") as fh:
        fh.write("\n".join(lines))
    sdm = swr.load_scene(path, s["basepath"])
    torch.cuda.synchronize()
    t2 = time.time()
    fresh = swr.Scene(sdm, builder="device")
    torch.cuda.synchronize()
    t3 = time.time()
    fresh_ms = _events_ms(lambda: fresh.render(cam, W, H, spp, depth, seed=1, out=out, stream=stream), args.steps,
                          flush)
    samples = W * H * spp
    step_ms = (sum(refit_ms) + sum(render_ms)) / args.steps
    print(json.dumps({
        "metric": "Msamples/s (moving objects: refit + render per frame)", "value": samples / (step_ms / 1e3) / 1e6,
        "unit": "Msamples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded scene files)",
        "config": {"workload": "terrain %d^2 cells + %d icospheres moving (random walk, sigma %.3g per frame) + %d "
                               "lights, %dx%d, %d spp, depth %d" % (cfg["cells"], cfg["spheres"], cfg["step"],
                                                                     cfg["lights"], W, H, spp, depth),
                   "triangles": int(sd.num_triangles), "objects": int(sd.num_objects),
                   "l2": "flushed between frames (256 MB write)"},
        "refit_ms": sum(refit_ms) / args.steps, "render_ms": sum(render_ms) / args.steps,
        "render_ms_fresh_tree": fresh_ms, "device_rebuild_s": t3 - t2, "setup_s": t1 - t0,
        "clocks": clk}))


def run_diff(args, cfg):
    """C4: physical-mode primal render vs the path-replay adjoint of an L2 image loss."""
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    tmp = args.scene_dir or tempfile.mkdtemp(prefix="swr_bench_c4_")
    s = scenes.cornell_tessellated(cfg["seed"], tmp)
    sd = swr.load_scene(s["scene"], s["basepath"])
    sc = swr.Scene(sd)
    W, H, spp, depth = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"]
    cam = swr.load_camera(s["camera"], W, H, use_fov_key=True)
    rng = np.random.default_rng(cfg["seed"])
    hidden = torch.from_numpy(rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)).cuda()
    guess = torch.from_numpy(rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)).cuda()
    sc.set_albedo(hidden)
    target = sc.render(cam, W, H, spp, depth, seed=99, mode=swr.MODE_PHYSICAL)
    sc.set_albedo(guess)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")

    def primal():
        sc.render(cam, W, H, spp, depth, seed=1, mode=swr.MODE_PHYSICAL, out=out)
    for _ in range(max(args.warmup, 3)):
        primal()
    p_ms = _events_ms(primal, args.steps, flush)
    dl = (2.0 * (out - target) / out.numel()).contiguous()

    def adjoint():
        sc.render_adjoint(cam, W, H, spp, depth, dl, seed=1)
    for _ in range(max(args.warmup, 3)):
        adjoint()
    a_ms = _events_ms(adjoint, args.steps, flush)
    print(json.dumps({
        "metric": "Msamples/s (physical primal)", "value": W * H * spp / (p_ms / 1e3) / 1e6, "unit": "Msamples/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": p_ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene files)",
        "config": {"workload": "tessellated cornell %d triangles, %dx%d, %d spp, depth %d" %
                   (sd.num_triangles, W, H, spp, depth)},
        "adjoint_ms": a_ms, "adjoint_over_primal": a_ms / p_ms}))


def run_inverse(args, cfg):
    """C5: per-triangle albedo of many scenes recovered by Adam through the batched autograd
    Function (one primal batch launch and one adjoint batch launch per step)."""
    import torch
    import master_thesis_b200 as swr
    from master_thesis_b200 import scenes
    from master_thesis_b200.diff import render_physical_batch
    rng = np.random.default_rng(cfg["seed"])
    jobs, hidden, emis = [], [], []
    t0 = time.time()
    for k in range(cfg["scenes"]):
        n = int(np.exp(rng.uniform(np.log(cfg["tris"][0]), np.log(cfg["tris"][1]))))
        side = int(rng.choice(cfg["sides"]))
        sd, cam = scenes.random_scene(cfg["seed"] * 7919 + k, n)
        sc = swr.Scene(sd)
        jobs.append(dict(scene=sc, cam=swr.make_camera(cam["position"], cam["angle"], side, side, fov_deg=40),
                         width=side, height=side, spp=cfg["spp"], depth=cfg["depth"], seed=0))
        hidden.append(torch.from_numpy(rng.uniform(0.1, 0.9, (sd.num_triangles, 3)).astype(np.float32)).cuda())
        emis.append(torch.from_numpy((sd.materials["color"] * sd.materials["light_strength"][:, None])
                                     .astype(np.float32)).cuda())
    setup_s = time.time() - t0
    tris = sum(j["scene"].data.num_triangles for j in jobs)
    samples = sum(j["width"] * j["height"] * j["spp"] for j in jobs)
    batch = swr.Batch()
    with torch.no_grad():  # targets: the hidden albedo rendered at higher spp with other seeds
        for j, a, e in zip(jobs, hidden, emis):
            j["scene"].set_albedo(a)
            j["scene"].set_emission(e)
        targets = batch.render([dict(j, spp=cfg["target_spp"], seed=10 ** 6 + k, mode=swr.MODE_PHYSICAL)
                                for k, j in enumerate(jobs)])
        targets = [t.clone() for t in targets]
    init = [torch.from_numpy(np.random.default_rng(cfg["seed"] + 1 + k).uniform(0.1, 0.9, tuple(h.shape))
                             .astype(np.float32)).cuda() for k, h in enumerate(hidden)]
    params = [a.clone().requires_grad_() for a in init]
    opt = torch.optim.Adam(params, lr=cfg["lr"])
    seen = [torch.zeros(h.shape[0], dtype=torch.bool, device="cuda") for h in hidden]

    def step(i):
        for k, j in enumerate(jobs):
            j["seed"] = 2 * (i * len(jobs) + k)
        opt.zero_grad(set_to_none=True)
        imgs = render_physical_batch(batch, jobs, params, emis, adjoint_seeds=[j["seed"] + 1 for j in jobs])
        loss = sum(((im - t) ** 2).mean() for im, t in zip(imgs, targets))
        loss.backward()
        for s_, p in zip(seen, params):
            s_ |= (p.grad != 0).any(dim=1)
        opt.step()
        with torch.no_grad():
            for p in params:
                p.clamp_(0.0, 1.0)
        return loss

    def rmse(only_seen):
        num, den = 0.0, 0
        for p, h, s_ in zip(params, hidden, seen):
            d = (p.detach() - h)[s_] if only_seen else (p.detach() - h)
            num += float((d.double() ** 2).sum())
            den += d.numel()
        return (num / max(den, 1)) ** 0.5

    def coverage(j):
        # pixels whose primary ray (pixel centre) hits each triangle first
        vi, pi, org = swr.camera_arrays(j["cam"])
        ys, xs = np.mgrid[0:j["height"], 0:j["width"]]
        v = np.stack([(2 * (xs + 0.5) / j["width"] - 1).ravel(), (2 * (ys + 0.5) / j["height"] - 1).ravel(),
                      np.ones(xs.size), np.ones(xs.size)], 1)
        t = (v @ pi.astype(np.float64))[:, :3]
        t /= np.linalg.norm(t, axis=1, keepdims=True)
        d = (np.concatenate([t, np.zeros((len(t), 1))], 1) @ vi.astype(np.float64))[:, :3]
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        ro = np.zeros((len(d), 4), np.float32)
        ro[:, :3] = org
        rd = np.zeros((len(d), 4), np.float32)
        rd[:, :3] = d
        tri = j["scene"].trace(ro, rd)[:, 0]
        tri = tri[tri != 0xFFFFFFFF].astype(np.int64)
        return torch.from_numpy(np.bincount(tri, minlength=j["scene"].data.num_triangles)).cuda()
    cover = [coverage(j) for j in jobs]

    def rmse_covered(ps, min_px):
        num, den = 0.0, 0
        for p, h, c in zip(ps, hidden, cover):
            d = (p.detach() - h)[c >= min_px]
            num += float((d.double() ** 2).sum())
            den += d.numel()
        return (num / max(den, 1)) ** 0.5

    def rmse_weighted(ps):
        # squared albedo error weighted by the pixels whose primary ray sees each triangle: what an
        # image loss can recover
        num, den = 0.0, 0.0
        for p, h, c in zip(ps, hidden, cover):
            w = c.double()
            num += float((w[:, None] * (p.detach() - h).double() ** 2).sum())
            den += 3.0 * float(w.sum())
        return (num / max(den, 1.0)) ** 0.5

    # parameter snapshots for the recovery curve (device copies, evaluated after the timed loop)
    marks = sorted({0, 25, 50, 100, 150, cfg["adam_steps"]})
    snaps = {0: [a.clone() for a in init]}
    warm = max(args.warmup, 3)
    first = None
    for i in range(warm):
        loss = step(i)
        first = float(loss.detach()) if first is None else first
        if i + 1 in marks:
            snaps[i + 1] = [p.detach().clone() for p in params]
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    last = None
    for i in range(warm, cfg["adam_steps"]):
        last = step(i)
        if i + 1 in marks:
            snaps[i + 1] = [p.detach().clone() for p in params]
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    curve = [{"step": k, "rmse_all": (sum(float(((a - h).double() ** 2).sum()) for a, h in zip(snaps[k], hidden)) /
                                      sum(h.numel() for h in hidden)) ** 0.5,
              "rmse_coverage_weighted": rmse_weighted(snaps[k]), "rmse_covering_4px": rmse_covered(snaps[k], 4)}
             for k in sorted(snaps)]
    timed = cfg["adam_steps"] - warm
    init_err = [float(((a - h).double() ** 2).sum()) for a, h in zip(init, hidden)]
    init_seen = (sum(float((((a - h)[s_]).double() ** 2).sum()) for a, h, s_ in zip(init, hidden, seen)) /
                 max(1, 3 * sum(int(s_.sum()) for s_ in seen))) ** 0.5
    print(json.dumps({
        "metric": "grad-steps/s (batched inverse rendering, %d scenes)" % len(jobs), "value": timed / (ms / 1e3),
        "unit": "grad-steps/s", "n_gpus": 1, "steps": timed, "warmup": warm, "ms_per_step": ms / timed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded in-memory scenes)",
        "config": {"workload": "%d scenes, %d triangles, %d samples primal + %d adjoint per step, depth %d, "
                               "Adam lr %g, %d steps" % (len(jobs), tris, samples, samples, cfg["depth"], cfg["lr"],
                                                        cfg["adam_steps"])},
        "loss_first_step": first, "loss_last_step": float(last.detach()),
        "albedo_rmse": {"initial_all": (sum(init_err) / sum(h.numel() for h in hidden)) ** 0.5,
                        "final_all": rmse(False), "initial_seen": init_seen, "final_seen": rmse(True),
                        "seen_triangles": int(sum(int(s_.sum()) for s_ in seen)), "triangles": tris,
                        "initial_covering_4px": rmse_covered(init, 4), "final_covering_4px": rmse_covered(params, 4),
                        "triangles_covering_4px": int(sum(int((c >= 4).sum()) for c in cover)),
                        "initial_coverage_weighted": rmse_weighted(init), "final_coverage_weighted":
                            rmse_weighted(params),
                        "triangles_seen_by_primary_rays": int(sum(int((c > 0).sum()) for c in cover)),
                        "curve": curve},
        "msamples_per_s_primal_plus_adjoint": 2 * samples * timed / (ms / 1e3) / 1e6, "setup_s": setup_s}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of reference CPU work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--scene-dir", default=None)
    ap.add_argument("--tune", action="store_true", help="autotune the launch shape (cached) before timing")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch the shade/trace rounds from the host instead of a CUDA graph (for profilers)")
    ap.add_argument("--split", default="images", choices=["images", "spp", "tiles"],
                    help="with N>1: independent images per GPU (weak scaling) or one image split by sample "
                         "range / pixel tile over the GPUs (strong scaling)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if cfg["kind"] in ("batch", "diff", "inverse", "animate"):
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference's software renderer has no batched, "
                                                                  "differentiable or moving-object rendering"}))
            return
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        {"batch": run_batch, "diff": run_diff, "inverse": run_inverse, "animate": run_animate}[cfg["kind"]](args, cfg)
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    W, H, spp, depth = cfg["W"], cfg["H"], cfg["spp"], cfg["depth"]
    workload = ("terrain %dx%d cells (%d tiles) + %d icospheres (subdiv %d) + %d emissive quads, %dx%d, %d spp, "
                "depth %d, reference semantics" % (cfg["cells"], cfg["cells"], (cfg["cells"] // cfg["tile"]) ** 2,
                                                  cfg["spheres"], cfg["subdiv"], cfg["lights"], W, H, spp, depth)
                if cfg["kind"] == "terrain" else
                "cornell 36 tris, %dx%d, %d spp, depth %d, reference semantics" % (W, H, spp, depth))
    bdpt = cfg.get("renderer") == "bdpt"
    rtp = cfg.get("renderer") == "rt"
    metric = "Msamples/s (bidirectional path tracer)" if bdpt else METRIC
    if bdpt:
        workload = "cornell 36 tris, %dx%d, %d spp, bidirectional: vision %d, light %d, maxDepth %d" % (
            W, H, spp, depth, cfg["light_jumps"], cfg["max_depth"])
    if rtp:
        metric = "Msamples/s (RayTrace PathTracer frame)"
        workload = "%s, %dx%d, RayTrace PathTracer: visionJumpCount %d, visionRayPerPixelCount %d" % (
            "cornell 36 tris" if cfg["kind"] == "cornell" else "terrain (as c2)", W, H, depth, spp)
    tmp = args.scene_dir or tempfile.mkdtemp(prefix="swr_bench_")
    files_path = os.path.join(tmp, "files.json")
    if os.path.exists(files_path):
        files = json.load(open(files_path))
    else:
        files = make_scene(cfg, tmp)
        json.dump(files, open(files_path, "w"))
    nproc = os.cpu_count() or 1

    if args.impl == "reference" and rtp:
        # the RayTrace program's shaders need a Vulkan ray tracing pipeline, which this machine
        # cannot bring up: its CPU restatement (the oracle) stands in as the reference arm
        if rank != 0:
            return
        r = rt_cpu_port(cfg, files, nproc, reference_pass_target(args), args.steps, args.warmup)
        sample = "%d image rows (%d of %d pixels), %d spp, %d threads; one pass per step" % (
            r["rows"], r["pixels"], W * H, spp, nproc)
        print(json.dumps(reference_line(args, cfg, files, workload, metric, r, "port", sample)))
        return
    if args.impl == "reference":
        if rank != 0:
            return
        from oracle import refdump
        if not os.path.exists(refdump.REF_BENCH):
            print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_bench was not built"}))
            return
        r = cpu_reference(cfg, files, nproc, reference_pass_target(args), refdump.REF_BENCH, args.steps,
                          args.warmup)
        sample = ("%d of %d pixels (every k-th), %d spp, depth %d, %d threads; one pass per step; reference "
                  "load+build %.1f s" % (r["pixels"], W * H, spp, depth, nproc, r["load_s"]))
        line = reference_line(args, cfg, files, workload, metric, r, "reference", sample)
        line["reference_load_s"] = r["load_s"]
        print(json.dumps(line))
        return

    import torch
    torch.cuda.set_device(local_rank)
    if bdpt:
        run_bdpt(args, cfg, files, workload)
        return
    if rtp:
        run_rt(args, cfg, files, workload)
        return
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        import datetime
        dist = dist_mod
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    import master_thesis_b200 as swr
    from master_thesis_b200 import sharding

    t0 = time.time()
    sd = swr.load_scene(files["scene"], files["basepath"])
    t1 = time.time()
    scene = swr.Scene(sd)
    torch.cuda.synchronize()
    t2 = time.time()
    stats = scene.stats()
    # the same scene through the device builder (timed for the setup report, then released)
    t3 = time.time()
    swr.Scene(sd, builder="device").close()
    torch.cuda.synchronize()
    t4 = time.time()
    cam = swr.load_camera(files["camera"], W, H)
    # launch shape: the configuration's paths in flight, or with --tune the autotuner's tree
    # (BVH width, leaf size; the scene is rebuilt with it) and launch shape (cached per workload)
    shape = {"wave_size": cfg.get("wave_size", 0)}
    tuned = None
    if args.tune:
        from master_thesis_b200 import autotune
        bo = autotune.tune_build(sd, cam, W, H, spp, depth)
        scene.close()
        scene = swr.Scene(sd, **bo)
        torch.cuda.synchronize()
        stats = scene.stats()
        shape = autotune.tune_render(scene, cam, W, H, spp, depth)
        tuned = {"build": bo, "launch": shape}
    if args.no_graph:  # every round launched from the host (kernels visible to a profiler one by one)
        shape = dict(shape, host_loop=True)
    # images: every rank renders its own image (seed 1000 + rank); spp / tiles: all ranks render
    # one image (seed 1000) split by sample range or pixel tile (sharding.render_split)
    split = args.split  # with one GPU a split renders the whole image as its one part
    if split == "spp" and spp < world:
        raise SystemExit("--split spp needs at least one sample per pixel per rank")
    seed = 1000 + rank if split == "images" else 1000
    out = torch.empty((H, W, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def render(o, **kw):
        if split == "images":
            return scene.render(cam, W, H, spp, depth, seed=seed, out=o, stream=stream, return_profile=True,
                                **shape, **kw)
        profile = []

        def part(pb, pc, sb, sc):
            r, pr = scene.render(cam, W, H, sc, depth, seed=seed, stream=stream, return_profile=True,
                                 pixel_begin=pb, pixel_count=pc, sample_begin=sb, spp_total=spp, **shape, **kw)
            profile.append(pr)
            return r.reshape(pc, 3)

        img = sharding.render_split(part, W, H, spp, rank, world, split=split, device="cuda")
        if isinstance(o, np.ndarray):
            torch.from_numpy(o).copy_(img, non_blocking=True)  # pinned host memory
            profile[-1]["d2h_bytes"] = W * H * 12
        else:
            o.copy_(img)
        return o, profile[-1]

    # traffic model: node visits and triangle tests of the bounce traversal (separate, untimed run
    # before the warm-up, so that the timed renders find their launch shape warmed up)
    _, cprof = render(out, count=True)
    torch.cuda.synchronize()
    for _ in range(max(args.warmup, 3)):
        render(out)
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    barrier()
    step_ms, plain = [], []
    for _ in range(args.steps):
        flush.fill_(1.0)  # evict L2 between steps (256 MB > 126 MB L2)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, pr = render(out)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        plain.append(pr)
    barrier()
    # per-kernel device times: the same K renders again with CUDA events around every launch (on
    # the launching stream); kept out of the steps above because the events cost a few us each
    profs = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        _, pr = render(out, profile=True)
        profs.append(pr)
    barrier()
    # end to end: the same call with a pinned host output buffer (warmed up like the device path:
    # the first host-output render allocates the library's staging image)
    host = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True).numpy()
    for _ in range(max(args.warmup, 3)):
        render(host)
    torch.cuda.synchronize()
    e2e_ms, e2e_prof = [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _, pr = render(host)
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
        e2e_prof.append(pr)
    barrier()
    micro = None
    if cfg.get("microbench_rays"):
        micro = traversal_microbench(scene, sd, cfg["microbench_rays"], args.steps, flush, stream)
    barrier()
    clk = clocks.stop()

    # the job's time is the slowest rank's (device time, each rank rendering its own images or
    # its part of the shared image)
    total_ms, total_e2e_ms = sharding.max_over_ranks([sum(step_ms), sum(e2e_ms)])
    samples = W * H * spp * (world if split == "images" else 1) * args.steps
    value = samples / (total_ms / 1e3) / 1e6
    e2e_value = samples / (total_e2e_ms / 1e3) / 1e6

    # roofline of the dominant kernel (bounce traversal): algorithmic bytes per launch =
    # rays * (32 B ray in + 8 B hit out) + node visits * 80 B + triangle tests * 48 B
    launches = sum(p["trace_launches"] for p in profs)
    trace_ms = sum(p["trace_ms"] for p in profs)
    rays_per_step = profs[-1]["bounce_rays"]
    bytes_per_step = rays_per_step * 40 + cprof["node_visits"] * 80 + cprof["tri_tests"] * 48
    per_launch_bytes = bytes_per_step * args.steps / max(launches, 1)
    per_launch_s = trace_ms / 1e3 / max(launches, 1)
    achieved = per_launch_bytes / per_launch_s / 1e9
    peak, peak_kind = measured_peaks()
    tp = profile_traffic()
    traffic = None
    if tp and tp.get("scene") == cfg["kind"]:
        # the captured launch's DRAM bytes per ray, scaled to this run's rays per launch
        traffic = tp["dram_bytes_per_ray"] * rays_per_step * args.steps / max(launches, 1)
    mrays = sum(p["rays"] for p in plain) / (sum(step_ms) / 1e3) / 1e6
    launches_total = sum(p["launches"] for p in plain)

    if rank == 0:
        cpu = cpu_shim = None
        if not args.no_cpu_baseline:
            from oracle import refdump
            if os.path.exists(refdump.REF_BENCH):
                try:
                    r = cpu_reference(cfg, files, nproc, args.cpu_budget, refdump.REF_BENCH)
                    cpu = {"value": r["msamples_per_s"], "unit": "Msamples/s", "cores": nproc, "kind": "reference",
                           "sample": "%d of %d pixels (every k-th), %d spp, depth %d; reference load+build %.1f s"
                                     % (r["pixels"], W * H, spp, depth, r["load_s"])}
                except Exception as ex:  # the baseline is reported, never required
                    cpu = {"value": None, "unit": "Msamples/s", "cores": nproc, "kind": "reference",
                           "sample": "failed: %s" % str(ex)[:200]}
            if os.path.exists(refdump.REF_BENCH_SHIM):
                # second row: the reference's path with the lock-free Philox shim instead of its
                # mutex-guarded generator
                try:
                    r = cpu_reference(cfg, files, nproc, args.cpu_budget / 2, refdump.REF_BENCH_SHIM)
                    cpu_shim = {"value": r["msamples_per_s"], "unit": "Msamples/s", "cores": nproc,
                                "kind": "reference (lock-free Philox RNG shim)",
                                "sample": "%d of %d pixels (every k-th), %d spp, depth %d"
                                          % (r["pixels"], W * H, spp, depth)}
                except Exception as ex:
                    cpu_shim = {"value": None, "sample": "failed: %s" % str(ex)[:200]}
        line = {
            "metric": METRIC, "value": value, "unit": "Msamples/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak" if split == "images" else "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded scene files)",
            "config": bench_config(cfg, files, world, workload, split),
            "bvh": {"nodes": stats["nodes"], "depth": stats["depth"]},
            "tuned": tuned,
            "e2e": {"value": e2e_value, "unit": "Msamples/s",
                    "h2d_bytes_per_step": int(e2e_prof[-1]["h2d_bytes"]),
                    "d2h_bytes_per_step": int(e2e_prof[-1]["d2h_bytes"]),
                    "step_ms": {"min": min(e2e_ms), "median": statistics.median(e2e_ms), "max": max(e2e_ms)}},
            "mrays_per_s": mrays,
            "rays_per_sample": profs[-1]["rays"] / (W * H * spp),
            "first_trace_rays": int(profs[-1]["first_trace_rays"]),
            "roofline": {"bound": "hbm", "kernel": "k_trace (bounce traversal)", "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                         "algorithmic_bytes_per_launch": per_launch_bytes,
                         "node_visits_per_ray": cprof["node_visits"] / max(cprof["bounce_rays"], 1),
                         "tri_tests_per_ray": cprof["tri_tests"] / max(cprof["bounce_rays"], 1)},
            "traversal_microbench": micro,
            "kernel_ms_per_step": {k: sum(p[k] for p in profs) / args.steps for k in
                                   ("trace_ms", "shade_ms", "camera_ms", "resolve_ms")},
            "kernel_timing": "per-kernel CUDA events over K further renders of the same image",
            "gpu_launches": int(launches_total),
            "clocks": clk,
            "cpu_baseline": cpu,
            "cpu_baseline_rng_shim": cpu_shim,
            "setup_s": {"load": t1 - t0, "build_upload": t2 - t1, "build_upload_device_builder": t4 - t3},
        }
        print(json.dumps(line))
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
