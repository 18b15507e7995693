// SoftwareRenderer command-line drop-in (software_renderer/main.cpp:28-87): the same positional
// arguments, the same renderer files (PathTracer and BidirectionalPathTracer), the same base-path
// rule for mesh files and the same P6 output, with the image rendered on the GPU through the C
// ABI instead of by host threads.
//
//   SoftwareRenderer renderer scene image_width image_height thread_count camera resultimage
//
// thread_count sets the host threads of the BVH build (the render itself runs on the GPU).
// The environment variable SWR_SEED (unsigned integer, default 0) selects the random-number
// stream; the reference draws from a shared host generator instead, so its images agree with
// these in distribution, not pixel by pixel. SWR_DEVICE selects the CUDA device (default 0);
// SWR_BUILDER=device builds the BVH on the GPU (same image).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "swr.h"

namespace {

int fail(const char* what) {
  std::cerr << "Error: " << what << ": " << swr_last_error() << std::endl;
  return 1;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

int main(int argc, char* argv[]) {
  if (argc != 8) {
    std::cout << "Error: wrong paramter count!" << std::endl;
    std::cout << "Usage: SoftwareRenderer renderer scene image_width image_height thread_count camera resultimage"
              << std::endl;
    return -1;
  }
  std::cout << argv[0];
  for (int i = 1; i < 7; ++i) std::cout << " " << argv[i];
  std::cout << std::endl;

  // mesh files are found relative to the executable's directory, as in the reference: the
  // executable path minus the length of "SoftwareRenderer"
  const std::string exec = argv[0];
  const size_t name_len = sizeof("SoftwareRenderer") - 1;
  const std::string basepath = exec.size() >= name_len ? exec.substr(0, exec.size() - name_len) : std::string();
  const char* renderer_path = argv[1];
  const char* scene_path = argv[2];
  const uint32_t width = (uint32_t)std::atoi(argv[3]);
  const uint32_t height = (uint32_t)std::atoi(argv[4]);
  const uint32_t threads = (uint32_t)std::atoi(argv[5]);
  const char* camera_path = argv[6];
  const char* out_path = argv[7];
  const char* seed_env = std::getenv("SWR_SEED");
  const uint64_t seed = seed_env ? std::strtoull(seed_env, nullptr, 10) : 0;

  auto t0 = std::chrono::steady_clock::now();
  swr_renderer_params rp;
  if (swr_renderer_load_params(renderer_path, &rp)) return fail("renderer");
  swr_host_scene* hs = nullptr;
  if (swr_host_scene_load(scene_path, basepath.c_str(), &hs)) return fail("scene");
  swr_camera cam;
  if (swr_camera_load(camera_path, width, height, 0, &cam)) return fail("camera");
  swr_scene_desc desc;
  if (swr_host_scene_desc(hs, &desc)) return fail("scene");
  const char* dev_env = std::getenv("SWR_DEVICE");
  if (cudaSetDevice(dev_env ? std::atoi(dev_env) : 0) != cudaSuccess) {
    std::cerr << "Error: no usable CUDA device" << std::endl;
    return 1;
  }
  swr_build_opts bo = {};
  bo.threads = threads;
  const char* builder_env = std::getenv("SWR_BUILDER");
  if (builder_env && std::string(builder_env) == "device") bo.builder = SWR_BUILD_DEVICE;
  swr_scene* scene = nullptr;
  if (swr_scene_create(&desc, &bo, &scene)) return fail("scene build");
  swr_host_scene_free(hs);
  const double t_load = seconds_since(t0);

  t0 = std::chrono::steady_clock::now();
  swr_render_opts ro = {};
  ro.width = width;
  ro.height = height;
  ro.spp = rp.spp;
  ro.max_depth = rp.vision_jumps;
  ro.seed = seed;
  ro.mode = SWR_MODE_REFERENCE;
  std::vector<float> rgb((size_t)width * height * 3);
  if (rp.kind == SWR_RENDERER_BIDIRECTIONAL) {
    swr_bdpt_opts bd = {};
    bd.light_jumps = rp.light_jumps;
    bd.max_depth = rp.max_depth;
    if (swr_render_bdpt(scene, &cam, &ro, &bd, rgb.data(), nullptr, nullptr)) return fail("render");
  } else {
    if (swr_render(scene, &cam, &ro, rgb.data(), nullptr, nullptr)) return fail("render");
  }
  if (swr_sync(nullptr)) return fail("render");
  const double t_render = seconds_since(t0);
  std::cout << "100% done" << std::endl;

  std::vector<uint8_t> rgb8(rgb.size());
  if (swr_quantize_rgb8(rgb.data(), width, height, rgb8.data())) return fail("image");
  if (swr_write_ppm(out_path, rgb8.data(), width, height)) return fail("image");
  swr_scene_destroy(scene);
  std::cout << "load+build " << t_load << " s, render " << t_render << " s" << std::endl;
  return 0;
}
