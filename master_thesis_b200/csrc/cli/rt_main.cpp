// Headless RayTrace command-line drop-in (src/main.cpp:100-239 of the reference's Vulkan program)
// for its PathTracer renderer and its denoisers: the same positional arguments, renderer files,
// scene files, camera files, mesh base-path rule and P6 output, rendered by the CUDA restatement
// of the shaders instead of a Vulkan ray tracing pipeline, with no window.
//
//   RayTrace renderer scene image_width image_height camera [resultimage renderrounds]
//
// With resultimage and renderrounds the program renders renderrounds frames and writes the last
// one to resultimage, as the reference does (its frames are identical: objects do not move when
// a render limit is given, and the PathTracer has no frame-to-frame state). Without them the
// reference opens an interactive window; here one frame is rendered and written where the
// reference's screenshot key writes it, out/<renderer name>_<n>.ppm. The form without a camera
// file is interactive only and is refused. SWR_DEVICE selects the CUDA device (default 0);
// SWR_BUILDER=device builds the BVH on the GPU.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
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

bool exists(const std::string& p) { return std::ifstream(p).good(); }

}  // namespace

int main(int argc, char* argv[]) {
  if (argc != 5 && argc != 6 && argc != 8) {
    std::cout << "Error: wrong paramter count!" << std::endl;
    std::cout << "Usage: RayTrace renderer scene image_width image_height [camera] [resultimage renderrounds]"
              << std::endl;
    return -1;
  }
  std::cout << argv[0];
  for (int i = 1; i < argc; ++i) std::cout << " " << argv[i];
  std::cout << std::endl;
  if (argc == 5) {
    std::cout << "Error: without a camera file RayTrace is interactive; this headless build needs one"
              << std::endl;
    return -1;
  }

  const std::string exec = argv[0];
  const size_t name_len = sizeof("RayTrace") - 1;
  const std::string basepath = exec.size() >= name_len ? exec.substr(0, exec.size() - name_len) : std::string();
  const std::string renderer_path = argv[1];
  const char* scene_path = argv[2];
  const uint32_t width = (uint32_t)std::atoi(argv[3]);
  const uint32_t height = (uint32_t)std::atoi(argv[4]);
  const char* camera_path = argv[5];
  const bool render_limit = argc == 8;
  const unsigned max_render = render_limit ? (unsigned)std::atoi(argv[7]) : 1u;

  // renderer name = file name without directory and extension (src/main.cpp:131-133)
  const size_t start = renderer_path.find_last_of('/') + 1;
  const size_t finish = renderer_path.find_last_of('.') - start;
  const std::string renderer_name = renderer_path.substr(start, finish);

  swr_rt_renderer_params rp;
  if (swr_rt_renderer_load(renderer_path.c_str(), &rp)) return fail("renderer");
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
  const char* builder_env = std::getenv("SWR_BUILDER");
  if (builder_env && std::string(builder_env) == "device") bo.builder = SWR_BUILD_DEVICE;
  swr_scene* scene = nullptr;
  if (swr_scene_create(&desc, &bo, &scene)) return fail("scene build");
  swr_host_scene_free(hs);

  swr_rt_opts ro = {};
  ro.width = width;
  ro.height = height;
  ro.vision_jumps = rp.vision_jumps;
  ro.spp = rp.spp;
  uint8_t* d_img = nullptr;
  const size_t bytes = (size_t)width * height * 4;
  if (cudaMalloc(&d_img, bytes) != cudaSuccess || cudaMemset(d_img, 0, bytes) != cudaSuccess) {
    std::cerr << "Error: device allocation failed" << std::endl;
    return 1;
  }
  for (unsigned r = 0; r < max_render; ++r) {
    const auto t0 = std::chrono::steady_clock::now();
    if (swr_rt_render_frame(scene, &cam, &ro, rp.denoisers, rp.num_denoisers, d_img, nullptr)) return fail("render");
    if (swr_sync(nullptr)) return fail("render");
    const float seconds = std::chrono::duration<float>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Render Time: %f (~%i FPS)\n", seconds, int(1.0f / seconds));
  }
  std::vector<uint8_t> rgba(bytes), rgb((size_t)width * height * 3);
  if (cudaMemcpy(rgba.data(), d_img, bytes, cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::cerr << "Error: image copy failed" << std::endl;
    return 1;
  }
  for (size_t i = 0; i < (size_t)width * height; ++i)
    for (int k = 0; k < 3; ++k) rgb[3 * i + k] = rgba[4 * i + k];
  std::string out_path;
  if (render_limit) {
    std::cout << "Render finished!" << std::endl;
    out_path = argv[6];
  } else {  // screenshot() naming (src/main.cpp:80-88)
    out_path = "out/" + renderer_name + "_0.ppm";
    for (unsigned i = 1; exists(out_path); ++i) out_path = "out/" + renderer_name + "_" + std::to_string(i) + ".ppm";
  }
  if (swr_write_ppm(out_path.c_str(), rgb.data(), width, height)) return fail("image");
  if (!render_limit) std::cout << "Saved screenshot " << out_path << std::endl;
  cudaFree(d_img);
  swr_scene_destroy(scene);
  return 0;
}
