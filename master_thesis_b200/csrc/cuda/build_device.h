// Device construction of the wide BVH (build.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace swr {

struct DeviceBuildOptions {
  uint32_t max_leaf = 3;    // triangles per leaf child (1..3)
  uint32_t radius = 16;     // clustering search radius in Morton order
  double prim_cost = 0.8;   // SAH cost of a triangle test relative to a wide-node visit
  uint32_t width = 8;       // children per wide node (2..8)
};

struct DeviceBvh {
  void* d_nodes = nullptr;           // 20 words per wide node (cudaMalloc; the caller frees)
  uint32_t* d_prim_order = nullptr;  // triangle slot -> primitive (cudaMalloc; the caller frees)
  uint32_t num_nodes = 0, depth = 0, binary_nodes = 0, rounds = 0;
};

// Builds over n conservative primitive boxes (6 floats each, device memory) on `stream`.
int build_wide_bvh_device(const float* d_prim_boxes, uint32_t n, const DeviceBuildOptions& opt, DeviceBvh& out,
                          cudaStream_t stream);

}  // namespace swr
