// Internal device-side data structures of the path tracer library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../../include/swr.h"
#include "../swr_bvh.cuh"

namespace swr {

int set_error(int code, const std::string& msg);

// Device view of one scene (all pointers are device memory).
struct DevScene {
  const float4* nodes;      // [num_nodes * 5]   wide BVH records
  const float4* tris;       // [num_slots * 3]   v0 | e0 | e1 | id rank obj (swr_bvh.cuh)
  const float4* shade;      // [num_slots * 4]   (d00 d01 d11 denom) (n0 .) (n1 .) (n2 .)
  const float* tri_boxes;   // [num_slots * 6]   reference triangle boxes
  const float* obj_boxes;   // [num_objects * 6] reference object boxes
  const float4* mats;       // [num_objects * 3] (rgb dT) (rT tT eta light) (Le.rgb strength)
  const float* albedo;      // [num_slots * 3]   physical-mode diffuse albedo per triangle slot
  const uint32_t* slot_of;  // [num_tris]        triangle id -> slot
  const uint4* lights;      // [num_lights]      first light triangle, count, object, 0
  const float4* light_tris; // [5 per triangle]  corners v0 v1 v2 and corner normals n0 n1 n2
  uint32_t num_nodes, num_slots, num_objects, num_tris, num_lights;
};

}  // namespace swr

struct swr_scene {
  swr::DevScene dev;
  // owned device allocations
  void* d_nodes = nullptr;
  void* d_tris = nullptr;
  void* d_shade = nullptr;
  void* d_tri_boxes = nullptr;
  void* d_obj_boxes = nullptr;
  void* d_mats = nullptr;
  void* d_albedo = nullptr;
  void* d_slot_of = nullptr;
  void* d_lights = nullptr;
  void* d_light_tris = nullptr;
  void* d_scratch = nullptr;  // small per-scene scratch (work counters)
  size_t scratch_bytes = 0;
  uint32_t depth = 0;
  uint64_t node_bytes = 0, tri_bytes = 0;
  int device = 0;
  int num_sms = 0;
  std::vector<uint32_t> slot_to_id;  // host copy
  void* workspace = nullptr;          // render workspace (render.cu), grown on demand
  void* instance = nullptr;           // object-space data for moving objects (instance.cu)
  void* rt_buf = nullptr;             // RayTrace frames: host-output staging and denoiser
  size_t rt_buf_bytes = 0;            //   ping-pong images (rt.cu), grown on demand
};

namespace swr {

// CUDA error helper: returns SWR_ERR_CUDA with a message when err != cudaSuccess.
int cuda_fail(cudaError_t err, const char* what);

#define SWR_CUDA(call)                                   \
  do {                                                   \
    cudaError_t _e = (call);                             \
    if (_e != cudaSuccess) return swr::cuda_fail(_e, #call); \
  } while (0)

// true when p is host memory that the device cannot address directly
bool is_host_pointer(const void* p);

// releases the render workspace of a scene (render.cu)
void free_workspace(swr_scene* s);
// releases the object-space data of a scene made from a host scene (instance.cu)
void free_instance(swr_scene* s);

}  // namespace swr
