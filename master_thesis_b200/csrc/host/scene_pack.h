// Host assembly of the device scene records: the wide BVH over conservatively enlarged
// reference boxes, triangle records in leaf order, shading records, boxes and materials.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../../include/swr.h"

namespace swr {

struct PackedScene {
  std::vector<uint32_t> nodes;    // 20 words per wide node
  std::vector<float4> tris;       // 3 per slot: v0|e0|e1|id rank obj
  std::vector<float4> shade;      // 4 per slot: (d00 d01 d11 denom) (n0) (n1) (n2)
  std::vector<float> tri_boxes;   // 6 per slot
  std::vector<float> obj_boxes;   // 6 per object
  std::vector<float4> mats;       // 3 per object
  std::vector<float> albedo;      // 3 per slot
  std::vector<uint32_t> slot_of;  // triangle id -> slot
  std::vector<uint32_t> slot_to_id;
  std::vector<float> prim_boxes;  // without the host BVH: 6 per triangle, the traversal boxes
  // light sources in object order (the reference's lightSources list, mesh_manager.cpp:52-56):
  // 4 words each (first light triangle, triangle count, object, 0), and per light triangle in
  // triangle-id order its corners v0 v1 v2 and corner normals n0 n1 n2 (20 floats, 18 used)
  std::vector<uint32_t> lights;
  std::vector<float4> light_tris;
  uint32_t num_nodes = 0, depth = 0;
};

// Validates and packs; returns SWR_OK or an error code (message in swr_last_error). With
// host_bvh false no BVH is built: the records are in triangle-id order (slot = id) and
// prim_boxes holds the boxes for the caller's builder.
int pack_scene(const swr_scene_desc* d, const swr_build_opts* opts, PackedScene& out, bool host_bvh = true);

}  // namespace swr
