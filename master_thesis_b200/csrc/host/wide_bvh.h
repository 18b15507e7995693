// Host construction of the traversal BVH: binned-SAH binary tree, collapsed into the compressed
// 8-wide node format of swr_bvh.cuh. This is an acceleration structure of this library only;
// the reference's own (agglomerative) tree matters solely for tie order, see ref_bvh.h.
#pragma once

#include <cstdint>
#include <vector>

namespace swr {

struct PrimBox {
  float lo[3], hi[3];
};

struct WideBvhOptions {
  // defaults measured on the terrain image (host SAH tree): 32 bins and cost 0.3 -> 29.24 ms per
  // image, cost 0.8 -> 28.73 ms, 64 bins and cost 0.8 -> 28.53 ms (costs 1.0-1.7 no better)
  uint32_t sah_bins = 64;
  uint32_t max_leaf = 3;       // triangles per leaf child (1..3)
  uint32_t threads = 0;        // 0 = hardware concurrency
  double prim_cost = 0.8;      // SAH cost of a triangle test relative to a wide-node visit
  uint32_t width = 8;          // children per wide node (2..8; the record always has 8 slots)
};

struct WideBvh {
  std::vector<uint32_t> words;     // 20 32-bit words per node (five float4)
  std::vector<uint32_t> prim_order;  // triangle record slot -> primitive index
  uint32_t num_nodes = 0;
  uint32_t depth = 0;              // deepest node level (root = 1)
  uint32_t binary_nodes = 0;
  double sah_cost = 0.0;           // SAH cost of the binary tree (traversal 1, intersection 1)
};

// Boxes must already include whatever safety margin the traversal needs.
WideBvh build_wide_bvh(const std::vector<PrimBox>& prims, const WideBvhOptions& opt);

}  // namespace swr
