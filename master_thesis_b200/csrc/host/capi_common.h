// Shared host helpers of the C ABI implementation.
#pragma once

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/swr.h"
#include "rmath.h"

namespace swr {

// Stores msg as the calling thread's last error and returns code.
int set_error(int code, const std::string& msg);

// Per-triangle and per-object data derived from a scene descriptor with the reference's float
// arithmetic (triangle.cpp:4-17 for edges, dot products and boxes; graphics_object.cpp:25 for the
// object box over all of the object's vertices, first one padded).
struct Derived {
  std::vector<V3> v0, e0, e1;
  std::vector<V4> den;  // d00 d01 d11 denom
  std::vector<Box> tri_box;
  std::vector<Box> obj_box;
};

// Runs f(begin, end) over [0, n) in contiguous blocks on up to `threads` host threads (0 = all
// cores); the calling thread takes the first block. For loops whose iterations are independent.
template <class F>
void parallel_for(size_t n, F f, unsigned threads = 0) {
  unsigned nt = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
  const size_t min_block = 4096;
  nt = (unsigned)std::max<size_t>(1, std::min<size_t>(nt, (n + min_block - 1) / min_block));
  if (nt <= 1) {
    f((size_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  const size_t step = (n + nt - 1) / nt;
  for (unsigned t = 1; t < nt; ++t) {
    const size_t b = std::min(n, t * step), e = std::min(n, b + step);
    pool.emplace_back([=] { f(b, e); });
  }
  f((size_t)0, std::min(n, step));
  for (auto& th : pool) th.join();
}

int validate_desc(const swr_scene_desc* d);
void derive(const swr_scene_desc& d, Derived& out);

// What a scene needs on the device to move its objects (swr_scene_set_transforms): the
// object-space meshes, where each world vertex comes from, and each triangle's position in its
// mesh's reference leaf order.
struct InstanceSource {
  std::vector<float> mesh_pos, mesh_nrm;       // [3 * mesh vertices] of all distinct meshes
  std::vector<uint32_t> vert_src, vert_obj;    // per world vertex: mesh vertex, object
  std::vector<uint32_t> obj_first_vertex;      // [objects + 1]
  std::vector<uint32_t> obj_first_tri;         // [objects + 1]
  std::vector<uint32_t> local_rank;            // per triangle id
  std::vector<swr_object_transform> xf;        // placements as loaded
  bool scene_order_exact = true;               // objects few enough for the reference's order
};
void instance_source(const swr_host_scene* hs, InstanceSource& out);
// M = I * S * R * T of a placement (graphics_object.cpp:54-62), row-major m[i*4 + j].
void object_matrix(const swr_object_transform& xf, float m[16]);
// The reference's scene-level leaf order of objects from their boxes (lo.xyz hi.xyz each), or
// the identity order when `exact` is false (too many objects for the reference's builder).
std::vector<uint32_t> object_order(const float* boxes, uint32_t n, bool exact);

}  // namespace swr
