// Shared host helpers of the C ABI implementation.
#pragma once

#include <string>
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

int validate_desc(const swr_scene_desc* d);
void derive(const swr_scene_desc& d, Derived& out);

}  // namespace swr
