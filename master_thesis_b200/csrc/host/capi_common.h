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

}  // namespace swr
