// Exact reproduction of the reference's BVH topology, used only to know the order in which the
// reference visits leaves (its closest-hit ties go to the first leaf in left-first DFS order).
//
// The reference (software_renderer/math/bounding_volume_hierachy.cpp:9-75) builds the tree by
// repeatedly merging the pair of live nodes whose box centres are closest (squared float
// distance, strict <, first pair in list-scan order on ties) and appending the parent at the end
// of the list. That is O(n^2) per merge. This implementation makes the same choices, in about
// O(n^2) total for small inputs and with a kd-tree of the live centres (near O(n log n) on
// spread-out inputs) from kRefIndexedMin boxes on; both are checked against the reference's own
// builder tree by tree, and against each other, in the tests.
#pragma once

#include <cstdint>
#include <vector>

#include "rmath.h"

namespace swr {

struct RefTree {
  // node i < n is leaf i (element i); node n+k is the k-th merge. left/right are -1 for leaves.
  std::vector<int32_t> left, right;
  int32_t root = -1;
};

// kAuto: the kd-tree build from kRefIndexedMin boxes on. The kd-tree build needs every box
// coordinate within +-1e18; other inputs always take the flat build.
enum class RefBuild { kAuto, kFlat, kIndexed };
constexpr int32_t kRefIndexedMin = 1024;

// Builds the tree over the given leaf boxes (in input order) and returns the element indices in
// left-first DFS order. If tree is non-null the full topology is returned too. threads: host
// threads for the kd-tree build's first nearest-node queries (0 = all cores); the rest of the
// build is sequential.
std::vector<uint32_t> ref_bvh_leaf_order(const std::vector<Box>& boxes, RefTree* tree = nullptr,
                                         RefBuild how = RefBuild::kAuto, unsigned threads = 1);

}  // namespace swr
