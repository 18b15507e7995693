// Closest-centre agglomerative clustering with the reference's exact tie rules
// (bounding_volume_hierachy.cpp:9-27 findClosestPair, :47-75 BVH::init).
//
// Selection rule being reproduced: among all pairs (i, j) of live nodes with i before j in the
// list (the list is ordered by creation: leaves in input order, then parents as they are made),
// take the smallest squared centre distance; on equal distances the pair that comes first in the
// i-outer / j-inner scan wins. The parent's left child is i, its right child is j, its box is the
// union, and it is appended to the end of the list.
//
// Equivalent formulation used here: every live node k keeps nn[k], the best node after it in
// the list (smallest distance, then earliest), with its distance nd[k]. The reference's choice is
// the k with the smallest (nd[k], position of k), paired with nn[k]. After a merge of (a, b) into
// c, only nodes whose partner was a or b need a rescan; every other node just compares its
// current partner with c (c is last, so it only wins on a strictly smaller distance).
#include "ref_bvh.h"

#include <limits>

namespace swr {

std::vector<uint32_t> ref_bvh_leaf_order(const std::vector<Box>& boxes, RefTree* tree) {
  const int32_t n = (int32_t)boxes.size();
  std::vector<uint32_t> order;
  if (n == 0) return order;
  const int32_t total = 2 * n - 1;
  // List order is creation order (parents are appended), so the live list is the set of live
  // node ids in increasing order: kept as a flat array, with the centres as separate coordinate
  // arrays, so every pass is a linear scan.
  std::vector<float> cx(total), cy(total), cz(total);
  std::vector<Box> box(total);
  std::vector<int32_t> left(total, -1), right(total, -1);
  std::vector<int32_t> nn(total, -1);
  std::vector<float> nd(total, std::numeric_limits<float>::infinity());
  std::vector<int32_t> live(n);
  for (int32_t i = 0; i < n; ++i) {
    box[i] = boxes[i];
    const V3 c = box[i].center();
    cx[i] = c[0];
    cy[i] = c[1];
    cz[i] = c[2];
    live[i] = i;
  }
  // squared centre distance, summed from +0 in x, y, z order (vector.h:227-241)
  auto d2 = [&](int32_t a, int32_t b) {
    const float dx = cx[a] - cx[b], dy = cy[a] - cy[b], dz = cz[a] - cz[b];
    float s = 0.0f;
    s += dx * dx;
    s += dy * dy;
    s += dz * dz;
    return s;
  };
  // best later partner of the node at live position p: smallest distance, then earliest
  auto rescan = [&](size_t p) {
    const int32_t k = live[p];
    int32_t best = -1;
    float bd = std::numeric_limits<float>::infinity();
    for (size_t q = p + 1; q < live.size(); ++q) {
      const float d = d2(k, live[q]);
      if (d < bd) {
        bd = d;
        best = live[q];
      }
    }
    nn[k] = best;
    nd[k] = bd;
  };
  for (size_t p = 0; p < live.size(); ++p) rescan(p);
  // the first live node with the smallest partner distance
  int32_t a = -1;
  {
    float best = std::numeric_limits<float>::infinity();
    for (int32_t k : live)
      if (nn[k] >= 0 && nd[k] < best) {
        best = nd[k];
        a = k;
      }
  }
  for (int32_t c = n; c < total; ++c) {
    if (a < 0) {
      // every remaining distance is NaN or infinite: the reference's scan finds no pair (its
      // iterators stay unset); merge the first two live nodes so the build still terminates.
      a = live[0];
      nn[a] = live[1];
    }
    const int32_t b = nn[a];
    left[c] = a;
    right[c] = b;
    box[c] = Box::merge(box[a], box[b]);
    const V3 cc = box[c].center();
    cx[c] = cc[0];
    cy[c] = cc[1];
    cz[c] = cc[2];
    // unlink a and b, append c
    size_t w = 0;
    for (size_t r = 0; r < live.size(); ++r)
      if (live[r] != a && live[r] != b) live[w++] = live[r];
    live.resize(w);
    live.push_back(c);
    nn[c] = -1;
    nd[c] = std::numeric_limits<float>::infinity();
    // partners: nodes that pointed at a or b rescan; every other node compares its partner with
    // c (c is last, so it only wins on a strictly smaller distance). The next pair is picked in
    // the same pass: each node's partner is final once the pass has reached it.
    int32_t na = -1;
    float best = std::numeric_limits<float>::infinity();
    for (size_t p = 0; p + 1 < live.size(); ++p) {
      const int32_t k = live[p];
      if (nn[k] == a || nn[k] == b) {
        rescan(p);
      } else {
        const float d = d2(k, c);
        if (d < nd[k]) {
          nd[k] = d;
          nn[k] = c;
        }
      }
      if (nn[k] >= 0 && nd[k] < best) {
        best = nd[k];
        na = k;
      }
    }
    a = na;
  }
  const int32_t root = total - 1;

  // left-first DFS over the leaves (bounding_volume_hierachy.cpp:85-101)
  order.reserve(n);
  std::vector<int32_t> stack;
  stack.push_back(root);
  while (!stack.empty()) {
    int32_t v = stack.back();
    stack.pop_back();
    if (left[v] < 0) {
      order.push_back((uint32_t)v);
    } else {
      stack.push_back(right[v]);
      stack.push_back(left[v]);
    }
  }
  if (tree) {
    tree->left = left;
    tree->right = right;
    tree->root = root;
  }
  return order;
}

}  // namespace swr
