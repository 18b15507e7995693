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
  std::vector<V3> ctr(total);
  std::vector<Box> box(total);
  std::vector<int32_t> left(total, -1), right(total, -1);
  std::vector<int32_t> prv(total, -1), nxt(total, -1);
  std::vector<int32_t> nn(total, -1);
  std::vector<float> nd(total, std::numeric_limits<float>::infinity());

  for (int32_t i = 0; i < n; ++i) {
    box[i] = boxes[i];
    ctr[i] = box[i].center();
    prv[i] = i - 1;
    nxt[i] = (i + 1 < n) ? i + 1 : -1;
  }
  int32_t head = 0, tail = n - 1;

  auto rescan = [&](int32_t k) {
    int32_t best = -1;
    float bd = std::numeric_limits<float>::infinity();
    for (int32_t j = nxt[k]; j != -1; j = nxt[j]) {
      float d = dist2(ctr[k], ctr[j]);
      if (d < bd) {
        bd = d;
        best = j;
      }
    }
    nn[k] = best;
    nd[k] = bd;
  };

  for (int32_t i = 0; i < n; ++i) rescan(i);

  for (int32_t c = n; c < total; ++c) {
    // pick the first node (in list order) with the smallest partner distance
    int32_t a = -1;
    float best = std::numeric_limits<float>::infinity();
    for (int32_t k = head; k != -1; k = nxt[k]) {
      if (nn[k] >= 0 && nd[k] < best) {
        best = nd[k];
        a = k;
      }
    }
    if (a < 0) {
      // every remaining distance is NaN or infinite: the reference's scan finds no pair (its
      // iterators stay unset); merge the first two live nodes so the build still terminates.
      a = head;
      nn[a] = nxt[head];
    }
    const int32_t b = nn[a];
    left[c] = a;
    right[c] = b;
    box[c] = Box::merge(box[a], box[b]);
    ctr[c] = box[c].center();
    // unlink a and b, append c
    for (int32_t r : {a, b}) {
      if (prv[r] >= 0) nxt[prv[r]] = nxt[r]; else head = nxt[r];
      if (nxt[r] >= 0) prv[nxt[r]] = prv[r]; else tail = prv[r];
      prv[r] = nxt[r] = -1;
    }
    if (tail >= 0) {
      nxt[tail] = c;
      prv[c] = tail;
    } else {
      head = c;
      prv[c] = -1;
    }
    nxt[c] = -1;
    tail = c;
    nn[c] = -1;
    nd[c] = std::numeric_limits<float>::infinity();
    for (int32_t k = head; k != c; k = nxt[k]) {
      if (nn[k] == a || nn[k] == b) {
        rescan(k);
      } else {
        float d = dist2(ctr[k], ctr[c]);
        if (d < nd[k]) {
          nd[k] = d;
          nn[k] = c;
        }
      }
    }
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
