// Closest-centre agglomerative clustering with the reference's exact tie rules
// (bounding_volume_hierachy.cpp:9-27 findClosestPair, :47-75 BVH::init).
//
// Selection rule being reproduced: among all pairs (i, j) of live nodes with i before j in the
// list (the list is ordered by creation: leaves in input order, then parents as they are made),
// take the smallest squared centre distance; on equal distances the pair that comes first in the
// i-outer / j-inner scan wins. The parent's left child is i, its right child is j, its box is the
// union, and it is appended to the end of the list. So list order is node-id order, and the pick
// is the lexicographic minimum of (distance, i, j) over pairs i < j.
//
// Two builds make that same choice at every merge:
//
// build_flat: every live node k keeps nn[k], the best node after it in the list (smallest
// distance, then earliest), with its distance nd[k]. The pick is the k with the smallest
// (nd[k], k), paired with nn[k]. After a merge of (a, b) into c, only nodes whose partner was a or
// b rescan the rest of the list; every other node compares its partner with c (c is last, so it
// only wins on a strictly smaller distance). About O(n^2) in total; used for small inputs and for
// inputs whose distances can be NaN or overflow.
//
// build_indexed: every live node k keeps its nearest live node in BOTH directions (smallest
// distance, then smallest id). The squared distance is symmetric in float (x - y rounds to
// -(y - x)), so with dmin the smallest pair distance, the smallest k whose nearest distance is
// dmin has no partner at dmin before it (that partner would be a smaller such k), and its
// nearest node is the smallest id at dmin after it: exactly the reference's (i, j). The pick is a
// tournament-tree minimum of (nd[k], k). After a merge, c queries a kd-tree for its nearest node,
// and a reverse query finds the nodes to which c is strictly closer than their current nearest
// (c has the largest id, so it never wins a tie). The nodes that pointed at a or b keep their old
// distance as a lower bound (removals only lengthen nearest distances; c is covered by the reverse
// query) and query again only when they reach the top of the tournament: a node at the top with a
// current nearest node is the reference's pick, since every other node's true key is at least its
// stored one. The kd-tree keeps, per subtree, a box around its live centres and the largest
// nearest-distance inside; both queries prune with a lower bound on the float distance (the
// geometric bound in double, less a relative 1e-5 and an absolute 1e-36 for rounding and
// underflow), so every node that the exact float comparison would accept is examined.
#include "ref_bvh.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

namespace swr {

namespace {

constexpr float kInf = std::numeric_limits<float>::infinity();

struct Centres {
  std::vector<float> x, y, z;
  explicit Centres(size_t n) : x(n), y(n), z(n) {}
  void set(int32_t i, const V3& c) {
    x[i] = c[0];
    y[i] = c[1];
    z[i] = c[2];
  }
  // squared centre distance, summed from +0 in x, y, z order (vector.h:227-241)
  float d2(int32_t a, int32_t b) const {
    const float dx = x[a] - x[b], dy = y[a] - y[b], dz = z[a] - z[b];
    float s = 0.0f;
    s += dx * dx;
    s += dy * dy;
    s += dz * dz;
    return s;
  }
};

// ---- build_flat ------------------------------------------------------------------------------

void build_flat(const std::vector<Box>& boxes, std::vector<int32_t>& left, std::vector<int32_t>& right) {
  const int32_t n = (int32_t)boxes.size();
  const int32_t total = 2 * n - 1;
  // List order is creation order (parents are appended), so the live list is the set of live
  // node ids in increasing order: kept as a flat array, with the centres as separate coordinate
  // arrays, so every pass is a linear scan.
  Centres cen(total);
  std::vector<Box> box(total);
  std::vector<int32_t> nn(total, -1);
  std::vector<float> nd(total, kInf);
  std::vector<int32_t> live(n);
  for (int32_t i = 0; i < n; ++i) {
    box[i] = boxes[i];
    cen.set(i, box[i].center());
    live[i] = i;
  }
  // best later partner of the node at live position p: smallest distance, then earliest
  auto rescan = [&](size_t p) {
    const int32_t k = live[p];
    int32_t best = -1;
    float bd = kInf;
    for (size_t q = p + 1; q < live.size(); ++q) {
      const float d = cen.d2(k, live[q]);
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
    float best = kInf;
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
    cen.set(c, box[c].center());
    // unlink a and b, append c
    size_t w = 0;
    for (size_t r = 0; r < live.size(); ++r)
      if (live[r] != a && live[r] != b) live[w++] = live[r];
    live.resize(w);
    live.push_back(c);
    nn[c] = -1;
    nd[c] = kInf;
    // partners: nodes that pointed at a or b rescan; every other node compares its partner with
    // c (c is last, so it only wins on a strictly smaller distance). The next pair is picked in
    // the same pass: each node's partner is final once the pass has reached it.
    int32_t na = -1;
    float best = kInf;
    for (size_t p = 0; p + 1 < live.size(); ++p) {
      const int32_t k = live[p];
      if (nn[k] == a || nn[k] == b) {
        rescan(p);
      } else {
        const float d = cen.d2(k, c);
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
}

// ---- build_indexed ---------------------------------------------------------------------------

// A subtree can hold a node at float distance <= limit only if its lower bound, less the rounding
// allowance, is <= limit. The bound is computed in float from the subtree box; with coordinates
// within +-1e18 nothing overflows, and its rounding (a few ulp) and the float distance's own
// rounding and underflow stay well inside the allowance.
inline float prune_bound(float lb) { return lb * 0.99999f - 1e-36f; }

class IndexedBuild {
 public:
  IndexedBuild(const std::vector<Box>& boxes, std::vector<int32_t>& left, std::vector<int32_t>& right,
               unsigned threads)
      : threads_(threads),
        n_((int32_t)boxes.size()),
        total_(2 * n_ - 1),
        cen_(total_),
        box_(total_),
        nn_(total_, -1),
        nd_(total_, kInf),
        alive_(total_, 0),
        leaf_of_(total_, -1),
        pointed_(total_),
        valid_(total_, 1),
        left_(left),
        right_(right) {
    for (int32_t i = 0; i < n_; ++i) {
      box_[i] = boxes[i];
      cen_.set(i, box_[i].center());
      alive_[i] = 1;
    }
    tour_size_ = 1;
    while (tour_size_ < total_) tour_size_ <<= 1;
    tour_.assign(2 * (size_t)tour_size_, -1);
  }

  void run() {
    std::vector<int32_t> ids(n_);
    for (int32_t i = 0; i < n_; ++i) ids[i] = i;
    rebuild(ids);
    // every leaf's nearest node: independent queries over the same tree, split across threads
    const unsigned nth = std::max(1u, std::min(threads_, (unsigned)(n_ / 1024)));
    if (nth > 1) {
      std::vector<std::thread> pool;
      for (unsigned t = 0; t < nth; ++t)
        pool.emplace_back([this, t, nth] {
          std::vector<std::pair<int32_t, float>> stack;
          for (int32_t i = (int32_t)((int64_t)n_ * t / nth); i < (int32_t)((int64_t)n_ * (t + 1) / nth); ++i)
            nearest_into(i, stack, nn_[i], nd_[i]);
        });
      for (std::thread& th : pool) th.join();
      for (int32_t i = 0; i < n_; ++i) pointed_[nn_[i]].push_back(i);
    } else {
      for (int32_t i = 0; i < n_; ++i) nearest(i);
    }
    for (size_t v = nodes_.size(); v-- > 0;) {  // children come after their parent
      Node& node = nodes_[v];
      node.maxnd = node.child < 0 ? leaf_max(node)
                                  : std::max(nodes_[node.child].maxnd, nodes_[node.child + 1].maxnd);
    }
    for (int32_t i = 0; i < n_; ++i) tour_set(i);
    int32_t live = n_;
    std::vector<int32_t> closer;
    for (int32_t c = n_; c < total_; ++c) {
      // the smallest (nd, id); a node whose nearest node has gone holds a lower bound there and
      // is looked up again when it comes to the top
      int32_t a = tour_[1];
      while (!valid_[a]) {
        nearest(a);
        refresh_leaf(leaf_of_[a]);
        tour_set(a);
        a = tour_[1];
      }
      const int32_t b = nn_[a];
      left_[c] = a;
      right_[c] = b;
      box_[c] = Box::merge(box_[a], box_[b]);
      cen_.set(c, box_[c].center());
      // a and b leave, c enters
      remove(a);
      remove(b);
      alive_[c] = 1;
      live -= 1;
      if (live == 1) break;
      if (live <= built_ / 2) {
        std::vector<int32_t> ids_live;
        ids_live.reserve(live);
        for (int32_t i = 0; i <= c; ++i)
          if (alive_[i]) ids_live.push_back(i);
        rebuild(ids_live);
      } else {
        insert(c);
      }
      // nodes whose nearest node was a or b keep that distance as a lower bound: removing nodes
      // only lengthens a nearest distance, and c (the one new node) is handled below
      for (int32_t dead : {a, b}) {
        for (int32_t k : pointed_[dead])
          if (alive_[k] && nn_[k] == dead) valid_[k] = 0;
        std::vector<int32_t>().swap(pointed_[dead]);
      }
      nearest(c);
      refresh_leaf(leaf_of_[c]);
      // nodes to which c is strictly closer than their nearest distance (or its lower bound):
      // c is then their nearest node
      closer.clear();
      reverse(c, closer);
      for (int32_t k : closer) refresh_leaf(leaf_of_[k]);
      for (int32_t k : closer) tour_set(k);
      tour_set(c);
    }
  }

 private:
  // kd-tree node; children are allocated in pairs (child, child + 1)
  struct Node {
    float lo[3], hi[3];  // box around the live centres inside (grows on insert)
    float maxnd;         // largest nd of a live centre inside, -inf if none
    int32_t child;       // -1 for leaves
    int32_t parent;
    int32_t axis;        // inner nodes: split axis and value
    float split;
    int32_t slab;        // leaves: first of kLeafCap slots in slots_
    int32_t count;       // leaves: slots in use
  };
  struct Slot {  // a live centre in a leaf
    float x, y, z;
    int32_t id;
  };
  static constexpr int kLeafSize = 8;  // leaves of a fresh tree
  static constexpr int kLeafCap = 32;  // a leaf that inserts fill up is split

  const unsigned threads_;
  const int32_t n_, total_;
  Centres cen_;
  std::vector<Box> box_;
  std::vector<int32_t> nn_;
  std::vector<float> nd_;
  std::vector<uint8_t> alive_;
  std::vector<int32_t> leaf_of_;
  std::vector<std::vector<int32_t>> pointed_;  // k with nn[k] == i at some time (checked on use)
  std::vector<uint8_t> valid_;  // 0: nn[k] has gone and nd[k] is a lower bound of the nearest distance
  std::vector<int32_t>& left_;
  std::vector<int32_t>& right_;
  std::vector<Node> nodes_;
  std::vector<Slot> slots_;
  std::vector<std::pair<int32_t, float>> stack_;
  int32_t built_ = 0;
  int32_t tour_size_ = 1;
  std::vector<int32_t> tour_;  // tournament tree over node ids: winner = smallest (nd, id)

  float coord(int32_t i, int axis) const { return axis == 0 ? cen_.x[i] : axis == 1 ? cen_.y[i] : cen_.z[i]; }

  // squared distance from q to a subtree box, in float
  static float lower_bound(const float q[3], const Node& node) {
    float s = 0.0f;
    for (int k = 0; k < 3; ++k) {
      const float d = std::max(0.0f, std::max(node.lo[k] - q[k], q[k] - node.hi[k]));
      s += d * d;
    }
    return s;
  }

  // the float distance of centres (Centres::d2), from a query point and a slot
  static float dist2(const float q[3], const Slot& s) {
    const float dx = q[0] - s.x, dy = q[1] - s.y, dz = q[2] - s.z;
    float r = 0.0f;
    r += dx * dx;
    r += dy * dy;
    r += dz * dz;
    return r;
  }

  void centre(int32_t i, float q[3]) const {
    q[0] = cen_.x[i];
    q[1] = cen_.y[i];
    q[2] = cen_.z[i];
  }

  float leaf_max(const Node& node) const {
    float m = -kInf;
    const Slot* s = &slots_[node.slab];
    for (int32_t j = 0; j < node.count; ++j) m = std::max(m, nd_[s[j].id]);
    return m;
  }

  // makes node v the subtree over ids[begin, end): tight box, children or slots, maxima
  void fill(int32_t v, std::vector<int32_t>& ids, size_t begin, size_t end) {
    Node* node = &nodes_[v];
    node->child = -1;
    for (int k = 0; k < 3; ++k) {
      node->lo[k] = kInf;
      node->hi[k] = -kInf;
    }
    for (size_t i = begin; i < end; ++i)
      for (int k = 0; k < 3; ++k) {
        const float c = coord(ids[i], k);
        node->lo[k] = std::min(node->lo[k], c);
        node->hi[k] = std::max(node->hi[k], c);
      }
    if (end - begin <= (size_t)kLeafSize) {
      node->slab = (int32_t)slots_.size();
      node->count = (int32_t)(end - begin);
      slots_.resize(slots_.size() + kLeafCap);
      for (size_t i = begin; i < end; ++i) {
        const int32_t p = ids[i];
        slots_[node->slab + (i - begin)] = Slot{cen_.x[p], cen_.y[p], cen_.z[p], p};
        leaf_of_[p] = v;
      }
      node->maxnd = leaf_max(*node);
      return;
    }
    int axis = 0;
    for (int k = 1; k < 3; ++k)
      if (node->hi[k] - node->lo[k] > node->hi[axis] - node->lo[axis]) axis = k;
    const size_t mid = begin + (end - begin) / 2;
    std::nth_element(ids.begin() + begin, ids.begin() + mid, ids.begin() + end, [&](int32_t p, int32_t q) {
      const float a = coord(p, axis), b = coord(q, axis);
      return a < b || (a == b && p < q);
    });
    node->axis = axis;
    node->split = coord(ids[mid], axis);
    const int32_t l = (int32_t)nodes_.size();
    nodes_.resize(nodes_.size() + 2);  // moves nodes_
    nodes_[l].parent = nodes_[l + 1].parent = v;
    nodes_[v].child = l;
    fill(l, ids, begin, mid);
    fill(l + 1, ids, mid, end);
    nodes_[v].maxnd = std::max(nodes_[l].maxnd, nodes_[l + 1].maxnd);
  }

  void rebuild(std::vector<int32_t>& ids) {
    nodes_.clear();
    slots_.clear();
    nodes_.reserve(ids.size() / 2 + 8);
    slots_.reserve((ids.size() / 4 + 2) * kLeafCap);
    built_ = (int32_t)ids.size();
    nodes_.emplace_back();
    nodes_[0].parent = -1;
    fill(0, ids, 0, ids.size());
  }

  void refresh_leaf(int32_t leaf) {
    nodes_[leaf].maxnd = leaf_max(nodes_[leaf]);
    refresh_up(leaf);
  }

  void refresh_up(int32_t v) {
    while (nodes_[v].parent >= 0) {
      v = nodes_[v].parent;
      const int32_t ch = nodes_[v].child;
      const float u = std::max(nodes_[ch].maxnd, nodes_[ch + 1].maxnd);
      if (u == nodes_[v].maxnd) break;
      nodes_[v].maxnd = u;
    }
  }

  // c joins the leaf whose split planes it falls in; its nd is set (and the maxima refreshed)
  // by the caller
  void insert(int32_t c) {
    float q[3];
    centre(c, q);
    int32_t v = 0;
    for (;;) {
      Node& node = nodes_[v];
      for (int k = 0; k < 3; ++k) {
        node.lo[k] = std::min(node.lo[k], q[k]);
        node.hi[k] = std::max(node.hi[k], q[k]);
      }
      if (node.child < 0) break;
      v = node.child + (q[node.axis] < node.split ? 0 : 1);
    }
    Node& leaf = nodes_[v];
    if (leaf.count < kLeafCap) {
      slots_[leaf.slab + leaf.count++] = Slot{q[0], q[1], q[2], c};
      leaf_of_[c] = v;
      return;
    }
    // full: the leaf's centres and c become a subtree (its slab is left unused)
    std::vector<int32_t> ids;
    ids.reserve(kLeafCap + 1);
    for (int32_t j = 0; j < leaf.count; ++j) ids.push_back(slots_[leaf.slab + j].id);
    ids.push_back(c);
    fill(v, ids, 0, ids.size());
    refresh_up(v);
  }

  void remove(int32_t i) {
    alive_[i] = 0;
    tour_set(i);
    Node& leaf = nodes_[leaf_of_[i]];
    Slot* s = &slots_[leaf.slab];
    for (int32_t j = 0; j < leaf.count; ++j)
      if (s[j].id == i) {
        s[j] = s[--leaf.count];
        break;
      }
    refresh_leaf(leaf_of_[i]);
  }

  void assign(int32_t k, int32_t j, float d) {
    nn_[k] = j;
    nd_[k] = d;
    valid_[k] = 1;
    pointed_[j].push_back(k);
  }

  // nearest live node of k (smallest float distance, then smallest id)
  void nearest(int32_t k) {
    int32_t j;
    float d;
    nearest_into(k, stack_, j, d);
    assign(k, j, d);
  }

  // the nearest live node of k and its distance; reads the tree only
  void nearest_into(int32_t k, std::vector<std::pair<int32_t, float>>& stack, int32_t& out_id,
                    float& out_d) const {
    float q[3];
    centre(k, q);
    // (distance, id) as one key: distances are >= +0, so their bit patterns order like the
    // values, and the smallest key is the smallest distance, then the smallest id
    const uint64_t none = ((uint64_t)bits(kInf) << 32) | 0xFFFFFFFFu;
    uint64_t best = none;
    stack.clear();
    stack.emplace_back(0, 0.0f);
    while (!stack.empty()) {
      const auto [v, lb] = stack.back();
      stack.pop_back();
      if (prune_bound(lb) > key_dist(best)) continue;
      const Node& node = nodes_[v];
      if (node.child < 0) {
        const Slot* s = &slots_[node.slab];
        for (int32_t j = 0; j < node.count; ++j) {
          const uint64_t key = ((uint64_t)bits(dist2(q, s[j])) << 32) | (uint32_t)s[j].id;
          const uint64_t cand = s[j].id == k ? none : key;
          best = cand < best ? cand : best;
        }
        continue;
      }
      // the nearer child is visited first
      const float l0 = lower_bound(q, nodes_[node.child]);
      const float l1 = lower_bound(q, nodes_[node.child + 1]);
      const int32_t near = l0 <= l1 ? node.child : node.child + 1;
      stack.emplace_back(2 * node.child + 1 - near, l0 <= l1 ? l1 : l0);
      stack.emplace_back(near, l0 <= l1 ? l0 : l1);
    }
    out_id = (int32_t)(uint32_t)best;
    out_d = key_dist(best);
  }

  static uint32_t bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
  }
  static float key_dist(uint64_t key) {
    const uint32_t u = (uint32_t)(key >> 32);
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  }

  // live nodes k != c with d2(k, c) < nd[k]: c becomes their nearest node
  void reverse(int32_t c, std::vector<int32_t>& out) {
    float q[3];
    centre(c, q);
    stack_.clear();
    stack_.emplace_back(0, 0.0f);
    while (!stack_.empty()) {
      const int32_t v = stack_.back().first;
      stack_.pop_back();
      const Node& node = nodes_[v];
      if (prune_bound(lower_bound(q, node)) >= node.maxnd) continue;
      if (node.child < 0) {
        const Slot* s = &slots_[node.slab];
        for (int32_t j = 0; j < node.count; ++j) {
          const int32_t p = s[j].id;
          if (p == c) continue;
          const float d = dist2(q, s[j]);
          if (d < nd_[p]) {
            assign(p, c, d);
            out.push_back(p);
          }
        }
        continue;
      }
      stack_.emplace_back(node.child, 0.0f);
      stack_.emplace_back(node.child + 1, 0.0f);
    }
  }

  bool wins(int32_t i, int32_t j) const {  // (nd, id) order; -1 (a dead node's slot) last
    if (j < 0) return true;
    if (i < 0) return false;
    return nd_[i] < nd_[j] || (nd_[i] == nd_[j] && i < j);
  }

  void tour_set(int32_t i) {
    size_t v = (size_t)tour_size_ + i;
    tour_[v] = alive_[i] ? i : -1;
    for (v >>= 1; v >= 1; v >>= 1) {
      const int32_t l = tour_[2 * v], r = tour_[2 * v + 1];
      tour_[v] = wins(l, r) ? l : r;
    }
  }
};

// The indexed build needs every pair distance finite: box coordinates within +-1e18 keep
// squared centre distances below 1.2e37.
bool indexable(const std::vector<Box>& boxes) {
  for (const Box& b : boxes)
    for (int k = 0; k < 3; ++k)
      if (!(std::fabs(b.lo[k]) <= 1e18f) || !(std::fabs(b.hi[k]) <= 1e18f)) return false;
  return true;
}

}  // namespace

std::vector<uint32_t> ref_bvh_leaf_order(const std::vector<Box>& boxes, RefTree* tree, RefBuild how,
                                         unsigned threads) {
  const int32_t n = (int32_t)boxes.size();
  std::vector<uint32_t> order;
  if (n == 0) return order;
  const int32_t total = 2 * n - 1;
  std::vector<int32_t> left(total, -1), right(total, -1);
  const bool indexed = how == RefBuild::kIndexed ||
                       (how == RefBuild::kAuto && n >= kRefIndexedMin);
  if (n > 1) {
    if (indexed && indexable(boxes)) {
      IndexedBuild(boxes, left, right, threads ? threads : std::max(1u, std::thread::hardware_concurrency())).run();
    } else {
      build_flat(boxes, left, right);
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
    tree->left = std::move(left);
    tree->right = std::move(right);
    tree->root = root;
  }
  return order;
}

}  // namespace swr
