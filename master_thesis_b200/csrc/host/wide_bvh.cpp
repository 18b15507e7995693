// Binned-SAH binary BVH (one primitive per leaf), collapsed into 8-wide nodes by the SAH-optimal
// dynamic program and quantised into the 80-byte records described in swr_bvh.cuh.
//
// Work layout: each primitive's centroid and box travel with its index through the partitions,
// so every pass over a node's range streams; all three axes are binned in one pass; the passes
// over large ranges are split across threads, and subtrees below the top levels are built by
// threads of their own; the collapse's dynamic program runs in the build's post-order, each node
// as soon as its children are done. The wide nodes are then laid out one level at a time: the
// nodes of a level are collapsed and encoded in parallel, and their child and triangle bases are
// prefix sums in breadth-first order. The result does not depend on the thread count.
#include "wide_bvh.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <thread>

namespace swr {

namespace {

struct Ref {  // a primitive as it moves through the partitions
  float lo[3], hi[3];
  uint32_t id;
  float c(int k) const { return 0.5f * (lo[k] + hi[k]); }  // centroid
};

struct BNode {
  float lo[3], hi[3];
  uint32_t left = 0, right = 0;  // children (internal)
  uint32_t first = 0, count = 0;  // position in the primitive array (leaf when count > 0)
};

inline float area(const float lo[3], const float hi[3]) {
  float dx = std::max(0.0f, hi[0] - lo[0]), dy = std::max(0.0f, hi[1] - lo[1]),
        dz = std::max(0.0f, hi[2] - lo[2]);
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// f(t, begin, end) over nt contiguous parts of [begin, end), part 0 on the calling thread
template <class F>
void split_range(uint32_t begin, uint32_t end, unsigned nt, F f) {
  if (nt <= 1) {
    f(0u, begin, end);
    return;
  }
  std::vector<std::thread> pool;
  const uint64_t n = end - begin;
  for (unsigned t = 1; t < nt; ++t)
    pool.emplace_back(f, t, begin + (uint32_t)(n * t / nt), begin + (uint32_t)(n * (t + 1) / nt));
  f(0u, begin, begin + (uint32_t)(n / nt));
  for (std::thread& th : pool) th.join();
}

struct Bounds {
  float lo[3], hi[3], clo[3], chi[3];
  void reset() {
    for (int k = 0; k < 3; ++k) {
      lo[k] = clo[k] = INFINITY;
      hi[k] = chi[k] = -INFINITY;
    }
  }
  void merge(const Bounds& o) {
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], o.lo[k]);
      hi[k] = std::max(hi[k], o.hi[k]);
      clo[k] = std::min(clo[k], o.clo[k]);
      chi[k] = std::max(chi[k], o.chi[k]);
    }
  }
};

struct Bin {
  float lo[3], hi[3];
  uint32_t n;
};

// The collapse's result for one binary node, passed to its parent: cost[i] = cheapest way to
// represent the subtree by at most i children of a wide node (i = 1..8); sah = the binary
// subtree's unnormalised SAH sum (area x primitives at leaves, area at inner nodes).
struct Sub {
  double cost[9];
  double sah;
};

constexpr uint32_t kParallelPass = 1u << 18;  // ranges this large split their passes
constexpr uint32_t kSparse = 32;               // ranges this small are binned sparsely

struct Builder {
  std::vector<Ref> refs;
  std::vector<BNode> nodes;
  std::vector<uint32_t> tri_count;
  // the dynamic program's choices per binary node n: dist_k[9n + j] = how many of the j children
  // of the best split come from the left subtree; fewer[n] bit i: cost[i] = cost[i - 1]
  std::vector<uint8_t> dist_k;
  std::vector<uint16_t> fewer;
  std::vector<uint8_t> as_leaf;
  std::atomic<uint32_t> next{1};
  uint32_t bins;
  int par_depth;
  unsigned hw;
  uint32_t max_leaf;
  double prim_cost;
  int width;  // children per wide node (2..8)

  Builder(const std::vector<PrimBox>& p, uint32_t b, int pd, unsigned threads, uint32_t ml, double pc, int w)
      : bins(b), par_depth(pd), hw(threads), max_leaf(ml), prim_cost(pc), width(w) {
    const size_t n = p.size();
    refs.resize(n);
    const size_t nb = std::max<size_t>(1, 2 * n - 1);
    nodes.resize(nb);
    tri_count.resize(nb);
    dist_k.resize(nb * 9);
    fewer.resize(nb);
    as_leaf.resize(nb);
    split_range(0, (uint32_t)n, std::min<unsigned>(hw, (unsigned)(n >> 16) + 1), [&](unsigned, uint32_t b0, uint32_t b1) {
      for (uint32_t i = b0; i < b1; ++i) {
        Ref& r = refs[i];
        r.id = i;
        for (int k = 0; k < 3; ++k) {
          r.lo[k] = p[i].lo[k];
          r.hi[k] = p[i].hi[k];
        }
      }
    });
  }

  unsigned pass_threads(uint32_t count, int depth) const {
    if (count < kParallelPass) return 1;
    const unsigned share = std::max(1u, hw >> std::min(depth, 16));
    return std::max(1u, std::min(share, count >> 16));
  }

  Bounds bounds(uint32_t begin, uint32_t end, unsigned nt) const {
    std::vector<Bounds> part(nt);
    split_range(begin, end, nt, [&](unsigned t, uint32_t b0, uint32_t b1) {
      Bounds bd;
      bd.reset();
      for (uint32_t i = b0; i < b1; ++i) {
        const Ref& r = refs[i];
        for (int k = 0; k < 3; ++k) {
          bd.lo[k] = std::min(bd.lo[k], r.lo[k]);
          bd.hi[k] = std::max(bd.hi[k], r.hi[k]);
          bd.clo[k] = std::min(bd.clo[k], r.c(k));
          bd.chi[k] = std::max(bd.chi[k], r.c(k));
        }
      }
      part[t] = bd;
    });
    Bounds all = part[0];
    for (unsigned t = 1; t < nt; ++t) all.merge(part[t]);
    return all;
  }

  // out[ax * B + b]: bins over the axes with a non-empty centroid extent, in one pass
  void bin(uint32_t begin, uint32_t end, unsigned nt, const bool use[3], const float clo[3], const float scale[3],
           std::vector<Bin>& out) const {
    const uint32_t B = bins;
    out.resize(3 * (size_t)B);
    std::vector<std::vector<Bin>> part(nt > 1 ? nt - 1 : 0, std::vector<Bin>(3 * (size_t)B));
    split_range(begin, end, nt, [&](unsigned t, uint32_t b0, uint32_t b1) {
      std::vector<Bin>& bb = t == 0 ? out : part[t - 1];
      for (Bin& b : bb) {
        for (int k = 0; k < 3; ++k) {
          b.lo[k] = INFINITY;
          b.hi[k] = -INFINITY;
        }
        b.n = 0;
      }
      for (uint32_t i = b0; i < b1; ++i) {
        const Ref& r = refs[i];
        for (int ax = 0; ax < 3; ++ax) {
          if (!use[ax]) continue;
          uint32_t bi = (uint32_t)((r.c(ax) - clo[ax]) * scale[ax]);
          if (bi >= B) bi = B - 1;
          Bin& b = bb[ax * B + bi];
          for (int k = 0; k < 3; ++k) {
            b.lo[k] = std::min(b.lo[k], r.lo[k]);
            b.hi[k] = std::max(b.hi[k], r.hi[k]);
          }
          b.n++;
        }
      }
    });
    for (const std::vector<Bin>& pt : part)
      for (size_t j = 0; j < out.size(); ++j) {
        for (int k = 0; k < 3; ++k) {
          out[j].lo[k] = std::min(out[j].lo[k], pt[j].lo[k]);
          out[j].hi[k] = std::max(out[j].hi[k], pt[j].hi[k]);
        }
        out[j].n += pt[j].n;
      }
  }

  // The same choice as the binned sweep below for a small range, from its occupied bins only:
  // an empty bin changes neither side's union box nor its count, so every split position inside
  // a run of empty bins has the cost of the run's last position, which the descending sweep meets
  // first and keeps (later ones are not strictly cheaper); positions with an empty side are
  // skipped by both. Costs are computed from the same unions in the same float operations.
  void sparse_sah(uint32_t begin, uint32_t end, const bool use[3], const float clo[3], const float scale[3],
                  float& best_cost, int& best_axis, uint32_t& best_split) const {
    const uint32_t B = bins, count = end - begin;
    struct Occ {
      uint32_t bin;
      float lo[3], hi[3];
      uint32_t n;
    };
    Occ occ[kSparse];
    float lcost[kSparse];
    for (int ax = 0; ax < 3; ++ax) {
      if (!use[ax]) continue;
      // occupied bins in ascending order (insertion into a short sorted list)
      uint32_t m = 0;
      for (uint32_t i = begin; i < end; ++i) {
        const Ref& r = refs[i];
        uint32_t bi = (uint32_t)((r.c(ax) - clo[ax]) * scale[ax]);
        if (bi >= B) bi = B - 1;
        uint32_t j = 0;
        while (j < m && occ[j].bin < bi) ++j;
        if (j == m || occ[j].bin != bi) {
          for (uint32_t q = m; q > j; --q) occ[q] = occ[q - 1];
          ++m;
          occ[j].bin = bi;
          occ[j].n = 0;
          for (int k = 0; k < 3; ++k) {
            occ[j].lo[k] = INFINITY;
            occ[j].hi[k] = -INFINITY;
          }
        }
        for (int k = 0; k < 3; ++k) {
          occ[j].lo[k] = std::min(occ[j].lo[k], r.lo[k]);
          occ[j].hi[k] = std::max(occ[j].hi[k], r.hi[k]);
        }
        occ[j].n++;
      }
      float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
      uint32_t an = 0;
      for (uint32_t j = 0; j < m; ++j) {
        for (int k = 0; k < 3; ++k) {
          alo[k] = std::min(alo[k], occ[j].lo[k]);
          ahi[k] = std::max(ahi[k], occ[j].hi[k]);
        }
        an += occ[j].n;
        lcost[j] = area(alo, ahi) * (float)an;
      }
      float blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
      uint32_t bn = 0;
      for (uint32_t j = m; j-- > 1;) {  // split before occupied bin j: bins < occ[j].bin go left
        for (int k = 0; k < 3; ++k) {
          blo[k] = std::min(blo[k], occ[j].lo[k]);
          bhi[k] = std::max(bhi[k], occ[j].hi[k]);
        }
        bn += occ[j].n;
        if (count - bn == 0 || bn == 0) continue;
        const float c = lcost[j - 1] + area(blo, bhi) * (float)bn;
        if (c < best_cost) {
          best_cost = c;
          best_axis = ax;
          best_split = occ[j].bin;
        }
      }
    }
  }

  // The collapse's dynamic program (Ylitie, Karras, Laine 2017, section 4.1) at node ni, from its
  // children's costs: as one child of a wide node, the subtree is either a leaf (at most
  // max_leaf triangles, cost area x count x prim_cost) or a wide node (area + the cheapest split
  // of its subtree into at most `width` (8 unless built narrower) children); dist[j] = cheapest
  // split of the two binary children into j children in total.
  void collapse(uint32_t ni, const Sub* L, const Sub* R, Sub& out) {
    const double INF = std::numeric_limits<double>::infinity();
    const BNode& b = nodes[ni];
    const double a = (double)area(b.lo, b.hi);
    double D[9];
    for (double& d : D) d = INF;
    const double leaf = tri_count[ni] <= max_leaf ? a * (double)tri_count[ni] * prim_cost : INF;
    double inner = INF;
    if (!b.count) {
      for (int j = 2; j <= width; ++j)
        for (int k = 1; k < j; ++k) {
          const double v = L->cost[k] + R->cost[j - k];
          if (v < D[j]) {
            D[j] = v;
            dist_k[(size_t)ni * 9 + j] = (uint8_t)k;
          }
        }
      inner = a * 1.0 + D[width];
    }
    as_leaf[ni] = leaf <= inner ? 1 : 0;
    double* C = out.cost;
    C[0] = INF;
    C[1] = std::min(leaf, inner);
    uint16_t fw = 0;
    for (int i = 2; i <= width; ++i) {
      if (C[i - 1] <= D[i]) {
        C[i] = C[i - 1];
        fw |= (uint16_t)(1u << i);
      } else {
        C[i] = D[i];
      }
    }
    fewer[ni] = fw;
    out.sah = (double)area(b.lo, b.hi) * (b.count ? (double)b.count : 1.0) + (b.count ? 0.0 : L->sah + R->sah);
  }

  void build(uint32_t ni, uint32_t begin, uint32_t end, int depth, Sub& out) {
    const uint32_t count = end - begin;
    const unsigned nt = pass_threads(count, depth);
    const Bounds bd = bounds(begin, end, nt);
    BNode& nd = nodes[ni];
    for (int k = 0; k < 3; ++k) {
      nd.lo[k] = bd.lo[k];
      nd.hi[k] = bd.hi[k];
    }
    if (count == 1) {
      nd.first = begin;
      nd.count = 1;
      tri_count[ni] = 1;
      collapse(ni, nullptr, nullptr, out);
      return;
    }
    // binned SAH over all three axes
    const uint32_t B = bins;
    bool use[3];
    float scale[3];
    for (int ax = 0; ax < 3; ++ax) {
      const float ext = bd.chi[ax] - bd.clo[ax];
      use[ax] = ext > 0.0f;
      scale[ax] = use[ax] ? (float)B / ext : 0.0f;
    }
    float best_cost = INFINITY;
    int best_axis = -1;
    uint32_t best_split = 0;
    if (count <= kSparse) {
      sparse_sah(begin, end, use, bd.clo, scale, best_cost, best_axis, best_split);
    } else if (use[0] || use[1] || use[2]) {
      thread_local std::vector<Bin> bb;
      thread_local std::vector<float> lcost;
      bin(begin, end, nt, use, bd.clo, scale, bb);
      lcost.resize(B);
      for (int ax = 0; ax < 3; ++ax) {
        if (!use[ax]) continue;
        const Bin* ab = &bb[ax * B];
        // left sweep
        float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t an = 0;
        for (uint32_t s = 0; s + 1 < B; ++s) {
          for (int k = 0; k < 3; ++k) {
            alo[k] = std::min(alo[k], ab[s].lo[k]);
            ahi[k] = std::max(ahi[k], ab[s].hi[k]);
          }
          an += ab[s].n;
          lcost[s] = an ? area(alo, ahi) * (float)an : 0.0f;
        }
        float blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t bn = 0;
        for (uint32_t s = B - 1; s >= 1; --s) {
          for (int k = 0; k < 3; ++k) {
            blo[k] = std::min(blo[k], ab[s].lo[k]);
            bhi[k] = std::max(bhi[k], ab[s].hi[k]);
          }
          bn += ab[s].n;
          const uint32_t ln = count - bn;
          if (ln == 0 || bn == 0) continue;
          const float c = lcost[s - 1] + area(blo, bhi) * (float)bn;
          if (c < best_cost) {
            best_cost = c;
            best_axis = ax;
            best_split = s;
          }
        }
      }
    }
    uint32_t mid = begin;
    if (best_axis >= 0) {
      const int ax = best_axis;
      const float lo = bd.clo[ax], sc = scale[ax];
      auto it = std::partition(refs.begin() + begin, refs.begin() + end, [&](const Ref& r) {
        uint32_t bi = (uint32_t)((r.c(ax) - lo) * sc);
        if (bi >= B) bi = B - 1;
        return bi < best_split;
      });
      mid = (uint32_t)(it - refs.begin());
      if (mid == begin || mid == end) best_axis = -1;
    }
    if (best_axis < 0) {
      // degenerate centroids: split the range at its median along the widest centroid axis
      int ax = 0;
      for (int k = 1; k < 3; ++k)
        if (bd.chi[k] - bd.clo[k] > bd.chi[ax] - bd.clo[ax]) ax = k;
      mid = begin + count / 2;
      std::nth_element(refs.begin() + begin, refs.begin() + mid, refs.begin() + end,
                       [&](const Ref& a, const Ref& b) { return a.c(ax) < b.c(ax); });
    }
    const uint32_t l = next.fetch_add(2), r = l + 1;
    nd.left = l;
    nd.right = r;
    nd.count = 0;
    Sub sl, sr;
    if (depth < par_depth && count > 65536) {
      std::thread th([&, l, begin, mid, depth] { build(l, begin, mid, depth + 1, sl); });
      build(r, mid, end, depth + 1, sr);
      th.join();
    } else {
      build(l, begin, mid, depth + 1, sl);
      build(r, mid, end, depth + 1, sr);
    }
    tri_count[ni] = tri_count[l] + tri_count[r];
    collapse(ni, &sl, &sr, out);
  }
};

void put_f(uint32_t* w, int i, float f) { std::memcpy(&w[i], &f, 4); }

// One wide node being laid out: its binary node, its children in slot order, and what the level
// pass derives from them.
struct WideTask {
  uint32_t bnode;
  int32_t child[8];   // binary node per slot, -1 when empty
  uint8_t leaf_mask;  // slots holding leaves
  uint32_t n_inner, n_tri;
  uint32_t child_base, tri_base;
};

}  // namespace

WideBvh build_wide_bvh(const std::vector<PrimBox>& prims, const WideBvhOptions& opt) {
  if (prims.empty()) throw std::invalid_argument("BVH over zero primitives");
  if (opt.max_leaf < 1 || opt.max_leaf > 3) throw std::invalid_argument("max_leaf must be 1..3");
  if (opt.width < 2 || opt.width > 8) throw std::invalid_argument("width must be 2..8");
  unsigned hw = opt.threads ? opt.threads : std::max(1u, std::thread::hardware_concurrency());
  int pd = 0;
  while ((1u << pd) < hw) ++pd;
  Builder B(prims, std::max(4u, opt.sah_bins), pd + 1, hw, opt.max_leaf, opt.prim_cost, (int)opt.width);
  Sub root;
  B.build(0, 0, (uint32_t)prims.size(), 0, root);
  const uint32_t nb = B.next.load();
  const std::vector<BNode>& bn = B.nodes;

  WideBvh out;
  out.binary_nodes = nb;
  out.sah_cost = root.sah / (double)std::max(area(bn[0].lo, bn[0].hi), 1e-30f);
  out.prim_order.resize(prims.size());

  // children of binary node n when it is spent on at most i wide-node slots, left to right
  auto spread = [&](uint32_t n0, int i0, std::vector<uint32_t>& ch) {
    std::pair<uint32_t, int> st[64];
    int sp = 0;
    st[sp++] = {n0, i0};
    while (sp) {
      auto [n, i] = st[--sp];
      while (i > 1 && (B.fewer[n] >> i) & 1u) --i;
      if (i == 1) {
        ch.push_back(n);
        continue;
      }
      const int k = B.dist_k[(size_t)n * 9 + i];
      st[sp++] = {bn[n].right, i - k};
      st[sp++] = {bn[n].left, k};
    }
  };

  // children and slots of one wide node (child towards octant corner s goes to slot s)
  auto layout = [&](WideTask& tk) {
    std::vector<uint32_t> ch;
    ch.reserve(8);
    if (bn[tk.bnode].count || B.as_leaf[tk.bnode]) {
      ch.push_back(tk.bnode);  // a scene small enough to be one leaf: a root with one leaf child
    } else {
      const int w = (int)opt.width;
      const int k = B.dist_k[(size_t)tk.bnode * 9 + w];
      spread(bn[tk.bnode].left, k, ch);
      spread(bn[tk.bnode].right, w - k, ch);
    }
    float ulo[3] = {INFINITY, INFINITY, INFINITY}, uhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t c : ch)
      for (int k = 0; k < 3; ++k) {
        ulo[k] = std::min(ulo[k], bn[c].lo[k]);
        uhi[k] = std::max(uhi[k], bn[c].hi[k]);
      }
    float pc[3];
    for (int k = 0; k < 3; ++k) pc[k] = 0.5f * (ulo[k] + uhi[k]);
    for (int s = 0; s < 8; ++s) tk.child[s] = -1;
    bool used_c[8] = {false}, used_s[8] = {false};
    for (size_t round = 0; round < ch.size(); ++round) {
      float bc = INFINITY;
      int bci = -1, bsi = -1;
      for (size_t ci = 0; ci < ch.size(); ++ci) {
        if (used_c[ci]) continue;
        const BNode& c = bn[ch[ci]];
        float cc[3];
        for (int k = 0; k < 3; ++k) cc[k] = 0.5f * (c.lo[k] + c.hi[k]) - pc[k];
        for (int s = 0; s < 8; ++s) {
          if (used_s[s]) continue;
          const float cost = -(cc[0] * ((s & 1) ? 1.0f : -1.0f) + cc[1] * ((s & 2) ? 1.0f : -1.0f) +
                               cc[2] * ((s & 4) ? 1.0f : -1.0f));
          if (cost < bc) {
            bc = cost;
            bci = (int)ci;
            bsi = s;
          }
        }
      }
      used_c[bci] = true;
      used_s[bsi] = true;
      tk.child[bsi] = (int32_t)ch[bci];
    }
    tk.leaf_mask = 0;
    tk.n_inner = tk.n_tri = 0;
    for (int s = 0; s < 8; ++s) {
      const int32_t c = tk.child[s];
      if (c < 0) continue;
      if (B.as_leaf[c] || (uint32_t)c == tk.bnode) {
        tk.leaf_mask |= (uint8_t)(1u << s);
        tk.n_tri += B.tri_count[c];
      } else {
        ++tk.n_inner;
      }
    }
  };

  // the 80-byte record of one wide node (index wi) and its leaves' primitives
  auto encode = [&](const WideTask& tk, uint32_t wi) {
    float ulo[3] = {INFINITY, INFINITY, INFINITY}, uhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int s = 0; s < 8; ++s) {
      const int32_t c = tk.child[s];
      if (c < 0) continue;
      for (int k = 0; k < 3; ++k) {
        ulo[k] = std::min(ulo[k], bn[c].lo[k]);
        uhi[k] = std::max(uhi[k], bn[c].hi[k]);
      }
    }
    uint32_t w[20];
    std::memset(w, 0, sizeof(w));
    uint8_t qlo[3][8], qhi[3][8];
    std::memset(qlo, 255, sizeof(qlo));
    std::memset(qhi, 0, sizeof(qhi));
    uint32_t ebyte[3];
    double e[3];
    for (int k = 0; k < 3; ++k) {
      const double ext = (double)uhi[k] - (double)ulo[k];
      int ex = -126;
      if (ext > 0.0) {
        int x;
        std::frexp(ext / 255.0, &x);  // ext/255 = m * 2^x, m in [0.5, 1)
        ex = x;
        if (std::ldexp(1.0, ex - 1) >= ext / 255.0) ex = ex - 1;
      }
      ex = std::max(-126, std::min(127, ex));
      ebyte[k] = (uint32_t)(ex + 127);
      e[k] = std::ldexp(1.0, ex);
    }
    uint32_t imask = 0;
    uint8_t meta[8] = {0};
    uint32_t tri_off = 0;
    uint32_t st[64];
    for (int s = 0; s < 8; ++s) {
      const int32_t c = tk.child[s];
      if (c < 0) continue;
      for (int k = 0; k < 3; ++k) {
        double lo = std::floor(((double)bn[c].lo[k] - (double)ulo[k]) / e[k]);
        double hi = std::ceil(((double)bn[c].hi[k] - (double)ulo[k]) / e[k]);
        qlo[k][s] = (uint8_t)std::max(0.0, std::min(255.0, lo));
        qhi[k][s] = (uint8_t)std::max(0.0, std::min(255.0, hi));
      }
      if (tk.leaf_mask & (1u << s)) {
        // the leaf's primitives, left-first
        const uint32_t cnt = B.tri_count[c];
        uint32_t* dst = &out.prim_order[tk.tri_base + tri_off];
        int sp = 0;
        st[sp++] = (uint32_t)c;
        while (sp) {
          const uint32_t v = st[--sp];
          if (bn[v].count) {
            for (uint32_t i = 0; i < bn[v].count; ++i) *dst++ = B.refs[bn[v].first + i].id;
          } else {
            st[sp++] = bn[v].right;
            st[sp++] = bn[v].left;
          }
        }
        meta[s] = (uint8_t)((cnt << 5) | tri_off);
        tri_off += cnt;
      } else {
        imask |= 1u << s;
      }
    }
    put_f(w, 0, ulo[0]);
    put_f(w, 1, ulo[1]);
    put_f(w, 2, ulo[2]);
    w[3] = ebyte[0] | (ebyte[1] << 8) | (ebyte[2] << 16) | (imask << 24);
    w[4] = tk.child_base;
    w[5] = tk.tri_base;
    w[6] = meta[0] | (meta[1] << 8) | (meta[2] << 16) | ((uint32_t)meta[3] << 24);
    w[7] = meta[4] | (meta[5] << 8) | (meta[6] << 16) | ((uint32_t)meta[7] << 24);
    auto pack = [](const uint8_t* b) {
      return (uint32_t)b[0] | ((uint32_t)b[1] << 8) | ((uint32_t)b[2] << 16) | ((uint32_t)b[3] << 24);
    };
    w[8] = pack(qlo[0]);
    w[9] = pack(qlo[0] + 4);
    w[10] = pack(qlo[1]);
    w[11] = pack(qlo[1] + 4);
    w[12] = pack(qlo[2]);
    w[13] = pack(qlo[2] + 4);
    w[14] = pack(qhi[0]);
    w[15] = pack(qhi[0] + 4);
    w[16] = pack(qhi[1]);
    w[17] = pack(qhi[1] + 4);
    w[18] = pack(qhi[2]);
    w[19] = pack(qhi[2] + 4);
    std::memcpy(&out.words[(size_t)wi * 20], w, sizeof(w));
  };

  // level by level: the root is wide node 0; a level's inner children become the next level, in
  // node then slot order, numbered from the running wide-node count (breadth-first order)
  std::vector<WideTask> level(1);
  level[0].bnode = 0;
  uint32_t level_first = 0, next_wide = 1, tri_total = 0;
  while (!level.empty()) {
    ++out.depth;
    const uint32_t nl = (uint32_t)level.size();
    const unsigned nt = std::min<unsigned>(hw, nl / 256 + 1);
    split_range(0, nl, nt, [&](unsigned, uint32_t b0, uint32_t b1) {
      for (uint32_t i = b0; i < b1; ++i) layout(level[i]);
    });
    for (WideTask& tk : level) {
      tk.child_base = next_wide;
      next_wide += tk.n_inner;
      tk.tri_base = tri_total;
      tri_total += tk.n_tri;
    }
    out.words.resize((size_t)next_wide * 20);
    split_range(0, nl, nt, [&](unsigned, uint32_t b0, uint32_t b1) {
      for (uint32_t i = b0; i < b1; ++i) encode(level[i], level_first + i);
    });
    std::vector<WideTask> nxt;
    nxt.reserve(next_wide - level_first - nl);
    for (const WideTask& tk : level)
      for (int s = 0; s < 8; ++s)
        if (tk.child[s] >= 0 && !(tk.leaf_mask & (1u << s))) {
          nxt.emplace_back();
          nxt.back().bnode = (uint32_t)tk.child[s];
        }
    level_first += nl;
    level.swap(nxt);
  }
  out.num_nodes = next_wide;
  return out;
}

}  // namespace swr
