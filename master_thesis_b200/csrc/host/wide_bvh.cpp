// Binned-SAH binary BVH (one primitive per leaf), collapsed top-down into 8-wide nodes and
// quantised into the 80-byte records described in swr_bvh.cuh.
#include "wide_bvh.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <deque>
#include <functional>
#include <limits>
#include <stdexcept>
#include <thread>

namespace swr {

namespace {

struct BNode {
  float lo[3], hi[3];
  uint32_t left = 0, right = 0;  // children (internal)
  uint32_t first = 0, count = 0;  // primitive range in the index array (leaf when count > 0)
};

inline float area(const float lo[3], const float hi[3]) {
  float dx = std::max(0.0f, hi[0] - lo[0]), dy = std::max(0.0f, hi[1] - lo[1]),
        dz = std::max(0.0f, hi[2] - lo[2]);
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct Builder {
  const std::vector<PrimBox>& prims;
  std::vector<float> cen;  // 3 per prim
  std::vector<uint32_t> idx;
  std::vector<BNode> nodes;
  std::atomic<uint32_t> next{1};
  uint32_t bins;
  int par_depth;

  Builder(const std::vector<PrimBox>& p, uint32_t b, int pd) : prims(p), bins(b), par_depth(pd) {
    const size_t n = p.size();
    cen.resize(3 * n);
    idx.resize(n);
    for (size_t i = 0; i < n; ++i) {
      idx[i] = (uint32_t)i;
      for (int k = 0; k < 3; ++k) cen[3 * i + k] = 0.5f * (p[i].lo[k] + p[i].hi[k]);
    }
    nodes.resize(std::max<size_t>(1, 2 * n - 1));
  }

  void build(uint32_t ni, uint32_t begin, uint32_t end, int depth) {
    BNode& nd = nodes[ni];
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < 3; ++k) {
      nd.lo[k] = INFINITY;
      nd.hi[k] = -INFINITY;
    }
    for (uint32_t i = begin; i < end; ++i) {
      const PrimBox& b = prims[idx[i]];
      for (int k = 0; k < 3; ++k) {
        nd.lo[k] = std::min(nd.lo[k], b.lo[k]);
        nd.hi[k] = std::max(nd.hi[k], b.hi[k]);
        const float c = cen[3 * idx[i] + k];
        clo[k] = std::min(clo[k], c);
        chi[k] = std::max(chi[k], c);
      }
    }
    const uint32_t count = end - begin;
    if (count == 1) {
      nd.first = begin;
      nd.count = 1;
      return;
    }
    // binned SAH over all three axes
    struct Bin {
      float lo[3], hi[3];
      uint32_t n;
    };
    std::vector<Bin> bb(bins);
    std::vector<float> lcost(bins);
    float best_cost = INFINITY;
    int best_axis = -1;
    uint32_t best_split = 0;
    for (int ax = 0; ax < 3; ++ax) {
      const float ext = chi[ax] - clo[ax];
      if (!(ext > 0.0f)) continue;
      for (auto& b : bb) {
        for (int k = 0; k < 3; ++k) {
          b.lo[k] = INFINITY;
          b.hi[k] = -INFINITY;
        }
        b.n = 0;
      }
      const float scale = (float)bins / ext;
      for (uint32_t i = begin; i < end; ++i) {
        const uint32_t p = idx[i];
        uint32_t bi = (uint32_t)((cen[3 * p + ax] - clo[ax]) * scale);
        if (bi >= bins) bi = bins - 1;
        Bin& b = bb[bi];
        for (int k = 0; k < 3; ++k) {
          b.lo[k] = std::min(b.lo[k], prims[p].lo[k]);
          b.hi[k] = std::max(b.hi[k], prims[p].hi[k]);
        }
        b.n++;
      }
      // left sweep
      float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
      uint32_t an = 0;
      for (uint32_t s = 0; s + 1 < bins; ++s) {
        for (int k = 0; k < 3; ++k) {
          alo[k] = std::min(alo[k], bb[s].lo[k]);
          ahi[k] = std::max(ahi[k], bb[s].hi[k]);
        }
        an += bb[s].n;
        lcost[s] = an ? area(alo, ahi) * (float)an : 0.0f;
      }
      float blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
      uint32_t bn = 0;
      for (uint32_t s = bins - 1; s >= 1; --s) {
        for (int k = 0; k < 3; ++k) {
          blo[k] = std::min(blo[k], bb[s].lo[k]);
          bhi[k] = std::max(bhi[k], bb[s].hi[k]);
        }
        bn += bb[s].n;
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
    uint32_t mid;
    if (best_axis >= 0) {
      const int ax = best_axis;
      const float ext = chi[ax] - clo[ax];
      const float scale = (float)bins / ext;
      auto it = std::partition(idx.begin() + begin, idx.begin() + end, [&](uint32_t p) {
        uint32_t bi = (uint32_t)((cen[3 * p + ax] - clo[ax]) * scale);
        if (bi >= bins) bi = bins - 1;
        return bi < best_split;
      });
      mid = (uint32_t)(it - idx.begin());
      if (mid == begin || mid == end) best_axis = -1;
    }
    if (best_axis < 0) {
      // degenerate centroids: split the range at its median along the widest centroid axis
      int ax = 0;
      for (int k = 1; k < 3; ++k)
        if (chi[k] - clo[k] > chi[ax] - clo[ax]) ax = k;
      mid = begin + count / 2;
      std::nth_element(idx.begin() + begin, idx.begin() + mid, idx.begin() + end,
                       [&](uint32_t a, uint32_t b) { return cen[3 * a + ax] < cen[3 * b + ax]; });
    }
    const uint32_t l = next.fetch_add(2), r = l + 1;
    nd.left = l;
    nd.right = r;
    nd.count = 0;
    if (depth < par_depth && count > 65536) {
      std::thread th([=] { build(l, begin, mid, depth + 1); });
      build(r, mid, end, depth + 1);
      th.join();
    } else {
      build(l, begin, mid, depth + 1);
      build(r, mid, end, depth + 1);
    }
  }
};

void put_f(uint32_t* w, int i, float f) { std::memcpy(&w[i], &f, 4); }

}  // namespace

WideBvh build_wide_bvh(const std::vector<PrimBox>& prims, const WideBvhOptions& opt) {
  if (prims.empty()) throw std::invalid_argument("BVH over zero primitives");
  if (opt.max_leaf < 1 || opt.max_leaf > 3) throw std::invalid_argument("max_leaf must be 1..3");
  unsigned hw = opt.threads ? opt.threads : std::max(1u, std::thread::hardware_concurrency());
  int pd = 0;
  while ((1u << pd) < hw) ++pd;
  Builder B(prims, std::max(4u, opt.sah_bins), pd + 1);
  B.build(0, 0, (uint32_t)prims.size(), 0);
  const uint32_t nb = B.next.load();
  std::vector<BNode>& bn = B.nodes;

  // subtree primitive counts (children always have larger indices than parents)
  std::vector<uint32_t> tri_count(nb, 0);
  for (int64_t i = (int64_t)nb - 1; i >= 0; --i)
    tri_count[i] = bn[i].count ? bn[i].count : tri_count[bn[i].left] + tri_count[bn[i].right];

  WideBvh out;
  out.binary_nodes = nb;
  {
    const float ra = std::max(area(bn[0].lo, bn[0].hi), 1e-30f);
    double c = 0.0;
    for (uint32_t i = 0; i < nb; ++i)
      c += (double)area(bn[i].lo, bn[i].hi) / ra * (bn[i].count ? (double)bn[i].count : 1.0);
    out.sah_cost = c;
  }

  // SAH-optimal collapse into 8-wide nodes (the dynamic program of Ylitie, Karras, Laine 2017,
  // section 4.1). For every binary node n: cost[n][i] = cheapest way to represent n's subtree by
  // at most i children of a wide node (i = 1..8); as one child it is either a leaf (at most
  // max_leaf triangles, cost area * count * kPrim) or a wide node (area * kNode + the cheapest
  // split of its subtree into at most 8 children). dist[n][j] = cheapest split of n's two binary
  // children into j children in total.
  const double kNode = 1.0, kPrim = opt.prim_cost;
  const double INF = std::numeric_limits<double>::infinity();
  std::vector<double> cost((size_t)nb * 9, INF), dist((size_t)nb * 9, INF);
  std::vector<uint8_t> dist_k((size_t)nb * 9, 0), from_fewer((size_t)nb * 9, 0), as_leaf(nb, 0);
  for (int64_t n = (int64_t)nb - 1; n >= 0; --n) {
    const BNode& b = bn[n];
    const double a = (double)area(b.lo, b.hi);
    double* C = &cost[(size_t)n * 9];
    double* D = &dist[(size_t)n * 9];
    const double leaf = tri_count[n] <= opt.max_leaf ? a * (double)tri_count[n] * kPrim : INF;
    double inner = INF;
    if (!b.count) {
      const double* CL = &cost[(size_t)b.left * 9];
      const double* CR = &cost[(size_t)b.right * 9];
      for (int j = 2; j <= 8; ++j)
        for (int k = 1; k < j; ++k) {
          const double v = CL[k] + CR[j - k];
          if (v < D[j]) {
            D[j] = v;
            dist_k[(size_t)n * 9 + j] = (uint8_t)k;
          }
        }
      inner = a * kNode + D[8];
    }
    as_leaf[n] = leaf <= inner ? 1 : 0;
    C[1] = std::min(leaf, inner);
    for (int i = 2; i <= 8; ++i) {
      if (C[i - 1] <= D[i]) {
        C[i] = C[i - 1];
        from_fewer[(size_t)n * 9 + i] = 1;
      } else {
        C[i] = D[i];
      }
    }
  }
  // children of binary node n when it is spent on at most i wide-node slots
  std::vector<uint32_t> ch;
  std::function<void(uint32_t, int)> spread = [&](uint32_t n, int i) {
    while (i > 1 && from_fewer[(size_t)n * 9 + i]) --i;
    if (i == 1) {
      ch.push_back(n);
      return;
    }
    const int k = dist_k[(size_t)n * 9 + i];
    spread(bn[n].left, k);
    spread(bn[n].right, i - k);
  };

  struct Task {
    uint32_t bnode, wide, depth;
  };
  std::deque<Task> q;
  q.push_back({0, 0, 1});
  uint32_t next_wide = 1;
  std::vector<uint32_t> gather;
  while (!q.empty()) {
    Task tk = q.front();
    q.pop_front();
    out.depth = std::max(out.depth, tk.depth);
    ch.clear();
    if (bn[tk.bnode].count || as_leaf[tk.bnode]) {
      ch.push_back(tk.bnode);  // a scene small enough to be one leaf: a root with one leaf child
    } else {
      const int k = dist_k[(size_t)tk.bnode * 9 + 8];
      spread(bn[tk.bnode].left, k);
      spread(bn[tk.bnode].right, 8 - k);
    }
    // slot assignment: child towards octant corner s goes to slot s
    float ulo[3] = {INFINITY, INFINITY, INFINITY}, uhi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t c : ch)
      for (int k = 0; k < 3; ++k) {
        ulo[k] = std::min(ulo[k], bn[c].lo[k]);
        uhi[k] = std::max(uhi[k], bn[c].hi[k]);
      }
    float pc[3];
    for (int k = 0; k < 3; ++k) pc[k] = 0.5f * (ulo[k] + uhi[k]);
    int slot_of[8];
    int child_in_slot[8];
    for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
    {
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
        slot_of[bci] = bsi;
        child_in_slot[bsi] = bci;
      }
    }
    // record
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
    const uint32_t child_base = next_wide;
    uint32_t n_inner = 0;
    const uint32_t tri_base = (uint32_t)out.prim_order.size();
    uint32_t tri_off = 0;
    for (int s = 0; s < 8; ++s) {
      const int ci = child_in_slot[s];
      if (ci < 0) continue;
      const uint32_t c = ch[ci];
      for (int k = 0; k < 3; ++k) {
        double lo = std::floor(((double)bn[c].lo[k] - (double)ulo[k]) / e[k]);
        double hi = std::ceil(((double)bn[c].hi[k] - (double)ulo[k]) / e[k]);
        qlo[k][s] = (uint8_t)std::max(0.0, std::min(255.0, lo));
        qhi[k][s] = (uint8_t)std::max(0.0, std::min(255.0, hi));
      }
      if (as_leaf[c] || (c == tk.bnode)) {
        gather.clear();
        std::vector<uint32_t> st{c};
        while (!st.empty()) {
          uint32_t v = st.back();
          st.pop_back();
          if (bn[v].count) {
            for (uint32_t i = 0; i < bn[v].count; ++i) gather.push_back(B.idx[bn[v].first + i]);
          } else {
            st.push_back(bn[v].right);
            st.push_back(bn[v].left);
          }
        }
        meta[s] = (uint8_t)((gather.size() << 5) | tri_off);
        tri_off += (uint32_t)gather.size();
        for (uint32_t p : gather) out.prim_order.push_back(p);
      } else {
        imask |= 1u << s;
        q.push_back({c, child_base + n_inner, tk.depth + 1});
        ++n_inner;
      }
    }
    (void)slot_of;
    next_wide += n_inner;
    put_f(w, 0, ulo[0]);
    put_f(w, 1, ulo[1]);
    put_f(w, 2, ulo[2]);
    w[3] = ebyte[0] | (ebyte[1] << 8) | (ebyte[2] << 16) | (imask << 24);
    w[4] = child_base;
    w[5] = tri_base;
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
    if (out.words.size() < (size_t)(tk.wide + 1) * 20) out.words.resize((size_t)(tk.wide + 1) * 20);
    std::memcpy(&out.words[(size_t)tk.wide * 20], w, sizeof(w));
  }
  out.num_nodes = next_wide;
  out.words.resize((size_t)next_wide * 20);
  return out;
}

}  // namespace swr
