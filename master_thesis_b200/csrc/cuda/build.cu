// Device construction of the traversal BVH (swr_build_opts.builder = SWR_BUILD_DEVICE).
//
// The same 80-byte wide-node records as the host builder (swr_bvh.cuh), built on the GPU:
//   1. Morton codes of the primitive-box centres (63 bits) and a radix sort (CUB).
//   2. Binary tree by locally-ordered clustering (PLOC: Meister and Bittner, "Parallel Locally-
//      Ordered Clustering for Bounding Volume Hierarchy Construction", TVCG 2018): in every round
//      each cluster finds, among the clusters within `radius` positions of it in Morton order, the
//      one whose union box has the smallest surface area; mutual nearest neighbours merge; the
//      survivors are compacted. Rounds repeat until one cluster is left.
//   3. The SAH-optimal collapse into 8-wide nodes (the dynamic program of Ylitie, Karras, Laine
//      2017, section 4.1, as the host builder runs it), bottom-up: a thread per leaf walks towards
//      the root and the second thread to reach a node evaluates it.
//   4. Wide nodes emitted level by level, one thread per node: its children by the DP's
//      decisions, octant slot order, 8-bit quantisation, triangle slots of its leaves.
// The tree differs from the host builder's, but any tree of conservative boxes gives the same
// closest hits; only the speed of the traversal depends on it.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "build_device.h"
#include "swr_internal.cuh"

namespace swr {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr int kBlock = 256;

struct Box6 {
  float lo[3], hi[3];
};

__device__ __forceinline__ Box6 load_box(const float* b, uint32_t i) {
  Box6 r;
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = b[6 * (size_t)i + k];
    r.hi[k] = b[6 * (size_t)i + 3 + k];
  }
  return r;
}

__device__ __forceinline__ void store_box(float* b, uint32_t i, const Box6& r) {
  for (int k = 0; k < 3; ++k) {
    b[6 * (size_t)i + k] = r.lo[k];
    b[6 * (size_t)i + 3 + k] = r.hi[k];
  }
}

__device__ __forceinline__ Box6 join(const Box6& a, const Box6& b) {
  Box6 r;
  for (int k = 0; k < 3; ++k) {
    r.lo[k] = fminf(a.lo[k], b.lo[k]);
    r.hi[k] = fmaxf(a.hi[k], b.hi[k]);
  }
  return r;
}

__device__ __forceinline__ float area(const Box6& b) {
  const float dx = fmaxf(0.0f, b.hi[0] - b.lo[0]), dy = fmaxf(0.0f, b.hi[1] - b.lo[1]),
              dz = fmaxf(0.0f, b.hi[2] - b.lo[2]);
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// ---- 1. centres, bounds, Morton codes -------------------------------------------------------

// floats as order-preserving ints (an involution), so that min/max can be integer atomics
__host__ __device__ __forceinline__ int ord_of(int bits) { return bits >= 0 ? bits : bits ^ 0x7FFFFFFF; }

__global__ void k_centre_bounds(const float* __restrict__ prim, uint32_t n, int* __restrict__ bounds) {
  // bounds: lo.xyz hi.xyz of the box centres (ordered ints)
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Box6 b = load_box(prim, i);
    for (int k = 0; k < 3; ++k) {
      const float c = 0.5f * (b.lo[k] + b.hi[k]);
      lo[k] = fminf(lo[k], c);
      hi[k] = fmaxf(hi[k], c);
    }
  }
  for (int k = 0; k < 3; ++k)
    for (int off = 16; off > 0; off >>= 1) {
      lo[k] = fminf(lo[k], __shfl_down_sync(0xffffffffu, lo[k], off));
      hi[k] = fmaxf(hi[k], __shfl_down_sync(0xffffffffu, hi[k], off));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) {
      atomicMin(&bounds[k], ord_of(__float_as_int(lo[k])));
      atomicMax(&bounds[3 + k], ord_of(__float_as_int(hi[k])));
    }
}

__device__ __forceinline__ float from_ord(int v) { return __int_as_float(ord_of(v)); }

// the low 21 bits of v spread to every third bit
__device__ __forceinline__ uint64_t spread21(uint64_t v) {
  v &= 0x1FFFFFull;
  v = (v | (v << 32)) & 0x1F00000000FFFFull;
  v = (v | (v << 16)) & 0x1F0000FF0000FFull;
  v = (v | (v << 8)) & 0x100F00F00F00F00Full;
  v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

__global__ void k_morton(const float* __restrict__ prim, uint32_t n, const int* __restrict__ bounds,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ ids) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float lo[3], scale[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = from_ord(bounds[k]);
    const float ext = from_ord(bounds[3 + k]) - lo[k];
    scale[k] = ext > 0.0f ? 2097151.0f / ext : 0.0f;
  }
  const Box6 b = load_box(prim, i);
  uint64_t q[3];
  for (int k = 0; k < 3; ++k) {
    const float c = (0.5f * (b.lo[k] + b.hi[k]) - lo[k]) * scale[k];
    q[k] = (uint64_t)fminf(fmaxf(c, 0.0f), 2097151.0f);
  }
  keys[i] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
  ids[i] = i;
}

// ---- 2. PLOC ---------------------------------------------------------------------------------
// Binary nodes: leaves are 0..n-1 (leaf i = i-th primitive in Morton order), inner nodes n..2n-2.

__global__ void k_leaves(const float* __restrict__ prim, const uint32_t* __restrict__ sorted, uint32_t n,
                         float* __restrict__ node_box, uint32_t* __restrict__ cl_id, float* __restrict__ cl_box) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Box6 b = load_box(prim, sorted[i]);
  store_box(node_box, i, b);
  store_box(cl_box, i, b);
  cl_id[i] = i;
}

// nearest neighbour of every cluster within `radius` positions (ties to the lower position, so
// the relation has no cycles longer than two)
__global__ void k_nearest(const float* __restrict__ cl_box, uint32_t m, int radius, uint32_t* __restrict__ nn) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const Box6 bi = load_box(cl_box, i);
  float best = INFINITY;
  uint32_t bj = kNone;
  const int lo = max(0, (int)i - radius), hi = min((int)m - 1, (int)i + radius);
  for (int j = lo; j <= hi; ++j) {
    if (j == (int)i) continue;
    const float a = area(join(bi, load_box(cl_box, (uint32_t)j)));
    if (a < best) {  // j ascending: ties keep the lower position
      best = a;
      bj = (uint32_t)j;
    }
  }
  nn[i] = bj;
}

// mutual pairs merge into a new node at the lower position; the higher position dies
__global__ void k_merge(const uint32_t* __restrict__ nn, uint32_t m, const uint32_t* __restrict__ cl_id,
                        const float* __restrict__ cl_box, uint32_t* __restrict__ keep, uint32_t* __restrict__ nid,
                        float* __restrict__ nbox, uint32_t* __restrict__ next_node, float* __restrict__ node_box,
                        uint32_t* __restrict__ left, uint32_t* __restrict__ right, uint32_t* __restrict__ parent) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const uint32_t j = nn[i];
  const bool mutual = j != kNone && nn[j] == i;
  if (mutual && i > j) {
    keep[i] = 0u;
    return;
  }
  keep[i] = 1u;
  if (!mutual) {
    nid[i] = cl_id[i];
    store_box(nbox, i, load_box(cl_box, i));
    return;
  }
  const uint32_t a = cl_id[i], b = cl_id[j];
  const uint32_t v = atomicAdd(next_node, 1u);
  const Box6 u = join(load_box(cl_box, i), load_box(cl_box, j));
  store_box(node_box, v, u);
  left[v] = a;
  right[v] = b;
  parent[a] = v;
  parent[b] = v;
  nid[i] = v;
  store_box(nbox, i, u);
}

__global__ void k_compact(const uint32_t* __restrict__ keep, const uint32_t* __restrict__ pos, uint32_t m,
                          const uint32_t* __restrict__ nid, const float* __restrict__ nbox,
                          uint32_t* __restrict__ cl_id, float* __restrict__ cl_box, uint32_t* __restrict__ count) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  if (i == m - 1) *count = pos[i] + keep[i];
  if (!keep[i]) return;
  const uint32_t p = pos[i];
  cl_id[p] = nid[i];
  store_box(cl_box, p, load_box(nbox, i));
}

// ---- 3. SAH-optimal collapse, bottom-up -----------------------------------------------------
// Per binary node: C[1..8] (cost of the subtree as at most i wide-node children), the split of
// the two children for every j (dist_k, 3 bits each), the "fewer children are no dearer" bits,
// whether it is spent as a leaf, and its primitive count.

struct Dp {
  float c[8];
  uint32_t dist_k;  // 3 bits per j = 2..8 at bit 3*(j-2)
  uint32_t flags;   // bit i-1 (i = 2..8): C[i] = C[i-1]; bit 8: as a leaf
  uint32_t count;
  uint32_t pad;
};

__device__ void eval_node(uint32_t v, uint32_t n, const float* __restrict__ node_box, const uint32_t* left,
                          const uint32_t* right, Dp* dp, uint32_t max_leaf, float kprim, int width) {
  const Box6 b = load_box(node_box, v);
  const float a = area(b);
  Dp r;
  r.dist_k = 0;
  r.flags = 0;
  r.pad = 0;
  float D[9];
  for (int j = 0; j < 9; ++j) D[j] = INFINITY;
  float inner = INFINITY;
  if (v < n) {
    r.count = 1;
  } else {
    // the children's tables were published by other threads before their atomic on this node;
    // read them from L2 (.cg), where those stores are visible
    const Dp* L = &dp[left[v]];
    const Dp* R = &dp[right[v]];
    float CL[8], CR[8];
    for (int k = 0; k < 8; ++k) {
      CL[k] = __ldcg(&L->c[k]);
      CR[k] = __ldcg(&R->c[k]);
    }
    r.count = __ldcg(&L->count) + __ldcg(&R->count);
    for (int j = 2; j <= width; ++j)
      for (int k = 1; k < j; ++k) {
        const float c = CL[k - 1] + CR[j - k - 1];
        if (c < D[j]) {
          D[j] = c;
          r.dist_k = (r.dist_k & ~(7u << (3 * (j - 2)))) | ((uint32_t)k << (3 * (j - 2)));
        }
      }
    inner = a + D[width];
  }
  const float leaf = r.count <= max_leaf ? a * (float)r.count * kprim : INFINITY;
  if (leaf <= inner) r.flags |= 1u << 8;
  r.c[0] = fminf(leaf, inner);
  for (int i = 2; i <= 8; ++i) {  // above width D is infinite: the width entry repeats as 'fewer'
    if (r.c[i - 2] <= D[i]) {
      r.c[i - 1] = r.c[i - 2];
      r.flags |= 1u << (i - 1);
    } else {
      r.c[i - 1] = D[i];
    }
  }
  dp[v] = r;
}

__global__ void k_collapse_up(uint32_t n, const float* __restrict__ node_box, const uint32_t* __restrict__ left,
                              const uint32_t* __restrict__ right, const uint32_t* __restrict__ parent,
                              uint32_t* __restrict__ visits, Dp* __restrict__ dp, uint32_t max_leaf, float kprim,
                              int width) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t v = i;
  eval_node(v, n, node_box, left, right, dp, max_leaf, kprim, width);
  // each inner node is reached by exactly two threads (one per child), so the walk is bounded by
  // the tree height and never waits
  for (;;) {
    const uint32_t p = parent[v];
    if (p == kNone) return;
    __threadfence();                               // publish dp[v] before announcing it
    if (atomicAdd(&visits[p], 1u) == 0u) return;  // the sibling subtree is not done yet
    __threadfence();
    eval_node(p, n, node_box, left, right, dp, max_leaf, kprim, width);
    v = p;
  }
}

// ---- 4. wide nodes, level by level ----------------------------------------------------------

struct Task {
  uint32_t bnode, wide, depth, pad;
};

struct EmitArgs {
  uint32_t n;
  const float* node_box;
  const uint32_t* left;
  const uint32_t* right;
  const Dp* dp;
  const uint32_t* sorted;  // Morton position -> primitive
  uint32_t* words;         // 20 per wide node
  uint32_t* prim_order;    // triangle slot -> primitive
  uint32_t* counters;      // [0] wide nodes, [1] triangle slots, [2] next-level tasks, [3] max depth
  int width;               // children per wide node (2..8)
};

__device__ __forceinline__ int dist_k_of(const Dp& d, int j) { return (int)((d.dist_k >> (3 * (j - 2))) & 7u); }
__device__ __forceinline__ bool fewer(const Dp& d, int i) { return (d.flags >> (i - 1)) & 1u; }
__device__ __forceinline__ bool as_leaf(const EmitArgs& A, uint32_t v) {
  return v < A.n || ((A.dp[v].flags >> 8) & 1u);
}

__global__ void k_emit(EmitArgs A, const Task* __restrict__ tasks, uint32_t ntasks, Task* __restrict__ next) {
  const uint32_t ti = blockIdx.x * blockDim.x + threadIdx.x;
  if (ti >= ntasks) return;
  const Task tk = tasks[ti];
  atomicMax(&A.counters[3], tk.depth);
  // children of the wide node: the binary nodes its 8 slots are spent on
  uint32_t ch[8];
  int nch = 0;
  if (as_leaf(A, tk.bnode)) {
    ch[nch++] = tk.bnode;  // a scene small enough to be one leaf: a root with one leaf child
  } else {
    uint32_t sn[16];
    int si[16];
    int sp = 0;
    const int k = dist_k_of(A.dp[tk.bnode], A.width);
    sn[sp] = A.right[tk.bnode];
    si[sp++] = A.width - k;
    sn[sp] = A.left[tk.bnode];
    si[sp++] = k;
    while (sp > 0) {
      --sp;
      const uint32_t v = sn[sp];
      int i = si[sp];
      const Dp d = A.dp[v];
      while (i > 1 && fewer(d, i)) --i;
      if (i == 1) {
        ch[nch++] = v;
        continue;
      }
      const int kk = dist_k_of(d, i);
      sn[sp] = A.right[v];
      si[sp++] = i - kk;
      sn[sp] = A.left[v];
      si[sp++] = kk;
    }
  }
  // union box and slot assignment: the child towards octant corner s takes slot s
  Box6 cb[8];
  float ulo[3] = {INFINITY, INFINITY, INFINITY}, uhi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int c = 0; c < nch; ++c) {
    cb[c] = load_box(A.node_box, ch[c]);
    for (int k = 0; k < 3; ++k) {
      ulo[k] = fminf(ulo[k], cb[c].lo[k]);
      uhi[k] = fmaxf(uhi[k], cb[c].hi[k]);
    }
  }
  float pc[3];
  for (int k = 0; k < 3; ++k) pc[k] = 0.5f * (ulo[k] + uhi[k]);
  int child_in_slot[8];
  for (int s = 0; s < 8; ++s) child_in_slot[s] = -1;
  {
    uint32_t used_c = 0, used_s = 0;
    for (int round = 0; round < nch; ++round) {
      float bc = INFINITY;
      int bci = -1, bsi = -1;
      for (int ci = 0; ci < nch; ++ci) {
        if (used_c & (1u << ci)) continue;
        float cc[3];
        for (int k = 0; k < 3; ++k) cc[k] = 0.5f * (cb[ci].lo[k] + cb[ci].hi[k]) - pc[k];
        for (int s = 0; s < 8; ++s) {
          if (used_s & (1u << s)) continue;
          const float cost = -(cc[0] * ((s & 1) ? 1.0f : -1.0f) + cc[1] * ((s & 2) ? 1.0f : -1.0f) +
                               cc[2] * ((s & 4) ? 1.0f : -1.0f));
          if (bci < 0 || cost < bc) {
            bc = cost;
            bci = ci;
            bsi = s;
          }
        }
      }
      used_c |= 1u << bci;
      used_s |= 1u << bsi;
      child_in_slot[bsi] = bci;
    }
  }
  // quantisation grid: per axis the smallest power of two e with 255 e >= extent
  uint32_t ebyte[3];
  double e[3];
  for (int k = 0; k < 3; ++k) {
    const double ext = (double)uhi[k] - (double)ulo[k];
    int ex = -126;
    if (ext > 0.0) {
      int x;
      frexp(ext / 255.0, &x);
      ex = x;
      if (ldexp(1.0, ex - 1) >= ext / 255.0) ex = ex - 1;
    }
    ex = max(-126, min(127, ex));
    ebyte[k] = (uint32_t)(ex + 127);
    e[k] = ldexp(1.0, ex);
  }
  // triangles of the leaf children and the count of inner children
  uint32_t leaf_tris[8];
  uint32_t n_inner = 0, n_tris = 0;
  for (int s = 0; s < 8; ++s) {
    const int ci = child_in_slot[s];
    leaf_tris[s] = 0;
    if (ci < 0) continue;
    const uint32_t v = ch[ci];
    if (as_leaf(A, v)) {
      leaf_tris[s] = v < A.n ? 1u : A.dp[v].count;
      n_tris += leaf_tris[s];
    } else {
      ++n_inner;
    }
  }
  const uint32_t child_base = n_inner ? atomicAdd(&A.counters[0], n_inner) : 0u;
  const uint32_t tri_base = n_tris ? atomicAdd(&A.counters[1], n_tris) : 0u;
  const uint32_t task_base = n_inner ? atomicAdd(&A.counters[2], n_inner) : 0u;
  uint8_t qlo[3][8], qhi[3][8], meta[8];
  for (int s = 0; s < 8; ++s) {
    meta[s] = 0;
    for (int k = 0; k < 3; ++k) {
      qlo[k][s] = 255;
      qhi[k][s] = 0;
    }
  }
  uint32_t imask = 0, inner_i = 0, tri_off = 0;
  for (int s = 0; s < 8; ++s) {
    const int ci = child_in_slot[s];
    if (ci < 0) continue;
    for (int k = 0; k < 3; ++k) {
      const double lo = floor(((double)cb[ci].lo[k] - (double)ulo[k]) / e[k]);
      const double hi = ceil(((double)cb[ci].hi[k] - (double)ulo[k]) / e[k]);
      qlo[k][s] = (uint8_t)fmax(0.0, fmin(255.0, lo));
      qhi[k][s] = (uint8_t)fmax(0.0, fmin(255.0, hi));
    }
    const uint32_t v = ch[ci];
    if (leaf_tris[s]) {
      // the leaf's primitives in depth-first order (at most max_leaf <= 3 of them)
      uint32_t st[8];
      int sp = 0;
      st[sp++] = v;
      uint32_t w = tri_base + tri_off;
      while (sp > 0) {
        const uint32_t u = st[--sp];
        if (u < A.n) {
          A.prim_order[w++] = A.sorted[u];
        } else {
          st[sp++] = A.right[u];
          st[sp++] = A.left[u];
        }
      }
      meta[s] = (uint8_t)((leaf_tris[s] << 5) | tri_off);
      tri_off += leaf_tris[s];
    } else {
      imask |= 1u << s;
      Task t;
      t.bnode = v;
      t.wide = child_base + inner_i;
      t.depth = tk.depth + 1;
      t.pad = 0;
      next[task_base + inner_i] = t;
      ++inner_i;
    }
  }
  uint32_t* w = A.words + (size_t)tk.wide * 20;
  w[0] = __float_as_uint(ulo[0]);
  w[1] = __float_as_uint(ulo[1]);
  w[2] = __float_as_uint(ulo[2]);
  w[3] = ebyte[0] | (ebyte[1] << 8) | (ebyte[2] << 16) | (imask << 24);
  w[4] = child_base;
  w[5] = tri_base;
  w[6] = meta[0] | (meta[1] << 8) | (meta[2] << 16) | ((uint32_t)meta[3] << 24);
  w[7] = meta[4] | (meta[5] << 8) | (meta[6] << 16) | ((uint32_t)meta[7] << 24);
  for (int k = 0; k < 3; ++k) {
    w[8 + 2 * k] = qlo[k][0] | (qlo[k][1] << 8) | (qlo[k][2] << 16) | ((uint32_t)qlo[k][3] << 24);
    w[9 + 2 * k] = qlo[k][4] | (qlo[k][5] << 8) | (qlo[k][6] << 16) | ((uint32_t)qlo[k][7] << 24);
    w[14 + 2 * k] = qhi[k][0] | (qhi[k][1] << 8) | (qhi[k][2] << 16) | ((uint32_t)qhi[k][3] << 24);
    w[15 + 2 * k] = qhi[k][4] | (qhi[k][5] << 8) | (qhi[k][6] << 16) | ((uint32_t)qhi[k][7] << 24);
  }
}

// ---- helpers --------------------------------------------------------------------------------

// stream-ordered scratch allocations, released on the stream when the build returns
struct Scratch {
  std::vector<void*> ptrs;
  cudaStream_t stream = nullptr;
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, stream);
  }
  template <class T>
  int get(T** p, size_t count) {
    void* q = nullptr;
    cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(count * sizeof(T), 16), stream);
    if (e != cudaSuccess) return set_error(SWR_ERR_ALLOC, "CUDA: BVH build scratch allocation failed");
    ptrs.push_back(q);
    *p = (T*)q;
    return SWR_OK;
  }
};

unsigned blocks(uint64_t n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

int build_wide_bvh_device(const float* d_prim_boxes, uint32_t n, const DeviceBuildOptions& opt, DeviceBvh& out,
                          cudaStream_t stream) {
  if (n == 0) return set_error(SWR_ERR_INVALID, "swr: BVH over zero primitives");
  if (n > (1u << 30)) return set_error(SWR_ERR_UNSUPPORTED, "swr: device BVH build handles at most 2^30 triangles");
  if (opt.max_leaf < 1 || opt.max_leaf > 3) return set_error(SWR_ERR_INVALID, "swr: max_leaf must be 1..3");
  if (opt.radius < 1 || opt.radius > 256) return set_error(SWR_ERR_INVALID, "swr: search radius must be 1..256");
  Scratch S;
  S.stream = stream;
  int rc;
  const size_t nn = 2 * (size_t)n - 1;
  uint64_t *keys, *keys2;
  uint32_t *ids, *sorted, *cl_id, *cl_id2, *near, *keep, *pos, *nid, *left, *right, *parent, *visits, *counters;
  int* bounds;
  float *node_box, *cl_box, *cl_box2, *nbox;
  Dp* dp;
  Task *tasks, *tasks2;
  if ((rc = S.get(&keys, n)) || (rc = S.get(&keys2, n)) || (rc = S.get(&ids, n)) || (rc = S.get(&sorted, n)) ||
      (rc = S.get(&cl_id, n)) || (rc = S.get(&cl_id2, n)) || (rc = S.get(&near, n)) || (rc = S.get(&keep, n)) ||
      (rc = S.get(&pos, n)) || (rc = S.get(&nid, n)) || (rc = S.get(&left, nn)) || (rc = S.get(&right, nn)) ||
      (rc = S.get(&parent, nn)) || (rc = S.get(&visits, nn)) || (rc = S.get(&counters, 8)) ||
      (rc = S.get(&bounds, 6)) || (rc = S.get(&node_box, nn * 6)) || (rc = S.get(&cl_box, (size_t)n * 6)) ||
      (rc = S.get(&cl_box2, (size_t)n * 6)) || (rc = S.get(&nbox, (size_t)n * 6)) || (rc = S.get(&dp, nn)) ||
      (rc = S.get(&tasks, n)) || (rc = S.get(&tasks2, n)))
    return rc;
  uint32_t* host = nullptr;  // pinned: [0..3] counters read back, [4] cluster count, [5] root
  SWR_CUDA(cudaMallocHost(&host, 8 * sizeof(uint32_t)));
  struct HostFree {
    uint32_t* p;
    ~HostFree() { cudaFreeHost(p); }
  } hf{host};

  // 1. Morton order
  {
    const int pinf = ord_of(0x7F800000), ninf = ord_of((int)0xFF800000u);
    const int init[6] = {pinf, pinf, pinf, ninf, ninf, ninf};
    SWR_CUDA(cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    SWR_CUDA(cudaStreamSynchronize(stream));  // init lives on this stack frame
    k_centre_bounds<<<std::min(blocks(n), 1184u), kBlock, 0, stream>>>(d_prim_boxes, n, bounds);
    k_morton<<<blocks(n), kBlock, 0, stream>>>(d_prim_boxes, n, bounds, keys, ids);
    size_t tmp_bytes = 0;
    SWR_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, ids, sorted, (int)n, 0, 63, stream));
    char* tmp;
    if ((rc = S.get(&tmp, tmp_bytes))) return rc;
    SWR_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, ids, sorted, (int)n, 0, 63, stream));
    SWR_CUDA(cudaGetLastError());
  }
  // 2. PLOC rounds
  SWR_CUDA(cudaMemsetAsync(parent, 0xFF, nn * sizeof(uint32_t), stream));
  SWR_CUDA(cudaMemsetAsync(visits, 0, nn * sizeof(uint32_t), stream));
  SWR_CUDA(cudaMemsetAsync(counters, 0, 8 * sizeof(uint32_t), stream));
  k_leaves<<<blocks(n), kBlock, 0, stream>>>(d_prim_boxes, sorted, n, node_box, cl_id, cl_box);
  host[6] = n;  // inner nodes are numbered from n
  SWR_CUDA(cudaMemcpyAsync(counters + 4, host + 6, sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
  size_t scan_bytes = 0;
  SWR_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, keep, pos, (int)n, stream));
  char* scan_tmp;
  if ((rc = S.get(&scan_tmp, scan_bytes))) return rc;
  uint32_t m = n, rounds = 0;
  while (m > 1) {
    if (++rounds > n + 64) return set_error(SWR_ERR_TIMEOUT, "swr: BVH clustering did not converge");
    k_nearest<<<blocks(m), kBlock, 0, stream>>>(cl_box, m, (int)opt.radius, near);
    k_merge<<<blocks(m), kBlock, 0, stream>>>(near, m, cl_id, cl_box, keep, nid, nbox, counters + 4, node_box,
                                              left, right, parent);
    SWR_CUDA(cub::DeviceScan::ExclusiveSum(scan_tmp, scan_bytes, keep, pos, (int)m, stream));
    k_compact<<<blocks(m), kBlock, 0, stream>>>(keep, pos, m, nid, nbox, cl_id2, cl_box2, counters + 5);
    SWR_CUDA(cudaGetLastError());
    SWR_CUDA(cudaMemcpyAsync(host + 4, counters + 5, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SWR_CUDA(cudaStreamSynchronize(stream));
    std::swap(cl_id, cl_id2);
    std::swap(cl_box, cl_box2);
    if (host[4] >= m) return set_error(SWR_ERR_TIMEOUT, "swr: BVH clustering made no progress");
    m = host[4];
  }
  SWR_CUDA(cudaMemcpyAsync(host + 5, cl_id, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  SWR_CUDA(cudaStreamSynchronize(stream));
  const uint32_t root = host[5];
  // 3. collapse costs bottom-up
  k_collapse_up<<<blocks(n), kBlock, 0, stream>>>(n, node_box, left, right, parent, visits, dp, opt.max_leaf,
                                                 (float)opt.prim_cost, (int)opt.width);
  SWR_CUDA(cudaGetLastError());
  // 4. wide nodes level by level. A wide node other than a single-leaf root has at least two
  // children and every leaf child holds a primitive, so there are at most n of them.
  void* words = nullptr;
  void* order = nullptr;
  SWR_CUDA(cudaMalloc(&words, ((size_t)n + 1) * 80));
  if (cudaMalloc(&order, (size_t)n * sizeof(uint32_t)) != cudaSuccess) {
    cudaFree(words);
    return set_error(SWR_ERR_ALLOC, "CUDA: BVH triangle order allocation failed");
  }
  out.d_nodes = words;
  out.d_prim_order = (uint32_t*)order;
  {
    Task* t0 = (Task*)(host);  // reuse the pinned words for the root task, then the counters
    t0->bnode = root;
    t0->wide = 0u;
    t0->depth = 1u;
    t0->pad = 0u;
    SWR_CUDA(cudaMemcpyAsync(tasks, t0, sizeof(Task), cudaMemcpyHostToDevice, stream));
    SWR_CUDA(cudaStreamSynchronize(stream));
    host[0] = 1u;
    host[1] = host[2] = host[3] = 0u;
    SWR_CUDA(cudaMemcpyAsync(counters, host, 4 * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
    SWR_CUDA(cudaStreamSynchronize(stream));
  }
  EmitArgs A;
  A.n = n;
  A.node_box = node_box;
  A.left = left;
  A.right = right;
  A.dp = dp;
  A.sorted = sorted;
  A.words = (uint32_t*)words;
  A.prim_order = out.d_prim_order;
  A.counters = counters;
  A.width = (int)opt.width;
  uint32_t ntasks = 1, levels = 0;
  while (ntasks > 0) {
    if (++levels > 64) return set_error(SWR_ERR_UNSUPPORTED, "swr: BVH deeper than the traversal stack");
    k_emit<<<blocks(ntasks), kBlock, 0, stream>>>(A, tasks, ntasks, tasks2);
    SWR_CUDA(cudaGetLastError());
    SWR_CUDA(cudaMemcpyAsync(host, counters, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SWR_CUDA(cudaStreamSynchronize(stream));
    ntasks = host[2];
    SWR_CUDA(cudaMemsetAsync(counters + 2, 0, sizeof(uint32_t), stream));
    std::swap(tasks, tasks2);
  }
  if (host[1] != n) return set_error(SWR_ERR_CUDA, "swr: device BVH lost primitives");
  out.num_nodes = host[0];
  out.depth = host[3];
  out.binary_nodes = (uint32_t)nn;
  out.rounds = rounds;
  return SWR_OK;
}

}  // namespace swr
