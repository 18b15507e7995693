// Moving objects on the GPU (C ABI: swr_scene_create_from_host, swr_scene_set_transforms).
//
// The reference places every object once, in GraphicsObject::init (graphics_object.cpp:12-52):
// world vertex = (p, 1) * M and world normal = (n, 0) * M with M = I*S*R*T in row-vector form,
// then the object's mesh BVH is copied and refit to the world triangles (BVH::rebuild,
// bounding_volume_hierachy.cpp:77-79,130-139). Here a scene made from a host scene keeps the
// object-space meshes on the device, and a new set of placements is applied by kernels:
//
//   k_inst_vertices  one thread per world vertex: its object's matrix applied to the mesh vertex
//                    and normal, each product and sum rounded as the host's float code does it.
//   k_inst_objbox    one warp per object: the reference's object box (first vertex padded by
//                    1e-4, then std::min/std::max), lanes over contiguous vertex ranges combined
//                    in order so that equal coordinates keep the first one, as sequentially.
//   k_inst_derive    one thread per triangle: edges, dot products, reference triangle box and
//                    corner normals, written to the triangle's BVH slot; the scene extent is
//                    reduced for the traversal boxes' margin.
//   k_inst_prims     traversal boxes (reference boxes widened by the margin of scene_pack.cpp).
//   k_refit          one launch per tree level, deepest first: each wide node's child boxes from
//                    its children's exact boxes or its leaves' traversal boxes, requantised on a
//                    new grid; the topology and the slot assignment are kept.
//   k_inst_lights    the light-triangle tables of the bidirectional tracer.
//   (host)           meanwhile, the scene-level leaf order of the object boxes (copied back right
//                    after k_inst_objbox) gives the tie ranks' bases,
//   k_inst_rank      and one thread per triangle writes its rank into its record.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../host/capi_common.h"
#include "swr_internal.cuh"

namespace swr {

// Device arrays of a scene's instance data (a plain view, passed to the kernels by value).
struct InstView {
  float4 *mesh_p, *mesh_n;      // [mesh vertices] object space
  uint32_t *vert_src, *vert_obj;
  float4 *vpos, *vnrm;          // [vertices] world space
  uint32_t* tri_v;              // [3 * triangles] world vertex ids
  uint32_t* tri_obj;
  uint32_t* local_rank;
  uint32_t* obj_first_vertex;   // [objects + 1]
  float* mats;                  // [16 * objects]
  uint32_t* base;               // [objects] rank base of each object
  uint32_t* light_src;          // [light triangles] triangle id
  float* prim_box;              // [6 * slots] traversal boxes
  float* node_box;              // [6 * nodes] exact union boxes
  uint32_t* order;              // nodes by level, deepest level first
  unsigned* ext;                // [6] ordered-int scene extent
  unsigned* bad;                // [1] set when a world vertex or normal comes out non-finite
  uint32_t nv, nt, no, nlt;
};

struct Instance {
  InstView v;
  std::vector<uint32_t> level_begin;  // offsets into order, one run per level
  std::vector<uint32_t> obj_num_tris;
  std::vector<swr_object_transform> xf;
  bool exact = true;
  std::vector<void*> allocs;
  float* host_boxes = nullptr;          // pinned [6 * objects + 1]: object boxes, then the bad flag
  cudaEvent_t boxes_ready = nullptr;    // recorded after that copy
  Instance() { std::memset(&v, 0, sizeof(v)); }
  ~Instance() {
    for (void* p : allocs) cudaFree(p);
    if (host_boxes) cudaFreeHost(host_boxes);
    if (boxes_ready) cudaEventDestroy(boxes_ready);
  }
  template <class T>
  int alloc(T** p, size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(n * sizeof(T), 16)) != cudaSuccess) {
      cudaGetLastError();
      return set_error(SWR_ERR_ALLOC, "CUDA: instance data allocation failed");
    }
    allocs.push_back(q);
    *p = (T*)q;
    return SWR_OK;
  }
  template <class T>
  int upload(T** p, const std::vector<T>& v) {
    int rc = alloc(p, v.size());
    if (rc) return rc;
    if (!v.empty()) SWR_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return SWR_OK;
  }
};

void free_instance(swr_scene* s) {
  delete (Instance*)s->instance;
  s->instance = nullptr;
}

namespace {

using swrx::fadd;
using swrx::fmul;
using swrx::fsub;

// row-vector transform r[j] = sum_i m[i][j] * v[i], accumulated from +0 over i (matrix.h:245-253)
__device__ __forceinline__ void xform(const float* m, const float v[4], float r[4]) {
  r[0] = r[1] = r[2] = r[3] = 0.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) r[j] = fadd(r[j], fmul(m[4 * i + j], v[i]));
}

__global__ void k_inst_vertices(InstView I) {
  const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= I.nv) return;
  const float* m = I.mats + 16 * (size_t)I.vert_obj[v];
  const uint32_t src = I.vert_src[v];
  const float4 p = I.mesh_p[src], n = I.mesh_n[src];
  const float pv[4] = {p.x, p.y, p.z, 1.0f}, nv[4] = {n.x, n.y, n.z, 0.0f};
  float r[4];
  xform(m, pv, r);
  I.vpos[v] = make_float4(r[0], r[1], r[2], 0.0f);
  // The object box check on the host misses a NaN in any vertex but an object's first one (the
  // reference's min/max keep the running bound against a NaN), and it never sees the normals:
  // every product that leaves finite coordinates non-finite is flagged here.
  bool bad = !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
  xform(m, nv, r);
  I.vnrm[v] = make_float4(r[0], r[1], r[2], 0.0f);
  bad |= isfinite(n.x) && isfinite(n.y) && isfinite(n.z) && !(isfinite(r[0]) && isfinite(r[1]) && isfinite(r[2]));
  if (bad) *I.bad = 1u;
}

// AABB::addPoint (aabb.cpp:26-37): the first point padded by 1e-4, then std::min(a,b) =
// (b < a) ? b : a and std::max(a,b) = (a < b) ? b : a against the running bounds
struct RefBox {
  float lo[3], hi[3];
  bool valid;
  __device__ void add(const float4& p, bool first) {
    const float q[3] = {p.x, p.y, p.z};
    if (!valid) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        lo[k] = first ? fsub(q[k], 0.0001f) : q[k];
        hi[k] = first ? fadd(q[k], 0.0001f) : q[k];
      }
      valid = true;
      return;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = (q[k] < lo[k]) ? q[k] : lo[k];
      hi[k] = (hi[k] < q[k]) ? q[k] : hi[k];
    }
  }
  // this box holds earlier vertices than b: on equal coordinates the earlier one stays
  __device__ void merge(const RefBox& b) {
    if (!b.valid) return;
    if (!valid) {
      *this = b;
      return;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      lo[k] = (b.lo[k] < lo[k]) ? b.lo[k] : lo[k];
      hi[k] = (hi[k] < b.hi[k]) ? b.hi[k] : hi[k];
    }
  }
};

__global__ void k_inst_objbox(InstView I, float* __restrict__ obj_boxes) {
  const uint32_t o = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned lane = threadIdx.x & 31u;
  if (o >= I.no) return;  // whole warps leave together
  const uint32_t v0 = I.obj_first_vertex[o], v1 = I.obj_first_vertex[o + 1];
  const uint32_t chunk = (v1 - v0 + 31u) / 32u;
  const uint32_t b = min(v1, v0 + lane * chunk), e = min(v1, b + chunk);
  RefBox box{{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, false};
  for (uint32_t v = b; v < e; ++v) box.add(I.vpos[v], v == v0);
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    RefBox other;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      other.lo[k] = __shfl_down_sync(0xffffffffu, box.lo[k], off);
      other.hi[k] = __shfl_down_sync(0xffffffffu, box.hi[k], off);
    }
    other.valid = __shfl_down_sync(0xffffffffu, box.valid ? 1 : 0, off) != 0;
    if ((lane & (2 * off - 1)) == 0) box.merge(other);
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      obj_boxes[6 * (size_t)o + k] = box.lo[k];
      obj_boxes[6 * (size_t)o + 3 + k] = box.hi[k];
    }
  }
}

// float <-> order-preserving unsigned int, for atomic min/max of floats
__device__ __forceinline__ unsigned ford(float f) {
  const unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float funord(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// dot product accumulated from +0 (vector.h:235-241)
__device__ __forceinline__ float dot0(const float a[3], const float b[3]) {
  return fadd(fadd(fadd(0.0f, fmul(a[0], b[0])), fmul(a[1], b[1])), fmul(a[2], b[2]));
}

__global__ void k_inst_derive(InstView I, DevScene sc, float4* __restrict__ tris, float4* __restrict__ shade,
                              float* __restrict__ tri_boxes) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  if (t < I.nt) {
    const uint32_t s = sc.slot_of[t];
    const uint32_t ia = I.tri_v[3 * (size_t)t], ib = I.tri_v[3 * (size_t)t + 1], ic = I.tri_v[3 * (size_t)t + 2];
    const float4 A = I.vpos[ia], B = I.vpos[ib], C = I.vpos[ic];
    const float a[3] = {A.x, A.y, A.z}, b[3] = {B.x, B.y, B.z}, c[3] = {C.x, C.y, C.z};
    float e0[3], e1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      e0[k] = fsub(b[k], a[k]);
      e1[k] = fsub(c[k], a[k]);
    }
    const float d00 = dot0(e0, e0), d01 = dot0(e0, e1), d11 = dot0(e1, e1);
    const float den = fsub(fmul(d00, d11), fmul(d01, d01));
    const uint32_t obj = I.tri_obj[t];
    tris[3 * (size_t)s + 0] = make_float4(a[0], a[1], a[2], e0[0]);
    tris[3 * (size_t)s + 1] = make_float4(e0[1], e0[2], e1[0], e1[1]);
    // the rank word is written by k_inst_rank once the object order is known
    tris[3 * (size_t)s + 2] = make_float4(e1[2], __uint_as_float(t), __uint_as_float(0u), __uint_as_float(obj));
    shade[4 * (size_t)s + 0] = make_float4(d00, d01, d11, den);
    shade[4 * (size_t)s + 1] = I.vnrm[ia];
    shade[4 * (size_t)s + 2] = I.vnrm[ib];
    shade[4 * (size_t)s + 3] = I.vnrm[ic];
    RefBox box{{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}, false};
    box.add(A, true);
    box.add(B, false);
    box.add(C, false);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      tri_boxes[6 * (size_t)s + k] = box.lo[k];
      tri_boxes[6 * (size_t)s + 3 + k] = box.hi[k];
      lo[k] = box.lo[k];
      hi[k] = box.hi[k];
    }
  }
  // scene extent: warp reduction, then one atomic per warp and bound
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float l = lo[k], h = hi[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      l = fminf(l, __shfl_xor_sync(0xffffffffu, l, off));
      h = fmaxf(h, __shfl_xor_sync(0xffffffffu, h, off));
    }
    if ((threadIdx.x & 31u) == 0) {
      if (l <= h) {
        atomicMin(&I.ext[k], ford(l));
        atomicMax(&I.ext[3 + k], ford(h));
      }
    }
  }
}

// the tie rank of triangle t (its object's base plus its place in its mesh's leaf order), into
// the rank word of its record
__global__ void k_inst_rank(InstView I, DevScene sc, float4* __restrict__ tris) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= I.nt) return;
  const uint32_t s = sc.slot_of[t];
  reinterpret_cast<uint32_t*>(tris + 3 * (size_t)s + 2)[2] = I.base[I.tri_obj[t]] + I.local_rank[t];
}

// traversal boxes: the reference triangle boxes widened by the margin scene_pack.cpp uses
__global__ void k_inst_prims(InstView I, const float* __restrict__ tri_boxes, uint32_t ns) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  float ext = 0.0f, mabs = 0.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float slo = funord(I.ext[k]), shi = funord(I.ext[3 + k]);
    ext = fmaxf(ext, fsub(shi, slo));
    mabs = fmaxf(mabs, fmaxf(fabsf(slo), fabsf(shi)));
  }
  const float eps = fadd(fadd(fmul(ext, 1.0f / 65536.0f), fmul(mabs, 1.0f / 1048576.0f)), 1e-30f);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    I.prim_box[6 * (size_t)s + k] = fsub(tri_boxes[6 * (size_t)s + k], eps);
    I.prim_box[6 * (size_t)s + 3 + k] = fadd(tri_boxes[6 * (size_t)s + 3 + k], eps);
  }
}

__global__ void k_refit(InstView I, uint32_t* __restrict__ words, uint32_t begin, uint32_t end) {
  const uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= end) return;
  const uint32_t n = I.order[k];
  uint32_t* w = words + (size_t)n * 20;
  const uint32_t imask = w[3] >> 24, child_base = w[4], tri_base = w[5];
  const uint32_t meta0 = w[6], meta1 = w[7];
  float clo[8][3], chi[8][3];
  bool used[8];
  float ulo[3] = {INFINITY, INFINITY, INFINITY}, uhi[3] = {-INFINITY, -INFINITY, -INFINITY};
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const uint32_t m = ((s < 4 ? meta0 : meta1) >> (8 * (s & 3))) & 0xFFu;
    const bool inner = (imask >> s) & 1u;
    used[s] = inner || m != 0u;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      clo[s][q] = INFINITY;
      chi[s][q] = -INFINITY;
    }
    if (inner) {
      const uint32_t c = child_base + (uint32_t)__popc(imask & ((1u << s) - 1u));
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        clo[s][q] = I.node_box[6 * (size_t)c + q];
        chi[s][q] = I.node_box[6 * (size_t)c + 3 + q];
      }
    } else if (m != 0u) {
      const uint32_t cnt = m >> 5, off = m & 31u;
      for (uint32_t j = 0; j < cnt; ++j) {
        const float* pb = I.prim_box + 6 * (size_t)(tri_base + off + j);
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          clo[s][q] = fminf(clo[s][q], pb[q]);
          chi[s][q] = fmaxf(chi[s][q], pb[3 + q]);
        }
      }
    }
    if (used[s]) {
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        ulo[q] = fminf(ulo[q], clo[s][q]);
        uhi[q] = fmaxf(uhi[q], chi[s][q]);
      }
    }
  }
  // quantisation grid of the builder: per axis the smallest power of two e with 255 e >= extent
  uint32_t ebyte[3];
  double e[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double ex_d = (double)uhi[q] - (double)ulo[q];
    int ex = -126;
    if (ex_d > 0.0) {
      int x;
      frexp(ex_d / 255.0, &x);
      ex = x;
      if (ldexp(1.0, ex - 1) >= ex_d / 255.0) ex = ex - 1;
    }
    ex = max(-126, min(127, ex));
    ebyte[q] = (uint32_t)(ex + 127);
    e[q] = ldexp(1.0, ex);
  }
  uint32_t qlo[3][2] = {{0, 0}, {0, 0}, {0, 0}}, qhi[3][2] = {{0, 0}, {0, 0}, {0, 0}};
#pragma unroll
  for (int s = 0; s < 8; ++s) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      uint32_t l = 255u, h = 0u;
      if (used[s]) {
        const double lo = floor(((double)clo[s][q] - (double)ulo[q]) / e[q]);
        const double hi = ceil(((double)chi[s][q] - (double)ulo[q]) / e[q]);
        l = (uint32_t)fmax(0.0, fmin(255.0, lo));
        h = (uint32_t)fmax(0.0, fmin(255.0, hi));
      }
      qlo[q][s >> 2] |= l << (8 * (s & 3));
      qhi[q][s >> 2] |= h << (8 * (s & 3));
    }
  }
  w[0] = __float_as_uint(ulo[0]);
  w[1] = __float_as_uint(ulo[1]);
  w[2] = __float_as_uint(ulo[2]);
  w[3] = ebyte[0] | (ebyte[1] << 8) | (ebyte[2] << 16) | (imask << 24);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    w[8 + 2 * q] = qlo[q][0];
    w[9 + 2 * q] = qlo[q][1];
    w[14 + 2 * q] = qhi[q][0];
    w[15 + 2 * q] = qhi[q][1];
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    I.node_box[6 * (size_t)n + q] = ulo[q];
    I.node_box[6 * (size_t)n + 3 + q] = uhi[q];
  }
}

// light tables (scene_pack.cpp): corners v0 v1 v2, then corner normals n0 n1 n2, 5 float4
__global__ void k_inst_lights(InstView I, float4* __restrict__ light_tris) {
  const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= I.nlt) return;
  const uint32_t t = I.light_src[q];
  float w[20];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const uint32_t v = I.tri_v[3 * (size_t)t + c];
    const float4 p = I.vpos[v], n = I.vnrm[v];
    w[3 * c] = p.x;
    w[3 * c + 1] = p.y;
    w[3 * c + 2] = p.z;
    w[9 + 3 * c] = n.x;
    w[9 + 3 * c + 1] = n.y;
    w[9 + 3 * c + 2] = n.z;
  }
  w[18] = w[19] = 0.0f;
#pragma unroll
  for (int k = 0; k < 5; ++k) light_tris[5 * (size_t)q + k] = make_float4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
}

unsigned blocks(size_t n, unsigned b) { return (unsigned)std::max<size_t>(1, (n + b - 1) / b); }

int attach(swr_scene* s, const swr_host_scene* hs, const swr_scene_desc& d) {
  InstanceSource src;
  instance_source(hs, src);
  std::unique_ptr<Instance> I(new Instance());
  I->v.nv = d.num_vertices;
  I->v.nt = d.num_triangles;
  I->v.no = d.num_objects;
  I->xf = src.xf;
  I->exact = src.scene_order_exact;
  I->obj_num_tris.resize(I->v.no);
  for (uint32_t o = 0; o < I->v.no; ++o) I->obj_num_tris[o] = src.obj_first_tri[o + 1] - src.obj_first_tri[o];
  const size_t nmv = src.mesh_pos.size() / 3;
  std::vector<float4> mp(nmv), mn(nmv);
  for (size_t i = 0; i < nmv; ++i) {
    mp[i] = make_float4(src.mesh_pos[3 * i], src.mesh_pos[3 * i + 1], src.mesh_pos[3 * i + 2], 0.0f);
    mn[i] = make_float4(src.mesh_nrm[3 * i], src.mesh_nrm[3 * i + 1], src.mesh_nrm[3 * i + 2], 0.0f);
  }
  int rc;
  if ((rc = I->upload(&I->v.mesh_p, mp))) return rc;
  if ((rc = I->upload(&I->v.mesh_n, mn))) return rc;
  if ((rc = I->upload(&I->v.vert_src, src.vert_src))) return rc;
  if ((rc = I->upload(&I->v.vert_obj, src.vert_obj))) return rc;
  if ((rc = I->alloc(&I->v.vpos, I->v.nv))) return rc;
  if ((rc = I->alloc(&I->v.vnrm, I->v.nv))) return rc;
  if ((rc = I->upload(&I->v.tri_v, std::vector<uint32_t>(d.tri_vertices, d.tri_vertices + 3 * (size_t)I->v.nt))))
    return rc;
  if ((rc = I->upload(&I->v.tri_obj, std::vector<uint32_t>(d.tri_object, d.tri_object + I->v.nt)))) return rc;
  if ((rc = I->upload(&I->v.local_rank, src.local_rank))) return rc;
  if ((rc = I->upload(&I->v.obj_first_vertex, src.obj_first_vertex))) return rc;
  if ((rc = I->alloc(&I->v.mats, 16 * (size_t)I->v.no))) return rc;
  if ((rc = I->alloc(&I->v.base, I->v.no))) return rc;
  // light triangles in the order scene_pack.cpp lists them: light objects in object order
  std::vector<uint32_t> lsrc;
  for (uint32_t o = 0; o < I->v.no; ++o)
    if (d.materials[o].light_source)
      for (uint32_t t = src.obj_first_tri[o]; t < src.obj_first_tri[o + 1]; ++t) lsrc.push_back(t);
  I->v.nlt = (uint32_t)lsrc.size();
  if ((rc = I->upload(&I->v.light_src, lsrc))) return rc;
  if ((rc = I->alloc(&I->v.prim_box, 6 * (size_t)s->dev.num_slots))) return rc;
  if ((rc = I->alloc(&I->v.node_box, 6 * (size_t)s->dev.num_nodes))) return rc;
  if ((rc = I->alloc(&I->v.ext, 6))) return rc;
  if ((rc = I->alloc(&I->v.bad, 1))) return rc;
  if (cudaMallocHost(&I->host_boxes, sizeof(float) * (6 * std::max<size_t>(I->v.no, 1) + 1)) != cudaSuccess) {
    cudaGetLastError();
    I->host_boxes = nullptr;
    return set_error(SWR_ERR_ALLOC, "CUDA: pinned host allocation failed");
  }
  SWR_CUDA(cudaEventCreateWithFlags(&I->boxes_ready, cudaEventDisableTiming));
  // tree levels from the node records: inner children of node n are child_base + i
  const uint32_t nn = s->dev.num_nodes;
  std::vector<uint32_t> words((size_t)nn * 20);
  SWR_CUDA(cudaMemcpy(words.data(), s->d_nodes, words.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  std::vector<uint32_t> level(nn, 0xFFFFFFFFu), q{0};
  level[0] = 0;
  uint32_t depth = 0;
  for (size_t h = 0; h < q.size(); ++h) {
    const uint32_t n = q[h];
    const uint32_t imask = words[(size_t)n * 20 + 3] >> 24, cb = words[(size_t)n * 20 + 4];
    for (uint32_t i = 0; i < (uint32_t)__builtin_popcount(imask); ++i) {
      const uint32_t c = cb + i;
      if (c >= nn || level[c] != 0xFFFFFFFFu) return set_error(SWR_ERR_INVALID, "swr: malformed BVH records");
      level[c] = level[n] + 1;
      depth = std::max(depth, level[c]);
      q.push_back(c);
    }
  }
  if (q.size() != nn) return set_error(SWR_ERR_INVALID, "swr: BVH records not reachable from the root");
  std::vector<uint32_t> order;
  order.reserve(nn);
  for (int L = (int)depth; L >= 0; --L) {
    I->level_begin.push_back((uint32_t)order.size());
    for (uint32_t n = 0; n < nn; ++n)
      if (level[n] == (uint32_t)L) order.push_back(n);
  }
  I->level_begin.push_back((uint32_t)order.size());
  if ((rc = I->upload(&I->v.order, order))) return rc;
  s->instance = I.release();
  return SWR_OK;
}

}  // namespace
}  // namespace swr

using swr::set_error;

extern "C" {

int swr_scene_create_from_host(const swr_host_scene* hs, const swr_build_opts* opts, swr_scene** out) {
  if (!hs || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  *out = nullptr;
  swr_scene_desc d;
  int rc = swr_host_scene_desc(hs, &d);
  if (rc) return rc;
  swr_scene* s = nullptr;
  if ((rc = swr_scene_create(&d, opts, &s))) return rc;
  try {
    rc = swr::attach(s, hs, d);
  } catch (const std::bad_alloc&) {
    rc = set_error(SWR_ERR_ALLOC, "swr: host allocation failed");
  }
  if (rc) {
    swr_scene_destroy(s);
    return rc;
  }
  *out = s;
  return SWR_OK;
}

int swr_scene_set_transforms(swr_scene* s, const swr_object_transform* xf, uint32_t n, void* stream_) {
  if (!s || !xf) return set_error(SWR_ERR_INVALID, "swr: null argument");
  swr::Instance* I = (swr::Instance*)s->instance;
  if (!I) return set_error(SWR_ERR_INVALID, "swr: the scene was not made by swr_scene_create_from_host");
  if (n != I->v.no) return set_error(SWR_ERR_INVALID, "swr: one transform per object is required");
  for (uint32_t o = 0; o < n; ++o) {
    const float* f = &xf[o].position[0];
    for (int k = 0; k < 10; ++k)
      if (!std::isfinite(f[k])) return set_error(SWR_ERR_INVALID, "swr: non-finite object transform");
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  std::vector<float> mats(16 * (size_t)n);
  for (uint32_t o = 0; o < n; ++o) swr::object_matrix(xf[o], mats.data() + 16 * (size_t)o);
  SWR_CUDA(cudaMemcpyAsync(I->v.mats, mats.data(), mats.size() * sizeof(float), cudaMemcpyHostToDevice, stream));
  SWR_CUDA(cudaMemsetAsync(I->v.bad, 0, sizeof(unsigned), stream));
  swr::k_inst_vertices<<<swr::blocks(I->v.nv, 256), 256, 0, stream>>>(I->v);
  swr::k_inst_objbox<<<swr::blocks((size_t)I->v.no * 32, 256), 256, 0, stream>>>(I->v, (float*)s->d_obj_boxes);
  SWR_CUDA(cudaGetLastError());
  // the object boxes come back first; the triangle records, traversal boxes, refit and light
  // tables (none of which needs the tie ranks) run on the GPU while the host orders the objects
  SWR_CUDA(cudaMemcpyAsync(I->host_boxes, s->d_obj_boxes, 6 * sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost,
                           stream));
  SWR_CUDA(cudaMemcpyAsync(I->host_boxes + 6 * (size_t)n, I->v.bad, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
  SWR_CUDA(cudaEventRecord(I->boxes_ready, stream));
  const unsigned init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  SWR_CUDA(cudaMemcpyAsync(I->v.ext, init, sizeof(init), cudaMemcpyHostToDevice, stream));
  swr::k_inst_derive<<<swr::blocks(I->v.nt, 256), 256, 0, stream>>>(I->v, s->dev, (float4*)s->d_tris,
                                                                   (float4*)s->d_shade, (float*)s->d_tri_boxes);
  swr::k_inst_prims<<<swr::blocks(s->dev.num_slots, 256), 256, 0, stream>>>(I->v, (const float*)s->d_tri_boxes,
                                                                              s->dev.num_slots);
  for (size_t L = 0; L + 1 < I->level_begin.size(); ++L) {
    const uint32_t b = I->level_begin[L], e = I->level_begin[L + 1];
    if (e > b) swr::k_refit<<<swr::blocks(e - b, 128), 128, 0, stream>>>(I->v, (uint32_t*)s->d_nodes, b, e);
  }
  if (I->v.nlt) swr::k_inst_lights<<<swr::blocks(I->v.nlt, 128), 128, 0, stream>>>(I->v, (float4*)s->d_light_tris);
  SWR_CUDA(cudaGetLastError());
  // tie ranks: the scene-level order of the moved objects' boxes (SceneBuilder::finish)
  SWR_CUDA(cudaEventSynchronize(I->boxes_ready));
  const float* boxes = I->host_boxes;
  unsigned bad = 0;
  std::memcpy(&bad, boxes + 6 * (size_t)n, sizeof(bad));
  for (size_t i = 0; i < 6 * (size_t)n && !bad; ++i) bad = !std::isfinite(boxes[i]);
  if (bad) {
    SWR_CUDA(cudaStreamSynchronize(stream));
    return set_error(SWR_ERR_INVALID, "swr: the transforms give non-finite coordinates or normals");
  }
  const std::vector<uint32_t> order = swr::object_order(boxes, n, I->exact);
  std::vector<uint32_t> base(n, 0);
  uint32_t acc = 0;
  for (uint32_t o : order) {
    base[o] = acc;
    acc += I->obj_num_tris[o];
  }
  SWR_CUDA(cudaMemcpyAsync(I->v.base, base.data(), base.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, stream));
  swr::k_inst_rank<<<swr::blocks(I->v.nt, 256), 256, 0, stream>>>(I->v, s->dev, (float4*)s->d_tris);
  SWR_CUDA(cudaGetLastError());
  std::copy(xf, xf + n, I->xf.begin());
  SWR_CUDA(cudaStreamSynchronize(stream));  // the host arrays above go out of scope
  return SWR_OK;
}

}  // extern "C"
