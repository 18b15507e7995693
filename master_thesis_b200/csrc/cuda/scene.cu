// Device scene construction and the closest-hit query (C ABI: swr_scene_create / destroy /
// stats / swr_trace_closest / swr_trace_closest_stats / swr_sync).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "../host/capi_common.h"
#include "../host/wide_bvh.h"
#include "swr_internal.cuh"

namespace swr {

int cuda_fail(cudaError_t err, const char* what) {
  return set_error(SWR_ERR_CUDA, std::string("CUDA: ") + what + ": " + cudaGetErrorString(err));
}

bool is_host_pointer(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeUnregistered;
}

namespace {

template <class T>
int upload(void** dst, const std::vector<T>& v) {
  const size_t bytes = std::max<size_t>(v.size() * sizeof(T), 16);
  cudaError_t e = cudaMalloc(dst, bytes);
  if (e != cudaSuccess) {
    *dst = nullptr;
    return set_error(SWR_ERR_ALLOC, std::string("CUDA: cudaMalloc of ") + std::to_string(bytes) +
                                        " bytes failed: " + cudaGetErrorString(e));
  }
  if (!v.empty()) SWR_CUDA(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return SWR_OK;
}

inline float ubits(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

constexpr int kTraceBlock = 128;

template <bool kStats>
__global__ void __launch_bounds__(kTraceBlock)
    k_trace_closest(DevScene sc, const float4* __restrict__ ro, const float4* __restrict__ rd,
                    uint64_t n, uint4* __restrict__ out, uint2* __restrict__ counts,
                    unsigned long long* __restrict__ cursor) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(cursor, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const uint64_t i = base + lane;
    if (i < n) {
      const float4 o = ro[i], d = rd[i];
      swrx::Hit h;
      swrx::TraceStats st{0, 0};
      swrx::trace_closest<kStats>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes,
                                  swrx::mk(o.x, o.y, o.z), swrx::mk(d.x, d.y, d.z),
                                  stack + threadIdx.x, kTraceBlock, h, &st);
      out[i] = make_uint4(h.id, h.obj, __float_as_uint(h.d2), __float_as_uint(h.t));
      if (kStats) counts[i] = make_uint2(st.nodes, st.tris);
    }
  }
}

int trace_impl(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n, swr_hit* out,
               uint32_t* counts, void* stream_) {
  if (!s || !ray_o || !ray_d || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (n == 0) return SWR_OK;
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  const bool ho = is_host_pointer(ray_o), hd = is_host_pointer(ray_d), hh = is_host_pointer(out);
  const bool hc = counts && is_host_pointer(counts);
  const float4* dro = (const float4*)ray_o;
  const float4* drd = (const float4*)ray_d;
  uint4* dout = (uint4*)out;
  uint2* dcnt = (uint2*)counts;
  void* tmp[4] = {nullptr, nullptr, nullptr, nullptr};
  auto cleanup = [&]() {
    for (void* p : tmp)
      if (p) cudaFreeAsync(p, stream);
  };
  const size_t rb = (size_t)n * 16;
  if (ho) {
    SWR_CUDA(cudaMallocAsync(&tmp[0], rb, stream));
    SWR_CUDA(cudaMemcpyAsync(tmp[0], ray_o, rb, cudaMemcpyHostToDevice, stream));
    dro = (const float4*)tmp[0];
  }
  if (hd) {
    SWR_CUDA(cudaMallocAsync(&tmp[1], rb, stream));
    SWR_CUDA(cudaMemcpyAsync(tmp[1], ray_d, rb, cudaMemcpyHostToDevice, stream));
    drd = (const float4*)tmp[1];
  }
  if (hh) {
    SWR_CUDA(cudaMallocAsync(&tmp[2], rb, stream));
    dout = (uint4*)tmp[2];
  }
  if (hc) {
    SWR_CUDA(cudaMallocAsync(&tmp[3], (size_t)n * 8, stream));
    dcnt = (uint2*)tmp[3];
  }
  if (((uintptr_t)dro | (uintptr_t)drd | (uintptr_t)dout) & 15) {
    cleanup();
    return set_error(SWR_ERR_INVALID, "swr: ray and hit buffers must be 16-byte aligned");
  }
  unsigned long long* cursor = (unsigned long long*)s->d_scratch;
  SWR_CUDA(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), stream));
  int per_sm = 0;
  if (counts)
    SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_closest<true>, kTraceBlock, 0));
  else
    SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_closest<false>, kTraceBlock, 0));
  per_sm = std::max(per_sm, 1);
  const uint64_t max_blocks = (n + kTraceBlock - 1) / kTraceBlock;
  const unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)s->num_sms * per_sm, max_blocks);
  if (counts)
    k_trace_closest<true><<<grid, kTraceBlock, 0, stream>>>(s->dev, dro, drd, n, dout, dcnt, cursor);
  else
    k_trace_closest<false><<<grid, kTraceBlock, 0, stream>>>(s->dev, dro, drd, n, dout, nullptr, cursor);
  SWR_CUDA(cudaGetLastError());
  if (hh) SWR_CUDA(cudaMemcpyAsync(out, dout, rb, cudaMemcpyDeviceToHost, stream));
  if (hc) SWR_CUDA(cudaMemcpyAsync(counts, dcnt, (size_t)n * 8, cudaMemcpyDeviceToHost, stream));
  cleanup();
  if (ho || hd || hh || hc) SWR_CUDA(cudaStreamSynchronize(stream));
  return SWR_OK;
}

}  // namespace
}  // namespace swr

using swr::set_error;

extern "C" {

int swr_sync(void* stream) {
  SWR_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  return SWR_OK;
}

int swr_scene_create(const swr_scene_desc* d, const swr_build_opts* opts, swr_scene** out) {
  if (!out) return set_error(SWR_ERR_INVALID, "swr: null output handle");
  *out = nullptr;
  int rc = swr::validate_desc(d);
  if (rc) return rc;
  try {
    swr::Derived dv;
    swr::derive(*d, dv);
    const uint32_t nt = d->num_triangles, no = d->num_objects;
    // traversal boxes: the reference boxes, enlarged by a margin tied to the scene's scale so
    // that rounding in the quantised slab tests can never lose a box the reference's test hits
    float slo[3] = {INFINITY, INFINITY, INFINITY}, shi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) {
        slo[k] = std::min(slo[k], dv.tri_box[t].lo[k]);
        shi[k] = std::max(shi[k], dv.tri_box[t].hi[k]);
      }
    float ext = 0.0f, mabs = 0.0f;
    for (int k = 0; k < 3; ++k) {
      ext = std::max(ext, shi[k] - slo[k]);
      mabs = std::max(mabs, std::max(std::fabs(slo[k]), std::fabs(shi[k])));
    }
    if (!std::isfinite(ext) || !std::isfinite(mabs))
      return set_error(SWR_ERR_INVALID, "swr: scene has non-finite vertex coordinates");
    const float eps = ext * (1.0f / 65536.0f) + mabs * (1.0f / 1048576.0f) + 1e-30f;
    std::vector<swr::PrimBox> prims(nt);
    for (uint32_t t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) {
        prims[t].lo[k] = dv.tri_box[t].lo[k] - eps;
        prims[t].hi[k] = dv.tri_box[t].hi[k] + eps;
      }
    swr::WideBvhOptions wo;
    if (opts) {
      if (opts->sah_bins) wo.sah_bins = opts->sah_bins;
      if (opts->max_leaf) wo.max_leaf = opts->max_leaf;
      wo.threads = opts->threads;
    }
    if (wo.max_leaf > 3) return set_error(SWR_ERR_INVALID, "swr: max_leaf must be 1..3");
    swr::WideBvh bvh = swr::build_wide_bvh(prims, wo);
    if (bvh.depth + 1 > (uint32_t)swrx::kStackTotal)
      return set_error(SWR_ERR_UNSUPPORTED, "swr: BVH deeper than the traversal stack");

    const uint32_t ns = (uint32_t)bvh.prim_order.size();
    std::vector<float4> tris((size_t)ns * 3), shade((size_t)ns * 4);
    std::vector<float> tboxes((size_t)ns * 6), albedo((size_t)ns * 3), oboxes((size_t)no * 6);
    std::vector<uint32_t> slot_of(nt);
    std::unique_ptr<swr_scene> s(new swr_scene());
    s->slot_to_id.resize(ns);
    for (uint32_t sl = 0; sl < ns; ++sl) {
      const uint32_t t = bvh.prim_order[sl];
      slot_of[t] = sl;
      s->slot_to_id[sl] = t;
      const uint32_t obj = d->tri_object[t];
      const uint32_t rank = d->tri_rank ? d->tri_rank[t] : t;
      const swr::V3 &v0 = dv.v0[t], &e0 = dv.e0[t], &e1 = dv.e1[t];
      tris[3 * (size_t)sl + 0] = make_float4(v0[0], v0[1], v0[2], e0[0]);
      tris[3 * (size_t)sl + 1] = make_float4(e0[1], e0[2], e1[0], e1[1]);
      tris[3 * (size_t)sl + 2] = make_float4(e1[2], swr::ubits(t), swr::ubits(rank), swr::ubits(obj));
      shade[4 * (size_t)sl] = make_float4(dv.den[t][0], dv.den[t][1], dv.den[t][2], dv.den[t][3]);
      for (int c = 0; c < 3; ++c) {
        const uint32_t vi = d->tri_vertices[3 * (size_t)t + c];
        const float* nv = d->vertex_normal + 3 * (size_t)vi;
        shade[4 * (size_t)sl + 1 + c] = make_float4(nv[0], nv[1], nv[2], 0.0f);
      }
      for (int k = 0; k < 3; ++k) {
        tboxes[6 * (size_t)sl + k] = dv.tri_box[t].lo[k];
        tboxes[6 * (size_t)sl + 3 + k] = dv.tri_box[t].hi[k];
        albedo[3 * (size_t)sl + k] = d->tri_albedo ? d->tri_albedo[3 * (size_t)t + k] : d->materials[obj].color[k];
      }
    }
    std::vector<float4> mats((size_t)no * 3);
    for (uint32_t o = 0; o < no; ++o) {
      const swr_material& m = d->materials[o];
      for (int k = 0; k < 3; ++k) {
        oboxes[6 * (size_t)o + k] = dv.obj_box[o].lo[k];
        oboxes[6 * (size_t)o + 3 + k] = dv.obj_box[o].hi[k];
      }
      mats[3 * (size_t)o + 0] = make_float4(m.color[0], m.color[1], m.color[2], m.diffuse_t);
      mats[3 * (size_t)o + 1] = make_float4(m.reflect_t, m.transparent_t, m.refraction_index,
                                            swr::ubits(m.light_source ? 1u : 0u));
      mats[3 * (size_t)o + 2] = make_float4(m.color[0] * m.light_strength, m.color[1] * m.light_strength,
                                            m.color[2] * m.light_strength, m.light_strength);
    }
    SWR_CUDA(cudaGetDevice(&s->device));
    SWR_CUDA(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device));
    struct Guard {
      swr_scene* p;
      ~Guard() {
        if (p) swr_scene_destroy(p);
      }
    } guard{s.get()};
    if ((rc = swr::upload(&s->d_nodes, bvh.words))) return rc;
    if ((rc = swr::upload(&s->d_tris, tris))) return rc;
    if ((rc = swr::upload(&s->d_shade, shade))) return rc;
    if ((rc = swr::upload(&s->d_tri_boxes, tboxes))) return rc;
    if ((rc = swr::upload(&s->d_obj_boxes, oboxes))) return rc;
    if ((rc = swr::upload(&s->d_mats, mats))) return rc;
    if ((rc = swr::upload(&s->d_albedo, albedo))) return rc;
    if ((rc = swr::upload(&s->d_slot_of, slot_of))) return rc;
    s->scratch_bytes = 256;
    SWR_CUDA(cudaMalloc(&s->d_scratch, s->scratch_bytes));
    SWR_CUDA(cudaMemset(s->d_scratch, 0, s->scratch_bytes));
    swr::DevScene& ds = s->dev;
    ds.nodes = (const float4*)s->d_nodes;
    ds.tris = (const float4*)s->d_tris;
    ds.shade = (const float4*)s->d_shade;
    ds.tri_boxes = (const float*)s->d_tri_boxes;
    ds.obj_boxes = (const float*)s->d_obj_boxes;
    ds.mats = (const float4*)s->d_mats;
    ds.albedo = (const float*)s->d_albedo;
    ds.slot_of = (const uint32_t*)s->d_slot_of;
    ds.num_nodes = bvh.num_nodes;
    ds.num_slots = ns;
    ds.num_objects = no;
    ds.num_tris = nt;
    s->depth = bvh.depth;
    s->node_bytes = (uint64_t)bvh.num_nodes * 80;
    s->tri_bytes = (uint64_t)ns * 48;
    guard.p = nullptr;
    *out = s.release();
    return SWR_OK;
  } catch (const std::bad_alloc&) {
    return set_error(SWR_ERR_ALLOC, "swr: host allocation failed");
  } catch (const std::exception& e) {
    return set_error(SWR_ERR_INVALID, std::string("swr: ") + e.what());
  }
}

void swr_scene_destroy(swr_scene* s) {
  if (!s) return;
  swr::free_workspace(s);
  for (void* p : {s->d_nodes, s->d_tris, s->d_shade, s->d_tri_boxes, s->d_obj_boxes, s->d_mats,
                  s->d_albedo, s->d_slot_of, s->d_scratch})
    if (p) cudaFree(p);
  delete s;
}

int swr_scene_stats(const swr_scene* s, uint64_t out[8]) {
  if (!s || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  out[0] = s->dev.num_nodes;
  out[1] = s->depth;
  out[2] = s->node_bytes;
  out[3] = s->tri_bytes;
  out[4] = s->dev.num_tris;
  out[5] = s->dev.num_objects;
  out[6] = 80;
  out[7] = 48;
  return SWR_OK;
}

int swr_trace_closest(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n, swr_hit* out,
                      void* stream) {
  return swr::trace_impl(s, ray_o, ray_d, n, out, nullptr, stream);
}

int swr_trace_closest_stats(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n,
                            swr_hit* out, uint32_t* counts, void* stream) {
  if (!counts) return set_error(SWR_ERR_INVALID, "swr: null counts");
  return swr::trace_impl(s, ray_o, ray_d, n, out, counts, stream);
}

}  // extern "C"
