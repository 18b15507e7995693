// Device scene construction and the closest-hit query (C ABI: swr_scene_create / destroy /
// stats / swr_trace_closest / swr_trace_closest_stats / swr_sync).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "../host/capi_common.h"
#include "../host/scene_pack.h"
#include "build_device.h"
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

// Triangle-id-ordered records -> leaf order of the device-built BVH.
__global__ void k_permute(const uint32_t* __restrict__ order, uint32_t n, const float4* __restrict__ tris_in,
                          const float4* __restrict__ shade_in, const float* __restrict__ box_in,
                          const float* __restrict__ alb_in, float4* __restrict__ tris, float4* __restrict__ shade,
                          float* __restrict__ boxes, float* __restrict__ alb, uint32_t* __restrict__ slot_of) {
  const uint32_t sl = blockIdx.x * blockDim.x + threadIdx.x;
  if (sl >= n) return;
  const uint32_t t = order[sl];
  for (int k = 0; k < 3; ++k) tris[3 * (size_t)sl + k] = tris_in[3 * (size_t)t + k];
  for (int k = 0; k < 4; ++k) shade[4 * (size_t)sl + k] = shade_in[4 * (size_t)t + k];
  for (int k = 0; k < 6; ++k) boxes[6 * (size_t)sl + k] = box_in[6 * (size_t)t + k];
  for (int k = 0; k < 3; ++k) alb[3 * (size_t)sl + k] = alb_in[3 * (size_t)t + k];
  slot_of[t] = sl;
}

// Device BVH build (swr_build_opts.builder == SWR_BUILD_DEVICE): pk holds the records in
// triangle-id order and the traversal boxes; the wide BVH is built on the GPU and the records
// are permuted into its leaf order there.
int device_pack(swr_scene* s, const swr_scene_desc* d, const swr_build_opts* opts, PackedScene& pk) {
  const uint32_t n = d->num_triangles;
  DeviceBuildOptions o;
  if (opts) {
    if (opts->max_leaf) o.max_leaf = opts->max_leaf;
    if (opts->radius) o.radius = opts->radius;
    if (opts->leaf_cost_pct) o.prim_cost = opts->leaf_cost_pct / 100.0;
    if (opts->width) o.width = opts->width;
  }
  cudaStream_t st = nullptr;
  void *boxes = nullptr, *tris = nullptr, *shade = nullptr, *tboxes = nullptr, *alb = nullptr;
  struct Free {
    void** p[5];
    ~Free() {
      for (void** q : p)
        if (*q) cudaFree(*q);
    }
  } fr{{&boxes, &tris, &shade, &tboxes, &alb}};
  int rc;
  if ((rc = upload(&boxes, pk.prim_boxes)) || (rc = upload(&tris, pk.tris)) || (rc = upload(&shade, pk.shade)) ||
      (rc = upload(&tboxes, pk.tri_boxes)) || (rc = upload(&alb, pk.albedo)))
    return rc;
  DeviceBvh bvh;
  rc = build_wide_bvh_device((const float*)boxes, n, o, bvh, st);
  s->d_nodes = bvh.d_nodes;  // released with the scene on every path
  struct FreeOrder {
    uint32_t* p;
    ~FreeOrder() {
      if (p) cudaFree(p);
    }
  } fo{bvh.d_prim_order};
  if (rc) return rc;
  if (2 * bvh.depth + 2 > 64) return set_error(SWR_ERR_UNSUPPORTED, "swr: BVH deeper than the traversal stack");
  SWR_CUDA(cudaMalloc(&s->d_tris, (size_t)n * 3 * sizeof(float4)));
  SWR_CUDA(cudaMalloc(&s->d_shade, (size_t)n * 4 * sizeof(float4)));
  SWR_CUDA(cudaMalloc(&s->d_tri_boxes, (size_t)n * 6 * sizeof(float)));
  SWR_CUDA(cudaMalloc(&s->d_albedo, (size_t)n * 3 * sizeof(float)));
  SWR_CUDA(cudaMalloc(&s->d_slot_of, (size_t)n * sizeof(uint32_t)));
  k_permute<<<(n + 255) / 256, 256, 0, st>>>(bvh.d_prim_order, n, (const float4*)tris, (const float4*)shade,
                                            (const float*)tboxes, (const float*)alb, (float4*)s->d_tris,
                                            (float4*)s->d_shade, (float*)s->d_tri_boxes, (float*)s->d_albedo,
                                            (uint32_t*)s->d_slot_of);
  SWR_CUDA(cudaGetLastError());
  pk.slot_to_id.resize(n);
  SWR_CUDA(cudaMemcpy(pk.slot_to_id.data(), bvh.d_prim_order, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  pk.num_nodes = bvh.num_nodes;
  pk.depth = bvh.depth;
  return SWR_OK;
}

constexpr int kTraceBlock = 128;

// albedo given per triangle id -> the per-slot array the kernels read
__global__ void k_set_albedo(const uint32_t* __restrict__ slot_of, const float* __restrict__ by_id,
                             float* __restrict__ by_slot, uint32_t n) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const uint32_t s = slot_of[t];
  by_slot[3 * (size_t)s + 0] = by_id[3 * (size_t)t + 0];
  by_slot[3 * (size_t)s + 1] = by_id[3 * (size_t)t + 1];
  by_slot[3 * (size_t)s + 2] = by_id[3 * (size_t)t + 2];
}

// emitted radiance per object -> the third record of each material
__global__ void k_set_emission(float4* __restrict__ mats, const float* __restrict__ em, uint32_t n) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  float4 m = mats[3 * (size_t)o + 2];
  m.x = em[3 * (size_t)o + 0];
  m.y = em[3 * (size_t)o + 1];
  m.z = em[3 * (size_t)o + 2];
  mats[3 * (size_t)o + 2] = m;
}

// copies host input to a temporary device buffer when needed; returns the device pointer
int device_input(const float* p, size_t bytes, cudaStream_t stream, void** tmp, const float** dev) {
  *tmp = nullptr;
  *dev = p;
  if (!is_host_pointer(p)) return SWR_OK;
  SWR_CUDA(cudaMallocAsync(tmp, bytes, stream));
  SWR_CUDA(cudaMemcpyAsync(*tmp, p, bytes, cudaMemcpyHostToDevice, stream));
  *dev = (const float*)*tmp;
  return SWR_OK;
}

// Persistent closest-hit queries with per-lane refill: each lane keeps one ray's resumable
// traversal; once at least kRefill lanes of a warp are idle the warp takes that many new rays
// with one atomic on the cursor, so lanes stay busy while long rays are still walking the tree.
constexpr unsigned kRefill = 8;

template <bool kStats, int kRule = swrx::kRuleReference>
__global__ void __launch_bounds__(kTraceBlock)
    k_trace_closest(DevScene sc, const float4* __restrict__ ro, const float4* __restrict__ rd,
                    uint64_t n, uint4* __restrict__ out, uint2* __restrict__ counts,
                    unsigned long long* __restrict__ cursor) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  swrx::Traversal tr;
  swrx::TraceStats st{0, 0};
  bool active = false, exhausted = false;
  uint64_t ray = 0;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= kRefill) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(cursor, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) exhausted = true;
      if (!active) {
        const uint64_t j = base + (unsigned)__popc(idle & lt);
        if (j < n) {
          const float4 o = ro[j], d = rd[j];
          tr.init(swrx::mk(o.x, o.y, o.z), swrx::mk(d.x, d.y, d.z), stack + threadIdx.x, kTraceBlock);
          st = swrx::TraceStats{0, 0};
          ray = j;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tr.template step<kStats, false, kRule>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, &st)) {
      const swrx::Hit h = tr.result(sc.tris);
      out[ray] = make_uint4(h.id, h.obj, __float_as_uint(h.d2), __float_as_uint(h.t));
      if (kStats) counts[ray] = make_uint2(st.nodes, st.tris);
      active = false;
    }
  }
}

int trace_impl(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n, swr_hit* out,
               uint32_t* counts, void* stream_, int rule = swrx::kRuleReference) {
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
  const bool rq = rule == swrx::kRuleRayQuery;
  if (rq)
    SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, k_trace_closest<false, swrx::kRuleRayQuery>, kTraceBlock, 0));
  else if (counts)
    SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_closest<true>, kTraceBlock, 0));
  else
    SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trace_closest<false>, kTraceBlock, 0));
  per_sm = std::max(per_sm, 1);
  const uint64_t max_blocks = (n + kTraceBlock - 1) / kTraceBlock;
  const unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)s->num_sms * per_sm, max_blocks);
  if (rq)
    k_trace_closest<false, swrx::kRuleRayQuery>
        <<<grid, kTraceBlock, 0, stream>>>(s->dev, dro, drd, n, dout, nullptr, cursor);
  else if (counts)
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
  try {
    const uint32_t builder = opts ? opts->builder : (uint32_t)SWR_BUILD_HOST;
    if (builder != SWR_BUILD_HOST && builder != SWR_BUILD_DEVICE)
      return set_error(SWR_ERR_INVALID, "swr: unknown builder");
    const bool on_device = builder == SWR_BUILD_DEVICE;
    swr::PackedScene pk;
    int rc = swr::pack_scene(d, opts, pk, !on_device);
    if (rc) return rc;
    std::unique_ptr<swr_scene> s(new swr_scene());
    SWR_CUDA(cudaGetDevice(&s->device));
    SWR_CUDA(cudaDeviceGetAttribute(&s->num_sms, cudaDevAttrMultiProcessorCount, s->device));
    struct Guard {
      swr_scene* p;
      ~Guard() {
        if (p) swr_scene_destroy(p);
      }
    } guard{s.get()};
    if (on_device) {
      if ((rc = swr::device_pack(s.get(), d, opts, pk))) return rc;
    } else {
      if ((rc = swr::upload(&s->d_nodes, pk.nodes))) return rc;
      if ((rc = swr::upload(&s->d_tris, pk.tris))) return rc;
      if ((rc = swr::upload(&s->d_shade, pk.shade))) return rc;
      if ((rc = swr::upload(&s->d_tri_boxes, pk.tri_boxes))) return rc;
      if ((rc = swr::upload(&s->d_albedo, pk.albedo))) return rc;
      if ((rc = swr::upload(&s->d_slot_of, pk.slot_of))) return rc;
    }
    if ((rc = swr::upload(&s->d_obj_boxes, pk.obj_boxes))) return rc;
    if ((rc = swr::upload(&s->d_mats, pk.mats))) return rc;
    if ((rc = swr::upload(&s->d_lights, pk.lights))) return rc;
    if ((rc = swr::upload(&s->d_light_tris, pk.light_tris))) return rc;
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
    ds.lights = (const uint4*)s->d_lights;
    ds.light_tris = (const float4*)s->d_light_tris;
    ds.num_lights = (uint32_t)(pk.lights.size() / 4);
    ds.num_nodes = pk.num_nodes;
    ds.num_slots = (uint32_t)pk.slot_to_id.size();
    ds.num_objects = d->num_objects;
    ds.num_tris = d->num_triangles;
    s->depth = pk.depth;
    s->node_bytes = (uint64_t)pk.num_nodes * 80;
    s->tri_bytes = (uint64_t)ds.num_slots * 48;
    s->slot_to_id = std::move(pk.slot_to_id);
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
  swr::free_instance(s);
  for (void* p : {s->d_nodes, s->d_tris, s->d_shade, s->d_tri_boxes, s->d_obj_boxes, s->d_mats,
                  s->d_albedo, s->d_slot_of, s->d_scratch, s->d_lights, s->d_light_tris, s->rt_buf})
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

int swr_scene_set_albedo(swr_scene* s, const float* albedo, void* stream_) {
  if (!s || !albedo) return set_error(SWR_ERR_INVALID, "swr: null argument");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  void* tmp;
  const float* dev;
  const uint32_t n = s->dev.num_tris;
  int rc = swr::device_input(albedo, (size_t)n * 3 * sizeof(float), stream, &tmp, &dev);
  if (rc) return rc;
  swr::k_set_albedo<<<(n + 255) / 256, 256, 0, stream>>>(s->dev.slot_of, dev, (float*)s->d_albedo, n);
  SWR_CUDA(cudaGetLastError());
  if (tmp) SWR_CUDA(cudaFreeAsync(tmp, stream));
  return SWR_OK;
}

int swr_scene_set_emission(swr_scene* s, const float* emission, void* stream_) {
  if (!s || !emission) return set_error(SWR_ERR_INVALID, "swr: null argument");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  void* tmp;
  const float* dev;
  const uint32_t n = s->dev.num_objects;
  int rc = swr::device_input(emission, (size_t)n * 3 * sizeof(float), stream, &tmp, &dev);
  if (rc) return rc;
  swr::k_set_emission<<<(n + 255) / 256, 256, 0, stream>>>((float4*)s->d_mats, dev, n);
  SWR_CUDA(cudaGetLastError());
  if (tmp) SWR_CUDA(cudaFreeAsync(tmp, stream));
  return SWR_OK;
}

int swr_trace_closest(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n, swr_hit* out,
                      void* stream) {
  return swr::trace_impl(s, ray_o, ray_d, n, out, nullptr, stream);
}

int swr_rt_trace_closest(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n,
                         swr_hit* out, void* stream) {
  return swr::trace_impl(s, ray_o, ray_d, n, out, nullptr, stream, swrx::kRuleRayQuery);
}

int swr_trace_closest_stats(swr_scene* s, const float* ray_o, const float* ray_d, uint64_t n,
                            swr_hit* out, uint32_t* counts, void* stream) {
  if (!counts) return set_error(SWR_ERR_INVALID, "swr: null counts");
  return swr::trace_impl(s, ray_o, ray_d, n, out, counts, stream);
}

}  // extern "C"
