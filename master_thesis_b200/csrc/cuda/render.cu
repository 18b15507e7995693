// Wavefront path tracer (C ABI: swr_render).
//
// Work decomposition: a global sample index g = pixel * spp + sample over the image (processed
// in pixel chunks). Per chunk:
//   k_camera   one thread per pixel: primary ray through the pixel centre and the reference's
//              back-face skipping prefix (path_tracer.cpp:50-57). This prefix uses no random
//              numbers, so it is the same for every sample of the pixel and is traced once per
//              pixel; its first scattering hit is stored in a per-pixel record.
//   loop until no path is live and every sample has been injected:
//     k_shade  shades the traced queue and injects new samples (taking their first hit from the
//              pixel record) up to the queue capacity; continuing paths are appended to the other
//              queue with one atomic per warp (ballot + popc compaction); finished samples write
//              their radiance to a per-sample slot.
//     k_trace  persistent closest-hit traversal over the new queue.
//   k_resolve  sums each pixel's sample slots in sample order and scales, as renderPixel does.
// Queue counters and the injection window live in a small device control block that the
// kernels advance themselves, so the host only launches kernels and polls completion.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "shading.cuh"
#include "swr_internal.cuh"

namespace swr {
namespace {

using swrx::f3;
using swrx::mk;

constexpr uint32_t kDeadSlot = 0xFFFFFFFFu;
constexpr int kTraceBlock = 128;
constexpr uint64_t kChunkSamples = 1ull << 27;
// chunks of at least this many samples, on scenes of at least kTwoWaveTriangles triangles, run as
// kSubWaves concurrent sub-wavefronts (SWR_RENDER_ONE_WAVEFRONT). Measured on B200: 28.02 vs 28.49
// ms for the 2.4 M-triangle terrain image; 1-2 % slower on the 36-triangle Cornell box, whose
// traversal launches have no long tail to fill.
constexpr uint64_t kTwoWaveSamples = 1ull << 20;
constexpr uint32_t kTwoWaveTriangles = 1u << 16;
constexpr int kSubWaves = 2;

struct Ctrl {
  unsigned int count[2];
  unsigned int cursor[2];
  unsigned int inj_n[2];
  unsigned int first_n;  // rays of the first non-empty bounce-traversal launch of the chunk
  unsigned int pixel0;   // image pixel of the chunk's first pixel (read by the shading kernel)
  unsigned long long inj_base[2];
  unsigned long long injected;
  unsigned long long total;
  unsigned long long rays;
  unsigned long long bounce_rays;
  unsigned long long nodes;
  unsigned long long tris;
  unsigned long long rounds;      // shade/trace rounds run by the device-side loop
  unsigned long long max_rounds;  // its bound (every path ends within depth rounds of injection)
  unsigned int status;            // 1: the device-side loop hit max_rounds without draining
  unsigned int cam_cursor;        // next pixel of the chunk for the camera kernel
};

struct Queue {
  float4* o;  // o.xyz | pixel (chunk-local)
  float4* d;  // d.xyz | sample
  float4* c;  // throughput | (i << 8) | v
  float4* l;  // physical: gathered radiance
  uint2* hit;  // slot | t
};

struct Frame {
  float vi[16], pi[16];
  float org[3];
  uint32_t W, H, spp, depth, mode, rr_depth;
  float rr_q;
  uint64_t seed;
  uint32_t pixel0;   // first pixel of the chunk
  uint32_t npix;     // pixels in the chunk
  uint32_t out0;     // pixel whose result goes to the start of the output image (pixel ranges)
  uint32_t sample0;  // image sample index of the call's first sample (sample ranges)
  uint32_t spp_scale;  // samples per pixel of the whole image: the resolve's and adjoint's 1/spp
  uint32_t capacity;
  uint32_t refill;   // idle lanes that trigger a refill in the bounce traversal
  uint32_t batch;    // adjoint: lanes with a finished trace that shade together
  float4* cam;       // [npix*2] per-pixel first hit: (o, t) (d, slot | i << 27)
  float4* contrib;   // [npix*spp] per-sample radiance + flag
};

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

// Camera prefix of every pixel of the chunk (PathTracer::renderPixel's ray and the first bounces
// of traceSinglePath up to the first front-facing hit, path_tracer.cpp:18-27,42-60): the same for
// every sample of the pixel, so it is traced once per pixel. Persistent with per-lane refill, as
// the bounce traversal: a lane keeps its pixel's resumable traversal and, after a back-facing hit,
// restarts it 0.01 further along the ray; when at least F.refill lanes of the warp are idle they
// take that many new pixels from the chunk's pixel cursor with one atomic.
__global__ void __launch_bounds__(kTraceBlock) k_camera(DevScene sc, Frame F, Ctrl* __restrict__ ctrl) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const unsigned refill = F.refill ? F.refill : 8u;
  const f3 org = mk(F.org[0], F.org[1], F.org[2]);
  swrx::Traversal tr;
  bool active = false, exhausted = false;
  uint32_t k = 0, i = 0;
  f3 d = mk(0.0f, 0.0f, 0.0f);
  unsigned traced = 0;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= refill) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&ctrl->cam_cursor, (unsigned)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= F.npix) exhausted = true;
      if (!active) {
        const unsigned j = base + __popc(idle & lt);
        if (j < F.npix) {
          k = j;
          i = 0;
          const uint32_t pix = F.pixel0 + k;
          d = swrx::primary_dir(F.vi, F.pi, pix % F.W, pix / F.W, F.W, F.H);
          tr.init(org, d, stack + threadIdx.x, kTraceBlock);
          ++traced;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tr.template step<false>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, nullptr)) {
      // depth slot i traced: a miss ends the prefix, a back face uses up the slot
      float4 rec0 = make_float4(0, 0, 0, 0), rec1 = make_float4(0, 0, 0, __uint_as_float(kDeadSlot));
      bool done = true;
      if (tr.hit.slot != 0xFFFFFFFFu) {
        const f3 o = tr.o;
        const f3 p = swrx::hit_point(o, d, tr.hit.t);
        const f3 n = swrx::shading_normal(sc.tris, sc.shade, tr.hit.slot, p);
        if (swrx::vdot(n, d) > 0.0f) {
          if (i + 1 < F.depth) {
            tr.init(swrx::vadd(p, swrx::vscale(0.01f, d)), d, stack + threadIdx.x, kTraceBlock);
            ++i;
            ++traced;
            done = false;
          }
        } else {
          rec0 = make_float4(o.x, o.y, o.z, tr.hit.t);
          rec1 = make_float4(d.x, d.y, d.z, __uint_as_float(tr.hit.slot | (i << 27)));
        }
      }
      if (done) {
        F.cam[2 * (size_t)k] = rec0;
        F.cam[2 * (size_t)k + 1] = rec1;
        active = false;
      }
    }
  }
  // count the traced camera-prefix rays: warp sum, one atomic per warp
  for (int off = 16; off > 0; off >>= 1) traced += __shfl_down_sync(0xffffffffu, traced, off);
  if (lane == 0 && traced) atomicAdd(&ctrl->rays, (unsigned long long)traced);
}

// persistent grid of the camera kernel for a chunk of np pixels
static unsigned camera_grid(const swr_scene* s, uint32_t np) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_camera, kTraceBlock, 0) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const uint64_t need = ((uint64_t)np + kTraceBlock - 1) / kTraceBlock;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)s->num_sms * std::max(per_sm, 1)));
}

// One entry of a shading round: a continuing path (its ray and the hit the traversal found) or an
// injected camera sample (its pixel's camera-prefix record).
struct ShadeEntry {
  swrx::PathState st;
  uint32_t pixel, sample, slot;
  float t;
};

__device__ __forceinline__ ShadeEntry load_entry(const Frame& F, const Queue& in, uint32_t i, uint32_t n_in,
                                                 unsigned long long inj_base) {
  ShadeEntry e;
  e.slot = kDeadSlot;
  e.t = 0.0f;
  if (i < n_in) {
    const float4 qo = __ldcs(in.o + i), qd = __ldcs(in.d + i), qc = __ldcs(in.c + i);
    const uint2 h = __ldcs(in.hit + i);
    e.pixel = __float_as_uint(qo.w);
    e.sample = __float_as_uint(qd.w);
    const uint32_t meta = __float_as_uint(qc.w);
    e.st.o = mk(qo.x, qo.y, qo.z);
    e.st.d = mk(qd.x, qd.y, qd.z);
    e.st.c = mk(qc.x, qc.y, qc.z);
    e.st.i = (meta >> 8) & 0xFFu;
    e.st.v = meta & 0xFFu;
    if (F.mode == 1) {
      const float4 ql = __ldcs(in.l + i);
      e.st.L = mk(ql.x, ql.y, ql.z);
    } else {
      e.st.L = mk(0, 0, 0);
    }
    e.slot = h.x;
    e.t = __uint_as_float(h.y);
  } else {
    const unsigned long long g = inj_base + (i - n_in);
    e.pixel = (uint32_t)(g / F.spp);
    e.sample = (uint32_t)(g % F.spp);
    const float4 r0 = F.cam[2 * (size_t)e.pixel], r1 = F.cam[2 * (size_t)e.pixel + 1];
    const uint32_t bits = __float_as_uint(r1.w);
    e.st.c = mk(1.0f, 1.0f, 1.0f);
    e.st.L = mk(0.0f, 0.0f, 0.0f);
    e.st.v = 0;
    e.st.o = mk(r0.x, r0.y, r0.z);
    e.st.d = mk(r1.x, r1.y, r1.z);
    e.st.i = bits >> 27;
    if (bits != kDeadSlot) {
      e.slot = bits & 0x07FFFFFFu;
      e.t = r0.w;
    }
  }
  return e;
}

// Shading round: entries [0, n_in) are the traced paths of the previous round, [n_in, n_in +
// n_inj) new camera samples. An entry without a hit (a ray that left the scene, a camera sample
// of a background pixel) ends dark at once. The grid is persistent: each warp walks chunks of 32
// entries, lists the entries with a hit in its own shared-memory list and shades them 32 at a
// time, so that the long shading code (Philox, double-precision trigonometry and normalisation)
// runs on full warps although most bounce rays miss, and no warp waits at a block barrier or
// leaves its block's slot idle. Results do not depend on which lane shades which entry.
template <int kBlock>
__global__ void __launch_bounds__(kBlock)
    k_shade(DevScene sc, Frame F, Ctrl* __restrict__ ctrl, Queue in, Queue out, int parity) {
  __shared__ uint32_t pending[kBlock / 32][64];
  const uint32_t n_in = ctrl->count[parity];
  const uint32_t n_inj = ctrl->inj_n[parity];
  const unsigned long long inj_base = ctrl->inj_base[parity];
  const uint32_t pixel0 = ctrl->pixel0;
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->cursor[parity ^ 1] = 0u;
  const uint64_t total = (uint64_t)n_in + n_inj;
  const uint32_t lane = lane_id();
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t* list = pending[threadIdx.x >> 5];
  const uint64_t stride = (uint64_t)gridDim.x * kBlock;
  uint32_t npend = 0;  // entries in the warp's list (the same in every lane)
  // the hit word of entry i (the traced slot, or the camera record's slot bits), kDeadSlot for none
  auto hit_word = [&](uint64_t i) -> uint32_t {
    if (i < n_in) return in.hit[i].x;
    if (i < total) return __float_as_uint(F.cam[2 * (size_t)((inj_base + (i - n_in)) / F.spp) + 1].w);
    return kDeadSlot;
  };
  uint64_t base = (uint64_t)blockIdx.x * kBlock + (threadIdx.x & ~31u);
  uint32_t word = hit_word(base + lane);
  for (;; base += stride) {
    const bool more = base < total;
    if (more) {
      // entries without a hit: their dark end; the rest: listed
      const uint64_t i = base + lane;
      bool has_hit = false;
      if (i < n_in) {
        if (word != kDeadSlot) {
          has_hit = true;
        } else {
          const uint32_t pixel = __float_as_uint(__ldcs(&in.o[i].w));
          const uint32_t sample = __float_as_uint(__ldcs(&in.d[i].w));
          float4 r = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          if (F.mode == 1) {
            const float4 ql = __ldcs(in.l + i);
            r = make_float4(ql.x, ql.y, ql.z, 1.0f);
          }
          __stcs(F.contrib + (size_t)pixel * F.spp + sample, r);
        }
      } else if (i < total) {
        if (word != kDeadSlot) {
          has_hit = true;
        } else {
          const unsigned long long g = inj_base + (i - n_in);
          const float4 r = (F.mode == 1) ? make_float4(0.0f, 0.0f, 0.0f, 1.0f) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          __stcs(F.contrib + (size_t)(g / F.spp) * F.spp + (uint32_t)(g % F.spp), r);
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, has_hit);
      if (has_hit) list[npend + __popc(m & lt)] = (uint32_t)i;
      npend += (uint32_t)__popc(m);
      __syncwarp();
      // the next chunk's hit words are fetched now, so that their loads overlap the shading below
      word = hit_word(base + stride + lane);
    }
    // a full warp of listed entries (or, after the last chunk, what is left) is shaded
    while (npend >= 32u || (!more && npend > 0u)) {
      const uint32_t cnt = npend < 32u ? npend : 32u;
      npend -= cnt;
      bool live = false;
      ShadeEntry e;
      if (lane < cnt) {
        e = load_entry(F, in, list[npend + lane], n_in, inj_base);
        swrx::ShadeParams P;
        P.seed = F.seed;
        P.pixel = pixel0 + e.pixel;
        P.sample = F.sample0 + e.sample;
        P.depth = F.depth;
        P.mode = F.mode;
        P.rr_depth = F.rr_depth;
        P.rr_q = F.rr_q;
        const uint32_t outcome = swrx::shade_vertex(sc.tris, sc.shade, sc.mats, sc.albedo, e.slot, e.t, P, e.st);
        if (outcome == swrx::kContinue) {
          live = true;
        } else {
          float4 r;
          if (F.mode == 0)
            r = (outcome == swrx::kEndLight) ? make_float4(e.st.c.x, e.st.c.y, e.st.c.z, 1.0f)
                                             : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          else
            r = make_float4(e.st.L.x, e.st.L.y, e.st.L.z, 1.0f);
          __stcs(F.contrib + (size_t)e.pixel * F.spp + e.sample, r);
        }
      }
      __syncwarp();  // the list slots just read may be refilled by the next chunk
      // warp-aggregated append of the live paths
      const unsigned mask = __ballot_sync(0xffffffffu, live);
      if (mask != 0u) {
        unsigned obase = 0;
        const unsigned leader = __ffs(mask) - 1;
        if (lane == leader) obase = atomicAdd(&ctrl->count[parity ^ 1], (unsigned)__popc(mask));
        obase = __shfl_sync(0xffffffffu, obase, leader);
        if (live) {
          const unsigned j = obase + __popc(mask & lt);
          __stcs(out.o + j, make_float4(e.st.o.x, e.st.o.y, e.st.o.z, __uint_as_float(e.pixel)));
          __stcs(out.d + j, make_float4(e.st.d.x, e.st.d.y, e.st.d.z, __uint_as_float(e.sample)));
          __stcs(out.c + j, make_float4(e.st.c.x, e.st.c.y, e.st.c.z, __uint_as_float((e.st.i << 8) | e.st.v)));
          if (F.mode == 1) __stcs(out.l + j, make_float4(e.st.L.x, e.st.L.y, e.st.L.z, 0.0f));
        }
      }
    }
    if (!more) break;
  }
}

// persistent grid of the shading kernel for a queue of cap entries
static unsigned shade_grid_for(const swr_scene* s, uint32_t cap, int block) {
  int per_sm = 0;
  cudaError_t e = block == 128   ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_shade<128>, 128, 0)
                  : block == 512 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_shade<512>, 512, 0)
                                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_shade<256>, 256, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const uint64_t need = ((uint64_t)cap + block - 1) / block;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)s->num_sms * std::max(per_sm, 1)));
}

template <bool kStats>
__global__ void __launch_bounds__(kTraceBlock)
    k_trace(DevScene sc, Frame F, Ctrl* __restrict__ ctrl, Queue q, int parity) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  // parity p: trace queue p^1, prepare the injection window of the next shade (parity p^1)
  const int qp = parity ^ 1;
  const unsigned n = ctrl->count[qp];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long rem = ctrl->total - ctrl->injected;
    const unsigned long long room = (unsigned long long)F.capacity - n;
    const unsigned long long m = rem < room ? rem : room;
    ctrl->inj_base[qp] = ctrl->injected;
    ctrl->inj_n[qp] = (unsigned)m;
    ctrl->injected += m;
    ctrl->count[parity] = 0u;
    ctrl->rays += n;
    ctrl->bounce_rays += n;
    if (ctrl->first_n == 0u) ctrl->first_n = n;
  }
  swrx::TraceStats st{0, 0};
  for (;;) {
    unsigned base = 0;
    if (lane_id() == 0) base = atomicAdd(&ctrl->cursor[qp], 32u);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    const unsigned i = base + lane_id();
    if (i < n) {
      const float4 o = q.o[i], d = q.d[i];
      swrx::Hit h;
      swrx::trace_closest<kStats>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, mk(o.x, o.y, o.z),
                                  mk(d.x, d.y, d.z), stack + threadIdx.x, kTraceBlock, h, &st);
      q.hit[i] = make_uint2(h.slot, __float_as_uint(h.t));
    }
  }
  if (kStats) {
    unsigned long long nv = st.nodes, tv = st.tris;
    for (int off = 16; off > 0; off >>= 1) {
      nv += __shfl_down_sync(0xffffffffu, nv, off);
      tv += __shfl_down_sync(0xffffffffu, tv, off);
    }
    if (lane_id() == 0) {
      atomicAdd(&ctrl->nodes, nv);
      atomicAdd(&ctrl->tris, tv);
    }
  }
}

// Persistent traversal with per-lane refill: each lane keeps its own ray's traversal state;
// when at least F.refill lanes of the warp have finished, the warp takes that many new rays from
// the queue with one atomic and the idle lanes start them. This keeps lanes busy while the
// slowest ray of a batch is still walking the tree.
// kMinBlocks > 0 caps the register budget so that many blocks fit on one SM.
template <bool kStats, int kMinBlocks, bool kPostpone>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks)
    k_trace_dyn(DevScene sc, Frame F, Ctrl* __restrict__ ctrl, Queue q, int parity) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const int qp = parity ^ 1;
  const unsigned n = ctrl->count[qp];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long rem = ctrl->total - ctrl->injected;
    const unsigned long long room = (unsigned long long)F.capacity - n;
    const unsigned long long m = rem < room ? rem : room;
    ctrl->inj_base[qp] = ctrl->injected;
    ctrl->inj_n[qp] = (unsigned)m;
    ctrl->injected += m;
    ctrl->count[parity] = 0u;
    ctrl->rays += n;
    ctrl->bounce_rays += n;
    if (ctrl->first_n == 0u) ctrl->first_n = n;
  }
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  swrx::TraceStats st{0, 0};
  swrx::Traversal tr;
  bool active = false, exhausted = false;
  unsigned ray = 0;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= F.refill) {
      unsigned base = 0;
      if (lane == 0) base = atomicAdd(&ctrl->cursor[qp], (unsigned)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) exhausted = true;
      if (!active) {
        const unsigned j = base + __popc(idle & lt);
        if (j < n) {
          const float4 o = __ldcs(q.o + j), d = __ldcs(q.d + j);
          tr.init(mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), stack + threadIdx.x, kTraceBlock);
          ray = j;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tr.template step<kStats, kPostpone>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, &st)) {
      __stcs(q.hit + ray, make_uint2(tr.hit.slot, __float_as_uint(tr.hit.t)));
      active = false;
    }
  }
  if (kStats) {
    unsigned long long nv = st.nodes, tv = st.tris;
    for (int off = 16; off > 0; off >>= 1) {
      nv += __shfl_down_sync(0xffffffffu, nv, off);
      tv += __shfl_down_sync(0xffffffffu, tv, off);
    }
    if (lane == 0) {
      atomicAdd(&ctrl->nodes, nv);
      atomicAdd(&ctrl->tris, tv);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Path-replay adjoint of the physical-mode image.
//
// Each lane carries one camera sample at a time: it re-creates the sample's path from its Philox
// counters (the same hits, directions and throughputs as the primal render), keeping for each
// scattering vertex the triangle slot, the throughput c_j before the vertex and the factor
// gq_j the vertex applied besides the albedo (2 cos / q for a diffuse bounce, 1 / q otherwise).
// The backward sweep is swrx::AdjointTape. Nothing of the primal pass is stored: the path is
// replayed, which is the checkpointing scheme. Lanes that finish a sample take a new one (refill
// as in the bounce traversal), and the traversal itself is the resumable Traversal.
using swrx::kAdjMaxDepth;

__global__ void __launch_bounds__(kTraceBlock)
    k_adjoint(DevScene sc, Frame F, Ctrl* __restrict__ ctrl, const float* __restrict__ dl,
              float* __restrict__ g_alb, float* __restrict__ g_em) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const unsigned long long total = ctrl->total;
  swrx::Traversal tr;
  swrx::PathState st;
  uint32_t pixel = 0, sample = 0;
  swrx::AdjointTape tape;
  tape.reset();
  bool active = false, tracing = false, exhausted = false;
  uint32_t pend_slot = 0;
  float pend_t = 0.0f;
  const float inv_spp = 1.0f / (float)F.spp_scale;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= F.refill) {
      unsigned long long base = 0;
      // inj_base[0] serves as the sample cursor of the adjoint launch
      if (lane == 0) base = atomicAdd(&ctrl->inj_base[0], (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) exhausted = true;
      if (!active) {
        const unsigned long long g = base + __popc(idle & lt);
        if (g < total) {
          pixel = (uint32_t)(g / F.spp);
          sample = (uint32_t)(g % F.spp);
          const float4 r0 = F.cam[2 * (size_t)pixel], r1 = F.cam[2 * (size_t)pixel + 1];
          const uint32_t bits = __float_as_uint(r1.w);
          if (bits != kDeadSlot) {
            st.o = mk(r0.x, r0.y, r0.z);
            st.d = mk(r1.x, r1.y, r1.z);
            st.c = mk(1.0f, 1.0f, 1.0f);
            st.L = mk(0.0f, 0.0f, 0.0f);
            st.i = bits >> 27;
            st.v = 0;
            pend_slot = bits & 0x07FFFFFFu;
            pend_t = r0.w;
            tape.reset();
            tracing = false;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tracing && tr.step<false, false>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, nullptr)) {
      tracing = false;
      if (tr.hit.slot == 0xFFFFFFFFu) {  // the path left the scene: no emitter, no gradient
        active = false;
      } else {
        pend_slot = tr.hit.slot;
        pend_t = tr.hit.t;
      }
    }
    // lanes with a pending hit wait until F.batch of them (or every active lane) shade together
    const unsigned waiting = __ballot_sync(0xffffffffu, active && !tracing);
    const unsigned inflight = __ballot_sync(0xffffffffu, active && tracing);
    if (waiting == 0u || ((unsigned)__popc(waiting) < F.batch && inflight != 0u)) continue;
    if (!active || tracing) continue;
    // shade the pending hit
    swrx::ShadeParams P;
    P.seed = F.seed;
    P.pixel = F.pixel0 + pixel;
    P.sample = F.sample0 + sample;
    P.depth = F.depth;
    P.mode = 1;
    P.rr_depth = F.rr_depth;
    P.rr_q = F.rr_q;
    const f3 c_before = st.c;
    swrx::AdjVertex av;
    const uint32_t outcome =
        swrx::shade_physical_adj(sc.tris, sc.shade, sc.mats, sc.albedo, pend_slot, pend_t, P, st, av);
    // a vertex after which the path goes on is kept for the sweep; a path that ends without an
    // emitter (depth reached, Russian roulette, escape) carries no radiance and no gradient
    if (outcome == swrx::kContinue) {
      tape.push(pend_slot, c_before, av);
      tr.init(st.o, st.d, stack + threadIdx.x, kTraceBlock);
      tracing = true;
      continue;
    }
    if (av.emit_front) {
      const float* dlp = dl + (size_t)(F.pixel0 + pixel) * 3;
      tape.sweep(sc.tris, sc.mats, sc.albedo, av.obj, c_before,
                 mk(dlp[0] * inv_spp, dlp[1] * inv_spp, dlp[2] * inv_spp), g_alb, g_em);
    }
    active = false;
  }
}

// ---------------------------------------------------------------------------------------------
// Bidirectional path tracer (BidirectionalPathTracer, bidirectional_path_tracer.cpp:20-168).
//
// Two persistent kernels per chunk of samples, each lane carrying one sample at a time:
//   k_bdpt_paths    the reference's first two stages: the vision path (starting from the
//                   per-pixel camera record, which already holds the back-face-skipping prefix and
//                   the first front hit) and a light subpath from a sampled point on a light
//                   source; every recorded vertex (point, normal, throughput) goes to a per-sample
//                   slot table in device memory.
//   k_bdpt_connect  the connections of every vision vertex with every light vertex
//                   (vi + li <= maxDepth) through occlusion queries (Scene::isOccluded,
//                   scene.cpp:58-83), summed in the reference's order.
// Splitting the stages keeps each kernel's lanes on the same code (path tracing, or occlusion
// queries) and the vertex tables out of registers and local memory. Every trace is the resumable
// Traversal; lanes whose trace finished wait until B.batch of them can run their stage code
// together. Random numbers: the sample's k-th draw of the reference (one per scattering vertex,
// four for the light point) is Philox vertex k of the sample. The vision slots of the skipped
// prefix hold the reference's zero-initialised hit points: their connections add exactly zero,
// so their occlusion queries are not run.
constexpr int kBdptMax = 16;
// measured on the Cornell BDPT image (256x256x16, 5/5/5): batch 1 / 8 / 16 / 20 / 24 ->
// 5.84 / 4.62 / 4.23 / 3.95 / 3.95 ms at refill 4 (identical images)
constexpr uint32_t kBdptBatch = 20;
constexpr uint32_t kConnectBatch = 16;
constexpr uint64_t kBdptTableBytes = 2048ull << 20;

struct BdptArgs {
  uint32_t vj, lj, md;
  uint32_t batch;     // lanes of a warp whose trace finished that advance their samples together
  uint32_t cbatch;    // the same for the connection queries
  uint32_t nsamp;     // samples of the chunk (pixels x spp)
  float4* vtx;        // [3 * (vj + max(lj, 1)) * nsamp]: connection point (the vertex moved 0.01
                      // along its normal), normal (vision vertices only) and throughput of vertex
                      // slot k of sample q at (3k + field) * nsamp + q; vision vertex i is slot i,
                      // light vertex i slot vj + i
  uint4* head;        // [nsamp] first vision slot, vision end, light count, 1 = already resolved
};

enum BdptPhase : uint32_t { kVision = 0, kVisionDone = 1, kLight = 2 };

// A connection runs from vision point + 0.01 * normal to light point + 0.01 * normal
// (bidirectional_path_tracer.cpp:56-57); those points are stored, rounded as there. Only the
// vision vertices' normals are read again (the cosine of a connection).
__device__ __forceinline__ void bd_put(const BdptArgs& B, uint32_t slot, uint32_t q, f3 p, f3 n, f3 c,
                                       bool vision) {
  const f3 e = swrx::vadd(p, swrx::vscale(0.01f, n));
  B.vtx[(size_t)(3 * slot + 0) * B.nsamp + q] = make_float4(e.x, e.y, e.z, 0.0f);
  if (vision) B.vtx[(size_t)(3 * slot + 1) * B.nsamp + q] = make_float4(n.x, n.y, n.z, 0.0f);
  B.vtx[(size_t)(3 * slot + 2) * B.nsamp + q] = make_float4(c.x, c.y, c.z, 0.0f);
}
__device__ __forceinline__ f3 bd_get(const BdptArgs& B, uint32_t slot, uint32_t field, uint32_t q) {
  const float4 v = __ldg(B.vtx + (size_t)(3 * slot + field) * B.nsamp + q);
  return mk(v.x, v.y, v.z);
}

template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks)
    k_bdpt_paths(DevScene sc, Frame F, Ctrl* __restrict__ ctrl, BdptArgs B) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const unsigned long long total = ctrl->total;
  swrx::Traversal tr;
  uint32_t pixel = 0, sample = 0, phase = kVision, i = 0, draws = 0, vfirst = 0, dv = 0, dl = 0;
  bool active = false, tracing = false, exhausted = false, vlight = false;
  f3 o = mk(0, 0, 0), d = mk(0, 0, 0), c = mk(1, 1, 1);
  uint32_t hslot = 0;
  float ht = 0.0f;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= F.refill) {
      unsigned long long base = 0;
      // inj_base[0] serves as the sample cursor of this launch
      if (lane == 0) base = atomicAdd(&ctrl->inj_base[0], (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) exhausted = true;
      if (!active) {
        const unsigned long long g = base + __popc(idle & lt);
        if (g < total) {
          pixel = (uint32_t)(g / F.spp);
          sample = (uint32_t)(g % F.spp);
          const float4 r0 = F.cam[2 * (size_t)pixel], r1 = F.cam[2 * (size_t)pixel + 1];
          const uint32_t bits = __float_as_uint(r1.w);
          if (bits == kDeadSlot) {  // no front hit within visionJumpCount: the sample adds nothing
            F.contrib[(size_t)pixel * F.spp + sample] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
            B.head[(size_t)pixel * F.spp + sample] = make_uint4(0u, 0u, 0u, 1u);
          } else {
            o = mk(r0.x, r0.y, r0.z);
            d = mk(r1.x, r1.y, r1.z);
            i = bits >> 27;
            vfirst = i;
            hslot = bits & 0x07FFFFFFu;
            ht = r0.w;
            draws = 0;
            dv = dl = 0;
            vlight = false;
            c = mk(1.0f, 1.0f, 1.0f);
            phase = kVision;
            tracing = false;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tracing && tr.step<false, false>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, nullptr)) {
      tracing = false;
      hslot = tr.hit.slot;
      ht = tr.hit.t;
    }
    // Lanes whose trace is finished wait until B.batch of them (or every active lane) can run
    // their stage code together, instead of running it for one or two lanes at a time.
    const unsigned waiting = __ballot_sync(0xffffffffu, active && !tracing);
    const unsigned inflight = __ballot_sync(0xffffffffu, active && tracing);
    if (waiting == 0u || ((unsigned)__popc(waiting) < B.batch && inflight != 0u)) continue;
    if (!active || tracing) continue;
    const uint32_t gpix = F.pixel0 + pixel;
    const uint32_t q = pixel * F.spp + sample;
    // advance the sample until it needs a trace or is finished
    while (active && !tracing) {
      if (phase == kVision || phase == kLight) {
        const bool vision = phase == kVision;
        if (hslot == 0xFFFFFFFFu) {
          if (vision) {
            phase = kVisionDone;
          } else {  // the light subpath left the scene: its vertices so far go to the connections
            B.head[q] = make_uint4(vfirst, dv, dl, 0u);
            active = false;
          }
          continue;
        }
        const f3 p = swrx::hit_point(o, d, ht);
        const f3 n = swrx::shading_normal(sc.tris, sc.shade, hslot, p);
        const uint32_t obj = __float_as_uint(__ldg(sc.tris + 3 * (size_t)hslot + 2).w);
        const swrx::Material m = swrx::load_material(sc.mats, obj);
        if (vision) dv = i + 1;
        else dl = i + 1;
        const swrx::Uniforms U = swrx::vertex_uniforms(F.seed, gpix, sample, draws++, 0);
        const float r = U.u[0];
        const f3 prev = d;
        f3 nd = d;
        if (r <= m.m0.w) nd = swrx::hemisphere_dir(n, U.u[1], U.u[2]);
        else if (r <= m.m1.x) nd = swrx::reflect_ref(d, n);
        else if (r <= m.m1.y) nd = swrx::custom_refract_ref(d, n, m.m1.z);
        o = swrx::vadd(p, swrx::vscale(0.01f, nd));
        d = nd;
        if (r <= m.m0.w) {
          const float cs = swrx::vdot(n, vision ? nd : prev);
          c = swrx::vmul(c, mk(__fmul_rn(m.m0.x, cs), __fmul_rn(m.m0.y, cs), __fmul_rn(m.m0.z, cs)));
        }
        bd_put(B, (vision ? 0u : B.vj) + i, q, p, n, c, vision);
        const bool light_hit = __float_as_uint(m.m1.w) != 0u && swrx::vdot(n, prev) <= 0.0f;
        ++i;
        if (light_hit || i >= (vision ? B.vj : B.lj)) {
          if (vision) {
            vlight = light_hit;
            phase = kVisionDone;
          } else {
            B.head[q] = make_uint4(vfirst, dv, dl, 0u);
            active = false;
          }
          continue;
        }
        tr.init(o, d, stack + threadIdx.x, kTraceBlock);
        tracing = true;
      } else if (phase == kVisionDone) {
        if (vlight) {  // c is the throughput recorded at the last vision vertex
          F.contrib[(size_t)pixel * F.spp + sample] = make_float4(c.x, c.y, c.z, 1.0f);
          B.head[q] = make_uint4(0u, 0u, 0u, 1u);
          active = false;
          continue;
        }
        // getRandomLightSourcePoint (bidirectional_path_tracer.cpp:140-168)
        swrx::Uniforms U = swrx::vertex_uniforms(F.seed, gpix, sample, draws++, 0);
        uint32_t light = __float2uint_rz(__fmul_rn(U.u[0], (float)sc.num_lights));
        light = min(light, sc.num_lights - 1u);
        U = swrx::vertex_uniforms(F.seed, gpix, sample, draws++, 0);
        const float sr1 = __fsqrt_rn(U.u[0]);
        U = swrx::vertex_uniforms(F.seed, gpix, sample, draws++, 0);
        const float r2 = U.u[0];
        U = swrx::vertex_uniforms(F.seed, gpix, sample, draws++, 0);
        const uint4 L = sc.lights[light];
        uint32_t ti = __float2uint_rz(__fmul_rn(U.u[0], (float)L.y));
        ti = min(ti, L.y - 1u);
        const float b0 = __fsub_rn(1.0f, sr1), b1 = __fmul_rn(sr1, __fsub_rn(1.0f, r2)), b2 = __fmul_rn(sr1, r2);
        const float4* lq = sc.light_tris + 5 * (size_t)(L.x + ti);
        const float4 q0 = __ldg(lq), q1 = __ldg(lq + 1), q2 = __ldg(lq + 2), q3 = __ldg(lq + 3), q4 = __ldg(lq + 4);
        const f3 v0 = mk(q0.x, q0.y, q0.z), v1 = mk(q0.w, q1.x, q1.y), v2 = mk(q1.z, q1.w, q2.x);
        const f3 n0 = mk(q2.y, q2.z, q2.w), n1 = mk(q3.x, q3.y, q3.z), n2 = mk(q3.w, q4.x, q4.y);
        const f3 lp = swrx::vadd(swrx::vadd(swrx::vscale(b0, v0), swrx::vscale(b1, v1)), swrx::vscale(b2, v2));
        f3 ln = swrx::vadd(mk(0.0f, 0.0f, 0.0f), swrx::vscale(b0, n0));
        ln = swrx::vadd(ln, swrx::vscale(b1, n1));
        ln = swrx::vadd(ln, swrx::vscale(b2, n2));
        ln = swrx::vnormalize(ln);
        const float4 lc = __ldg(sc.mats + 3 * (size_t)L.z);
        bd_put(B, B.vj, q, lp, ln, mk(lc.x, lc.y, lc.z), false);
        o = lp;
        d = swrx::hemisphere_dir(ln, U.u[1], U.u[2]);
        c = mk(1.0f, 1.0f, 1.0f);
        i = 1;
        if (B.lj > 1) {
          phase = kLight;
          tr.init(o, d, stack + threadIdx.x, kTraceBlock);
          tracing = true;
        } else {
          B.head[q] = make_uint4(vfirst, dv, dl, 0u);
          active = false;
        }
      }
    }
  }
}


// Connections of one sample (bidirectional_path_tracer.cpp:51-70): for vi from the first vision
// slot, for li from 0, every pair with vi + li <= maxDepth is joined by an occlusion query between
// the two points lifted by 0.01 along their normals; an unoccluded pair adds
// (vision throughput * light throughput) * cos at the vision vertex. The sum, in that order, is
// divided by maxDepth.
template <int kMinBlocks>
__global__ void __launch_bounds__(kTraceBlock, kMinBlocks)
    k_bdpt_connect(DevScene sc, Frame F, Ctrl* __restrict__ ctrl, BdptArgs B) {
  __shared__ uint2 stack[swrx::kStackShared * kTraceBlock];
  const unsigned lane = lane_id();
  const unsigned lt = (1u << lane) - 1u;
  const unsigned long long total = B.nsamp;
  swrx::Traversal tr;
  uint32_t q = 0, vi = 0, li = 0, dv = 0, dl = 0;
  bool active = false, tracing = false, exhausted = false, pending = false;
  f3 acc = mk(0.0f, 0.0f, 0.0f), dn = mk(0.0f, 0.0f, 0.0f);
  const float inv_md = 1.0f / (float)B.md;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= F.refill) {
      unsigned long long base = 0;
      // inj_base[1] serves as the sample cursor of the connection launch
      if (lane == 0) base = atomicAdd(&ctrl->inj_base[1], (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) exhausted = true;
      if (!active) {
        const unsigned long long g = base + __popc(idle & lt);
        if (g < total) {
          const uint4 h = B.head[g];
          if (h.w == 0u) {
            q = (uint32_t)g;
            vi = h.x;
            dv = h.y;
            dl = h.z;
            li = 0;
            acc = mk(0.0f, 0.0f, 0.0f);
            pending = false;
            tracing = false;
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tracing && tr.step<false, false>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, nullptr))
      tracing = false;
    const unsigned waiting = __ballot_sync(0xffffffffu, active && !tracing);
    const unsigned inflight = __ballot_sync(0xffffffffu, active && tracing);
    if (waiting == 0u || ((unsigned)__popc(waiting) < B.cbatch && inflight != 0u)) continue;
    if (!active || tracing) continue;
    if (pending) {  // the query of pair (vi, li) is answered
      if (tr.hit.slot == 0xFFFFFFFFu) {  // not occluded
        const float cs = swrx::vdot(dn, bd_get(B, vi, 1, q));
        const f3 vc = bd_get(B, vi, 2, q), lc = bd_get(B, B.vj + li, 2, q);
        acc = swrx::vadd(acc, mk(__fmul_rn(__fmul_rn(vc.x, lc.x), cs), __fmul_rn(__fmul_rn(vc.y, lc.y), cs),
                                 __fmul_rn(__fmul_rn(vc.z, lc.z), cs)));
      }
      ++li;
      pending = false;
    }
    for (;;) {
      if (vi >= dv) {
        const uint32_t pixel = q / F.spp, sample = q % F.spp;
        const f3 r = swrx::vscale(inv_md, acc);
        F.contrib[(size_t)pixel * F.spp + sample] = make_float4(r.x, r.y, r.z, 1.0f);
        active = false;
        break;
      }
      if (li >= dl) {
        ++vi;
        li = 0;
        continue;
      }
      if (vi + li > B.md) {
        ++li;
        continue;
      }
      const f3 a = bd_get(B, vi, 0, q), b = bd_get(B, B.vj + li, 0, q);
      const f3 dd = swrx::vsub(b, a);
      const float dist2 = swrx::vdot(dd, dd);
      dn = swrx::vnormalize(dd);
      tr.init_occlusion(a, dn, dist2, stack + threadIdx.x, kTraceBlock);
      tracing = true;
      pending = true;
      break;
    }
  }
}

// Per-pixel sum of the sample slots in sample order (path_tracer.cpp:28-37), 256 pixels per block.
// A warp takes 32 consecutive pixels and loads their slots 8 samples at a time with coalesced loads
// (each load instruction reads whole 128-byte lines) into a shared-memory tile padded to 9 slots
// per pixel (conflict-free reads); each lane then adds its pixel's slots in sample order, as the
// reference's renderPixel does.
__global__ void __launch_bounds__(256) k_resolve(Frame F, float* __restrict__ img) {
  __shared__ float4 tile[8][32 * 9];
  const uint32_t w = threadIdx.x >> 5, lane = lane_id();
  const uint64_t p0 = ((uint64_t)blockIdx.x * 8 + w) * 32;  // the warp's first pixel
  if (p0 >= F.npix) return;
  const uint32_t np = (uint32_t)((F.npix - p0) < 32 ? (F.npix - p0) : 32);
  const uint32_t spp = F.spp;
  float4* t = tile[w];
  float r = 0.0f, g = 0.0f, b = 0.0f;
  for (uint32_t s0 = 0; s0 < spp; s0 += 8) {
    const uint32_t ns = (spp - s0) < 8 ? (spp - s0) : 8;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const uint32_t e = lane + 32u * j, pe = e >> 3, se = e & 7u;
      if (pe < np && se < ns) t[pe * 9 + se] = __ldcs(F.contrib + (size_t)(p0 + pe) * spp + s0 + se);
    }
    __syncwarp();
    if (lane < np) {
      for (uint32_t k = 0; k < ns; ++k) {
        const float4 v = t[lane * 9 + k];
        if (v.w != 0.0f) {
          r = __fadd_rn(r, v.x);
          g = __fadd_rn(g, v.y);
          b = __fadd_rn(b, v.z);
        }
      }
    }
    __syncwarp();
  }
  if (lane >= np) return;
  // reference: finalColor *= 2.0f * M_PI * (1.0f / float(spp)), scalar and products in double
  const float inv = __fdiv_rn(1.0f, (float)F.spp_scale);
  const double s = (F.mode == 0) ? __dmul_rn(6.283185307179586, (double)inv) : (double)inv;
  float* o = img + (size_t)(F.pixel0 - F.out0 + p0 + lane) * 3;
  o[0] = __double2float_rn(__dmul_rn((double)r, s));
  o[1] = __double2float_rn(__dmul_rn((double)g, s));
  o[2] = __double2float_rn(__dmul_rn((double)b, s));
}

struct Workspace {
  size_t qbytes = 0, cam_px = 0, contrib_n = 0, stage_n = 0, bd_vtx_n = 0, bd_head_n = 0;
  void* qbuf = nullptr;
  void* cam = nullptr;
  void* contrib = nullptr;
  void* stage = nullptr;  // device image for callers that pass a host output buffer
  void* bd_vtx = nullptr;   // bidirectional tracer: per-sample vertex tables
  void* bd_head = nullptr;  // bidirectional tracer: per-sample vertex counts
  Ctrl* ctrl = nullptr;       // [4] control blocks (one per concurrent sub-wavefront)
  Ctrl* host_ctrl = nullptr;  // [4] pinned copies
  // round-loop graphs per sub-wavefront, the last kGraphsKept launch shapes each (a render that
  // alternates, e.g. counting and plain renders, reuses them instead of rebuilding)
  struct GraphEntry {
    std::vector<char> key;
    cudaGraphExec_t exec = nullptr;
    uint64_t used = 0;
  };
  std::vector<GraphEntry> graphs[4];
  uint64_t graph_clock = 0;
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};  // streams of sub-wavefronts 1..3
  cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
};

// End of one iteration of the device-side round loop (eight shade/trace rounds, after which the
// next shade reads parity 0): continue while paths are queued or samples wait for injection; stop
// with status 1 once the proven bound on rounds is exceeded (never reached unless the wavefront
// logic is broken), so the loop always ends.
__global__ void k_round_check(Ctrl* __restrict__ ctrl, cudaGraphConditionalHandle loop) {
  Ctrl& c = *ctrl;
  c.rounds += 8;
  const bool drained = c.count[0] == 0u && c.inj_n[0] == 0u && c.injected == c.total;
  unsigned go = drained ? 0u : 1u;
  if (!drained && c.rounds > c.max_rounds) {
    c.status = 1u;
    go = 0u;
  }
  cudaGraphSetConditional(loop, go);
}

constexpr size_t kGraphsKept = 4;

// The round-loop graph for `key` from the cache (built when missing, evicting the least recently
// used beyond kGraphsKept): a WHILE node whose body is `rounds` (eight shade/trace rounds, enqueued
// on the given stream) followed by k_round_check. The key holds every argument baked into it.
template <class Enqueue>
int round_loop_graph(Workspace* ws, int slot, const std::vector<char>& key, Ctrl* ctrl, Enqueue rounds,
                     cudaGraphExec_t* out) {
  auto& cache = ws->graphs[slot];
  for (auto& e : cache)
    if (e.key == key) {
      e.used = ++ws->graph_clock;
      *out = e.exec;
      return SWR_OK;
    }
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t g = nullptr;
  cudaStream_t cs = nullptr;
  auto build = [&]() -> int {
    SWR_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle loop;
    SWR_CUDA(cudaGraphConditionalHandleCreate(&loop, g, 1u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {cudaGraphNodeTypeConditional};
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    SWR_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    SWR_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    SWR_CUDA(cudaStreamBeginCaptureToGraph(cs, cp.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
    rounds(cs);
    k_round_check<<<1, 1, 0, cs>>>(ctrl, loop);
    cudaGraph_t captured = nullptr;
    SWR_CUDA(cudaStreamEndCapture(cs, &captured));
    SWR_CUDA(cudaGraphInstantiate(&exec, g, 0));
    return SWR_OK;
  };
  const int rc = build();
  if (cs) cudaStreamDestroy(cs);
  if (g) cudaGraphDestroy(g);
  if (rc) {
    if (exec) cudaGraphExecDestroy(exec);
    return rc;
  }
  if (cache.size() >= kGraphsKept) {
    size_t lru = 0;
    for (size_t i = 1; i < cache.size(); ++i)
      if (cache[i].used < cache[lru].used) lru = i;
    cudaGraphExecDestroy(cache[lru].exec);
    cache.erase(cache.begin() + (long)lru);
  }
  Workspace::GraphEntry e;
  e.key = key;
  e.exec = exec;
  e.used = ++ws->graph_clock;
  cache.push_back(std::move(e));
  *out = exec;
  return SWR_OK;
}

int ensure(void** p, size_t& have, size_t want, size_t elem) {
  if (have >= want && *p) return SWR_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  have = 0;
  cudaError_t e = cudaMalloc(p, std::max<size_t>(want * elem, 256));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(SWR_ERR_ALLOC, std::string("CUDA: workspace allocation of ") +
                                        std::to_string(want * elem) + " bytes failed");
  }
  have = want;
  return SWR_OK;
}

}  // namespace

// Per-scene workspace storage (kept behind an opaque pointer in the scene).
struct RenderWorkspace : Workspace {};

static RenderWorkspace* workspace_of(swr_scene* s);

namespace {

// Records CUDA events around kernel launches of one kind and sums their durations.
struct KernelTimer {
  std::vector<cudaEvent_t> ev;
  std::vector<int> kind;
  size_t used = 0;
  double ms[4] = {0, 0, 0, 0};
  bool on = false;
  cudaError_t begin(cudaStream_t st, int k) {
    if (!on) return cudaSuccess;
    if (used + 2 > ev.size()) {
      for (int i = 0; i < 2; ++i) {
        cudaEvent_t e;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) return r;
        ev.push_back(e);
      }
      kind.push_back(0);
    }
    kind[used / 2] = k;
    return cudaEventRecord(ev[used], st);
  }
  cudaError_t end(cudaStream_t st) {
    if (!on) return cudaSuccess;
    cudaError_t r = cudaEventRecord(ev[used + 1], st);
    used += 2;
    return r;
  }
  // call after a stream synchronize: folds the recorded pairs into the totals
  cudaError_t collect() {
    for (size_t i = 0; i < used; i += 2) {
      float t = 0.0f;
      cudaError_t r = cudaEventElapsedTime(&t, ev[i], ev[i + 1]);
      if (r != cudaSuccess) return r;
      ms[kind[i / 2]] += t;
    }
    used = 0;
    return cudaSuccess;
  }
  ~KernelTimer() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

enum { kTimeTrace = 0, kTimeShade = 1, kTimeCamera = 2, kTimeResolve = 3 };

}  // namespace

// The part of the image a call renders (swr_render_opts: sample_begin, spp_total, pixel_begin,
// pixel_count). allow_pixels: the entry point supports pixel ranges; allow_samples: sample ranges.
struct ImagePart {
  uint32_t sample0 = 0, spp_scale = 0;
  uint64_t pixel0 = 0, npix = 0;
};

static int image_part(const swr_render_opts* o, bool allow_samples, bool allow_pixels, ImagePart* part,
                      const char* who) {
  const uint64_t total = (uint64_t)o->width * o->height;
  part->sample0 = o->sample_begin;
  part->spp_scale = o->spp_total ? o->spp_total : o->spp;
  part->pixel0 = o->pixel_begin;
  part->npix = o->pixel_count ? o->pixel_count : (o->pixel_begin < total ? total - o->pixel_begin : 0);
  const bool samples = o->sample_begin != 0 || o->spp_total != 0;
  const bool pixels = o->pixel_begin != 0 || o->pixel_count != 0;
  if (samples && !allow_samples) return set_error(SWR_ERR_UNSUPPORTED, std::string("swr: ") + who +
                                                  " renders whole images (sample_begin and spp_total must be 0)");
  if (pixels && !allow_pixels) return set_error(SWR_ERR_UNSUPPORTED, std::string("swr: ") + who +
                                                " renders whole images (pixel_begin and pixel_count must be 0)");
  if ((uint64_t)o->sample_begin + o->spp > part->spp_scale)
    return set_error(SWR_ERR_INVALID, "swr: sample_begin + spp exceeds spp_total");
  if (o->pixel_begin >= total || part->npix == 0 || (uint64_t)o->pixel_begin + part->npix > total)
    return set_error(SWR_ERR_INVALID, "swr: pixel range outside the image");
  return SWR_OK;
}

int render_impl(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, float* rgb_out,
                float* samples_out, void* stream_, swr_render_profile* prof) {
  if (!s || !cam || !o || !rgb_out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (o->width == 0 || o->height == 0 || o->spp == 0)
    return set_error(SWR_ERR_INVALID, "swr: zero image size or samples");
  if (o->max_depth == 0 || o->max_depth > 31)
    return set_error(SWR_ERR_INVALID, "swr: max_depth must be 1..31");
  if (o->mode > 1) return set_error(SWR_ERR_INVALID, "swr: unknown mode");
  if (o->mode == 1 && o->rr_depth != 0 && !(o->rr_survive > 0.0f && o->rr_survive <= 1.0f))
    return set_error(SWR_ERR_INVALID, "swr: rr_survive must be in (0, 1]");
  if ((uint64_t)o->width * o->height >= (1ull << 32))
    return set_error(SWR_ERR_INVALID, "swr: image too large");
  if ((o->flags & SWR_RENDER_SAMPLES_OUT) && !samples_out)
    return set_error(SWR_ERR_INVALID, "swr: SWR_RENDER_SAMPLES_OUT without a samples buffer");
  int block = o->block_size ? (int)o->block_size : 256;
  if (block != 128 && block != 256 && block != 512)
    return set_error(SWR_ERR_INVALID, "swr: block_size must be 128, 256 or 512");
  ImagePart part;
  int rc = image_part(o, true, true, &part, "swr_render");
  if (rc) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  RenderWorkspace* ws = workspace_of(s);
  if (!ws) return set_error(SWR_ERR_ALLOC, "swr: workspace");
  swr_render_profile P;
  std::memset(&P, 0, sizeof(P));
  KernelTimer timer;
  timer.on = (o->flags & SWR_RENDER_PROFILE) != 0;
  const bool count = (o->flags & SWR_RENDER_COUNT) != 0;

  // the pixels this call renders (the whole image unless a pixel range is given)
  const uint64_t npix_total = part.npix;
  const uint64_t px_per_chunk = std::max<uint64_t>(1, std::min<uint64_t>(npix_total, kChunkSamples / o->spp));
  uint32_t cap = o->wave_size ? o->wave_size : (1u << 23);
  cap = (uint32_t)std::min<uint64_t>(cap, px_per_chunk * o->spp);
  cap = std::max<uint32_t>(32, (cap + 255u) & ~255u);
  const size_t qbytes = (size_t)cap * (4 * sizeof(float4) + sizeof(uint2)) * 2;
  if ((rc = ensure(&ws->qbuf, ws->qbytes, qbytes, 1))) return rc;
  if ((rc = ensure(&ws->cam, ws->cam_px, px_per_chunk, 2 * sizeof(float4)))) return rc;
  if ((rc = ensure(&ws->contrib, ws->contrib_n, px_per_chunk * o->spp, sizeof(float4)))) return rc;
  if (!ws->ctrl) {
    SWR_CUDA(cudaMalloc(&ws->ctrl, 4 * sizeof(Ctrl)));
    SWR_CUDA(cudaMallocHost(&ws->host_ctrl, 4 * sizeof(Ctrl)));
  }

  Queue Q[2];
  {
    char* b = (char*)ws->qbuf;
    for (int p = 0; p < 2; ++p) {
      Q[p].o = (float4*)b; b += (size_t)cap * sizeof(float4);
      Q[p].d = (float4*)b; b += (size_t)cap * sizeof(float4);
      Q[p].c = (float4*)b; b += (size_t)cap * sizeof(float4);
      Q[p].l = (float4*)b; b += (size_t)cap * sizeof(float4);
      Q[p].hit = (uint2*)b; b += (size_t)cap * sizeof(uint2);
    }
  }

  // output staging for host pointers
  float* img = rgb_out;
  float* img_dev = nullptr;
  const bool host_img = is_host_pointer(rgb_out);
  if (host_img) {
    if ((rc = ensure(&ws->stage, ws->stage_n, npix_total * 3, sizeof(float)))) return rc;
    img_dev = (float*)ws->stage;
    img = img_dev;
  }
  const bool want_samples = (o->flags & SWR_RENDER_SAMPLES_OUT) != 0;
  const bool host_samples = want_samples && is_host_pointer(samples_out);

  Frame F;
  std::memset(&F, 0, sizeof(F));  // every byte, padding included, is part of the round-loop graph's key
  std::memcpy(F.vi, cam->view_inv, sizeof(F.vi));
  std::memcpy(F.pi, cam->proj_inv, sizeof(F.pi));
  std::memcpy(F.org, cam->origin, sizeof(F.org));
  F.W = o->width;
  F.H = o->height;
  F.spp = o->spp;
  F.sample0 = part.sample0;
  F.spp_scale = part.spp_scale;
  F.out0 = (uint32_t)part.pixel0;
  F.depth = o->max_depth;
  F.mode = o->mode;
  F.rr_depth = (o->mode == 1) ? o->rr_depth : 0;
  F.rr_q = (o->mode == 1 && o->rr_depth) ? o->rr_survive : 1.0f;
  F.seed = o->seed;
  F.capacity = cap;
  F.cam = (float4*)ws->cam;
  F.contrib = (float4*)ws->contrib;

  using TraceKernel = void (*)(DevScene, Frame, Ctrl*, Queue, int);
  const bool static_fetch = (o->flags & SWR_RENDER_STATIC_FETCH) != 0;
  TraceKernel trace_kernel;
  const bool postpone = (o->flags & SWR_RENDER_POSTPONE) != 0;
  switch (o->trace_blocks) {
    case 0:  // default: 9 blocks per SM (56 registers, no spills; measured faster than the
             // compiler's own choice of 64 registers and 8 blocks)
    case 9:
      trace_kernel = postpone ? (count ? k_trace_dyn<true, 9, true> : k_trace_dyn<false, 9, true>)
                              : (count ? k_trace_dyn<true, 9, false> : k_trace_dyn<false, 9, false>);
      break;
    case 10:
      trace_kernel = postpone ? (count ? k_trace_dyn<true, 10, true> : k_trace_dyn<false, 10, true>)
                              : (count ? k_trace_dyn<true, 10, false> : k_trace_dyn<false, 10, false>);
      break;
    default: return set_error(SWR_ERR_INVALID, "swr: trace_blocks must be 0, 9 or 10");
  }
  if (static_fetch) trace_kernel = count ? k_trace<true> : k_trace<false>;
  if (o->refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  F.refill = o->refill ? o->refill : 8;
  int trace_per_sm = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&trace_per_sm, trace_kernel, kTraceBlock, 0));
  const unsigned trace_grid = (unsigned)(s->num_sms * std::max(trace_per_sm, 1));
  const unsigned shade_grid = shade_grid_for(s, cap, block);

  // Sub-wavefront h of a chunk: pixels [off, off + n) of it, queues of capw paths carved from the
  // h-th half of the queue buffer (the whole buffer when the chunk runs as one wavefront), control
  // block h; everything it launches goes to stream st. Graph path only.
  auto launch_wave = [&](int h, cudaStream_t st, uint64_t p0, uint64_t off, uint32_t n, uint32_t capw) -> int {
    Queue Qh[2];
    {
      char* b = (char*)ws->qbuf + (size_t)h * ((size_t)capw * (4 * sizeof(float4) + sizeof(uint2)) * 2);
      for (int q = 0; q < 2; ++q) {
        Qh[q].o = (float4*)b; b += (size_t)capw * sizeof(float4);
        Qh[q].d = (float4*)b; b += (size_t)capw * sizeof(float4);
        Qh[q].c = (float4*)b; b += (size_t)capw * sizeof(float4);
        Qh[q].l = (float4*)b; b += (size_t)capw * sizeof(float4);
        Qh[q].hit = (uint2*)b; b += (size_t)capw * sizeof(uint2);
      }
    }
    Ctrl* ctrl = ws->ctrl + h;
    Frame Fh = F;
    Fh.pixel0 = (uint32_t)(p0 + off);
    Fh.npix = n;
    Fh.cam = F.cam + 2 * off;
    Fh.contrib = F.contrib + off * o->spp;
    Fh.capacity = capw;
    const uint64_t total = (uint64_t)n * o->spp;
    // every path ends within max_depth rounds of its injection and each round injects up to the
    // queue capacity, so this many rounds always suffice; more means a logic error
    Ctrl init;
    std::memset(&init, 0, sizeof(init));
    init.total = total;
    init.inj_n[0] = (unsigned)std::min<uint64_t>(capw, total);
    init.injected = init.inj_n[0];
    init.pixel0 = Fh.pixel0;
    init.max_rounds = (total / capw + 2) * (uint64_t)(o->max_depth + 2) + 64;
    ws->host_ctrl[h] = init;
    SWR_CUDA(cudaMemcpyAsync(ctrl, ws->host_ctrl + h, sizeof(Ctrl), cudaMemcpyHostToDevice, st));
    P.h2d_bytes += sizeof(Ctrl);
    k_camera<<<camera_grid(s, n), kTraceBlock, 0, st>>>(s->dev, Fh, ctrl);
    SWR_CUDA(cudaGetLastError());
    // the shading and traversal kernels read the first pixel from the control block, so their
    // arguments (and a graph made of them) are the same for every chunk
    Frame FR = Fh;
    FR.pixel0 = 0;
    FR.npix = 0;
    const unsigned sgrid = shade_grid_for(s, capw, block);
    std::vector<char> key(sizeof(DevScene) + sizeof(Frame) + sizeof(Qh) + 5 * sizeof(void*));
    {
      char* kp = key.data();
      std::memset(kp, 0, key.size());
      std::memcpy(kp, &s->dev, sizeof(DevScene));
      std::memcpy(kp + sizeof(DevScene), &FR, sizeof(Frame));
      std::memcpy(kp + sizeof(DevScene) + sizeof(Frame), Qh, sizeof(Qh));
      const void* extra[5] = {ctrl, (void*)trace_kernel, (void*)(uintptr_t)block, (void*)(uintptr_t)trace_grid,
                              (void*)(uintptr_t)sgrid};
      std::memcpy(kp + sizeof(DevScene) + sizeof(Frame) + sizeof(Qh), extra, sizeof(extra));
    }
    cudaGraphExec_t graph = nullptr;
    int grc = round_loop_graph(ws, h, key, ctrl, [&](cudaStream_t cs) {
      for (int c = 0; c < 8; ++c) {
        const int q = c & 1;
        switch (block) {
          case 128: k_shade<128><<<sgrid, 128, 0, cs>>>(s->dev, FR, ctrl, Qh[q], Qh[q ^ 1], q); break;
          case 512: k_shade<512><<<sgrid, 512, 0, cs>>>(s->dev, FR, ctrl, Qh[q], Qh[q ^ 1], q); break;
          default: k_shade<256><<<sgrid, 256, 0, cs>>>(s->dev, FR, ctrl, Qh[q], Qh[q ^ 1], q); break;
        }
        trace_kernel<<<trace_grid, kTraceBlock, 0, cs>>>(s->dev, FR, ctrl, Qh[q ^ 1], q);
      }
    }, &graph);
    if (grc) return grc;
    SWR_CUDA(cudaGraphLaunch(graph, st));
    SWR_CUDA(cudaGetLastError());
    k_resolve<<<(n + 255) / 256, 256, 0, st>>>(Fh, img);
    SWR_CUDA(cudaGetLastError());
    if (host_img) {  // this part of a host image goes out while the other sub-wavefronts still run
      const size_t first = (size_t)(Fh.pixel0 - F.out0) * 3;
      SWR_CUDA(cudaMemcpyAsync(rgb_out + first, img_dev + first, (size_t)n * 3 * sizeof(float),
                               cudaMemcpyDeviceToHost, st));
      P.d2h_bytes += (size_t)n * 3 * sizeof(float);
    }
    SWR_CUDA(cudaMemcpyAsync(ws->host_ctrl + h, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    P.d2h_bytes += sizeof(Ctrl);
    return SWR_OK;
  };
  // what a drained sub-wavefront reports
  auto collect = [&](const Ctrl& hc) -> int {
    if (hc.status) return set_error(SWR_ERR_TIMEOUT, "swr: wavefront did not drain");
    P.rays += hc.rays;
    P.bounce_rays += hc.bounce_rays;
    if (P.first_trace_rays == 0) P.first_trace_rays = hc.first_n;
    P.node_visits += hc.nodes;
    P.tri_tests += hc.tris;
    P.iterations += hc.rounds;
    P.launches += 2 + 2 * hc.rounds + hc.rounds / 8;  // camera, resolve, rounds, checks
    P.trace_launches += hc.rounds;
    return SWR_OK;
  };

  for (uint64_t q0 = 0; q0 < npix_total; q0 += px_per_chunk) {
    const uint32_t np = (uint32_t)std::min<uint64_t>(px_per_chunk, npix_total - q0);
    const uint64_t p0 = part.pixel0 + q0;  // image pixel of the chunk's first pixel
    F.pixel0 = (uint32_t)p0;
    F.npix = np;
    const uint64_t total = (uint64_t)np * o->spp;
    SWR_CUDA(cudaStreamSynchronize(stream));  // the pinned control blocks may still be in flight
    if (!timer.on && !(o->flags & SWR_RENDER_HOST_LOOP)) {
      // Large chunks of large scenes run as kSubWaves sub-wavefronts (a share of the pixels and of
      // the paths in flight each) on as many streams: when one's traversal launch runs out of rays and its SMs
      // idle while the last rays finish, the others' kernels fill them. Per-pixel results do not
      // depend on it.
      const int nsub = (!(o->flags & SWR_RENDER_ONE_WAVEFRONT) && total >= kTwoWaveSamples &&
                        s->dev.num_tris >= kTwoWaveTriangles && np >= (uint32_t)kSubWaves &&
                        cap >= 256u * kSubWaves) ? kSubWaves : 1;
      if (nsub > 1) {
        if (!ws->fork) {
          SWR_CUDA(cudaEventCreateWithFlags(&ws->fork, cudaEventDisableTiming));
          for (int h = 0; h < 3; ++h) {
            SWR_CUDA(cudaStreamCreateWithFlags(&ws->side[h], cudaStreamNonBlocking));
            SWR_CUDA(cudaEventCreateWithFlags(&ws->join[h], cudaEventDisableTiming));
          }
        }
        const uint32_t capw = (cap / nsub) & ~255u;
        SWR_CUDA(cudaEventRecord(ws->fork, stream));
        for (int h = 0; h < nsub; ++h) {
          const uint64_t a = (uint64_t)np * h / nsub, b = (uint64_t)np * (h + 1) / nsub;
          cudaStream_t st = h ? ws->side[h - 1] : stream;
          if (h) SWR_CUDA(cudaStreamWaitEvent(st, ws->fork, 0));
          if ((rc = launch_wave(h, st, p0, a, (uint32_t)(b - a), capw))) return rc;
          if (h) SWR_CUDA(cudaEventRecord(ws->join[h - 1], st));
        }
        for (int h = 1; h < nsub; ++h) SWR_CUDA(cudaStreamWaitEvent(stream, ws->join[h - 1], 0));
        SWR_CUDA(cudaStreamSynchronize(stream));
        for (int h = 0; h < nsub; ++h)
          if ((rc = collect(ws->host_ctrl[h]))) return rc;
      } else {
        if ((rc = launch_wave(0, stream, p0, 0, np, cap))) return rc;
        SWR_CUDA(cudaStreamSynchronize(stream));
        if ((rc = collect(ws->host_ctrl[0]))) return rc;
      }
    } else {
      // profiled (or SWR_RENDER_HOST_LOOP): one wavefront whose loop the host runs, so that every
      // launch has its CUDA events and a profiler sees each launch
      const uint64_t max_rounds = (total / cap + 2) * (uint64_t)(o->max_depth + 2) + 64;
      Ctrl init;
      std::memset(&init, 0, sizeof(init));
      init.total = total;
      init.inj_n[0] = (unsigned)std::min<uint64_t>(cap, total);
      init.injected = init.inj_n[0];
      init.pixel0 = (uint32_t)p0;
      init.max_rounds = max_rounds;
      *ws->host_ctrl = init;
      SWR_CUDA(cudaMemcpyAsync(ws->ctrl, ws->host_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, stream));
      P.h2d_bytes += sizeof(Ctrl);
      SWR_CUDA(timer.begin(stream, kTimeCamera));
      k_camera<<<camera_grid(s, np), kTraceBlock, 0, stream>>>(s->dev, F, ws->ctrl);
      SWR_CUDA(timer.end(stream));
      SWR_CUDA(cudaGetLastError());
      P.launches++;
      Frame FR = F;
      FR.pixel0 = 0;
      FR.npix = 0;
      uint64_t k = 0;
      for (;;) {
        if (k > max_rounds) return set_error(SWR_ERR_TIMEOUT, "swr: wavefront did not drain");
        const int kChunk = 8;
        for (int c = 0; c < kChunk; ++c, ++k) {
          const int p = (int)(k & 1);
          SWR_CUDA(timer.begin(stream, kTimeShade));
          switch (block) {
            case 128: k_shade<128><<<shade_grid, 128, 0, stream>>>(s->dev, FR, ws->ctrl, Q[p], Q[p ^ 1], p); break;
            case 512: k_shade<512><<<shade_grid, 512, 0, stream>>>(s->dev, FR, ws->ctrl, Q[p], Q[p ^ 1], p); break;
            default: k_shade<256><<<shade_grid, 256, 0, stream>>>(s->dev, FR, ws->ctrl, Q[p], Q[p ^ 1], p); break;
          }
          SWR_CUDA(timer.end(stream));
          SWR_CUDA(timer.begin(stream, kTimeTrace));
          trace_kernel<<<trace_grid, kTraceBlock, 0, stream>>>(s->dev, FR, ws->ctrl, Q[p ^ 1], p);
          SWR_CUDA(timer.end(stream));
          P.launches += 2;
          P.trace_launches++;
        }
        SWR_CUDA(cudaGetLastError());
        SWR_CUDA(cudaMemcpyAsync(ws->host_ctrl, ws->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream));
        P.d2h_bytes += sizeof(Ctrl);
        SWR_CUDA(cudaStreamSynchronize(stream));
        SWR_CUDA(timer.collect());
        const Ctrl& h = *ws->host_ctrl;
        const int np_ = (int)(k & 1);
        if (h.count[np_] == 0 && h.inj_n[np_] == 0 && h.injected == h.total) {
          P.rays += h.rays;
          P.bounce_rays += h.bounce_rays;
          if (P.first_trace_rays == 0) P.first_trace_rays = h.first_n;
          P.node_visits += h.nodes;
          P.tri_tests += h.tris;
          P.iterations += k;
          break;
        }
      }
      SWR_CUDA(timer.begin(stream, kTimeResolve));
      k_resolve<<<(np + 255) / 256, 256, 0, stream>>>(F, img);
      SWR_CUDA(timer.end(stream));
      SWR_CUDA(cudaGetLastError());
      P.launches++;
    }
    if (want_samples) {
      const size_t bytes = (size_t)np * o->spp * sizeof(float4);
      SWR_CUDA(cudaMemcpyAsync(samples_out + (size_t)q0 * o->spp * 4, F.contrib, bytes,
                               host_samples ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, stream));
      if (host_samples) P.d2h_bytes += bytes;
    }
  }
  if (host_img && timer.on) {  // the graph path copied each sub-wavefront's part as it finished
    SWR_CUDA(cudaMemcpyAsync(rgb_out, img_dev, npix_total * 3 * sizeof(float), cudaMemcpyDeviceToHost, stream));
    P.d2h_bytes += npix_total * 3 * sizeof(float);
  }
  if (host_img || host_samples || timer.on) SWR_CUDA(cudaStreamSynchronize(stream));
  if (timer.on) SWR_CUDA(timer.collect());
  P.trace_ms = timer.ms[kTimeTrace];
  P.shade_ms = timer.ms[kTimeShade];
  P.camera_ms = timer.ms[kTimeCamera];
  P.resolve_ms = timer.ms[kTimeResolve];
  if (prof) *prof = P;
  return SWR_OK;
}

static RenderWorkspace* workspace_of(swr_scene* s) {
  if (!s->workspace) s->workspace = new RenderWorkspace();
  return (RenderWorkspace*)s->workspace;
}

void free_workspace(swr_scene* s) {
  RenderWorkspace* ws = (RenderWorkspace*)s->workspace;
  if (!ws) return;
  if (ws->qbuf) cudaFree(ws->qbuf);
  if (ws->cam) cudaFree(ws->cam);
  if (ws->contrib) cudaFree(ws->contrib);
  if (ws->stage) cudaFree(ws->stage);
  if (ws->bd_vtx) cudaFree(ws->bd_vtx);
  if (ws->bd_head) cudaFree(ws->bd_head);
  if (ws->ctrl) cudaFree(ws->ctrl);
  if (ws->host_ctrl) cudaFreeHost(ws->host_ctrl);
  for (auto& cache : ws->graphs)
    for (auto& e : cache) cudaGraphExecDestroy(e.exec);
  for (int h = 0; h < 3; ++h) {
    if (ws->side[h]) cudaStreamDestroy(ws->side[h]);
    if (ws->join[h]) cudaEventDestroy(ws->join[h]);
  }
  if (ws->fork) cudaEventDestroy(ws->fork);
  delete ws;
  s->workspace = nullptr;
}

int render_adjoint_impl(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, const float* dl,
                        float* g_alb, float* g_em, void* stream_, double* ms_out) {
  if (!s || !cam || !o || !dl || !g_alb || !g_em) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (o->mode != SWR_MODE_PHYSICAL)
    return set_error(SWR_ERR_INVALID, "swr: the adjoint is defined for SWR_MODE_PHYSICAL");
  if (o->width == 0 || o->height == 0 || o->spp == 0)
    return set_error(SWR_ERR_INVALID, "swr: zero image size or samples");
  if (o->max_depth == 0 || o->max_depth > (uint32_t)kAdjMaxDepth)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: the adjoint supports max_depth 1..16");
  if (o->rr_depth != 0 && !(o->rr_survive > 0.0f && o->rr_survive <= 1.0f))
    return set_error(SWR_ERR_INVALID, "swr: rr_survive must be in (0, 1]");
  if ((uint64_t)o->width * o->height >= (1ull << 32)) return set_error(SWR_ERR_INVALID, "swr: image too large");
  if (o->refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  if (o->shade_batch > 32) return set_error(SWR_ERR_INVALID, "swr: shade_batch must be 0..32");
  ImagePart part;
  int rc = image_part(o, true, false, &part, "swr_render_adjoint");
  if (rc) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  if (is_host_pointer(dl) || is_host_pointer(g_alb) || is_host_pointer(g_em))
    return set_error(SWR_ERR_INVALID, "swr: the adjoint takes device buffers");
  RenderWorkspace* ws = workspace_of(s);
  const uint64_t npix_total = (uint64_t)o->width * o->height;
  const uint64_t px_per_chunk = std::max<uint64_t>(1, std::min<uint64_t>(npix_total, kChunkSamples / o->spp));
  if ((rc = ensure(&ws->cam, ws->cam_px, px_per_chunk, 2 * sizeof(float4)))) return rc;
  if (!ws->ctrl) {
    SWR_CUDA(cudaMalloc(&ws->ctrl, 4 * sizeof(Ctrl)));
    SWR_CUDA(cudaMallocHost(&ws->host_ctrl, 4 * sizeof(Ctrl)));
  }
  SWR_CUDA(cudaMemsetAsync(g_alb, 0, (size_t)s->dev.num_tris * 3 * sizeof(float), stream));
  SWR_CUDA(cudaMemsetAsync(g_em, 0, (size_t)s->dev.num_objects * 3 * sizeof(float), stream));
  Frame F;
  std::memset(&F, 0, sizeof(F));
  std::memcpy(F.vi, cam->view_inv, sizeof(F.vi));
  std::memcpy(F.pi, cam->proj_inv, sizeof(F.pi));
  std::memcpy(F.org, cam->origin, sizeof(F.org));
  F.W = o->width;
  F.H = o->height;
  F.spp = o->spp;
  F.sample0 = part.sample0;
  F.spp_scale = part.spp_scale;
  F.out0 = 0;
  F.depth = o->max_depth;
  F.mode = 1;
  F.rr_depth = o->rr_depth;
  F.rr_q = o->rr_depth ? o->rr_survive : 1.0f;
  F.seed = o->seed;
  F.refill = o->refill ? o->refill : 8;
  F.batch = o->shade_batch ? o->shade_batch : swrx::kAdjointBatch;
  F.cam = (float4*)ws->cam;
  int per_sm = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_adjoint, kTraceBlock, 0));
  const unsigned grid = (unsigned)(s->num_sms * std::max(per_sm, 1));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms_out) {
    SWR_CUDA(cudaEventCreate(&e0));
    SWR_CUDA(cudaEventCreate(&e1));
    SWR_CUDA(cudaEventRecord(e0, stream));
  }
  for (uint64_t p0 = 0; p0 < npix_total; p0 += px_per_chunk) {
    const uint32_t np = (uint32_t)std::min<uint64_t>(px_per_chunk, npix_total - p0);
    F.pixel0 = (uint32_t)p0;
    F.npix = np;
    Ctrl init;
    std::memset(&init, 0, sizeof(init));
    init.total = (uint64_t)np * o->spp;
    SWR_CUDA(cudaStreamSynchronize(stream));  // the pinned control block may still be in flight
    *ws->host_ctrl = init;
    SWR_CUDA(cudaMemcpyAsync(ws->ctrl, ws->host_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, stream));
    k_camera<<<camera_grid(s, np), kTraceBlock, 0, stream>>>(s->dev, F, ws->ctrl);
    k_adjoint<<<grid, kTraceBlock, 0, stream>>>(s->dev, F, ws->ctrl, dl, g_alb, g_em);
    SWR_CUDA(cudaGetLastError());
  }
  if (ms_out) {
    SWR_CUDA(cudaEventRecord(e1, stream));
    SWR_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    SWR_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *ms_out = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  return SWR_OK;
}

int render_bdpt_impl(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, const swr_bdpt_opts* b,
                     float* rgb_out, float* samples_out, void* stream_) {
  if (!s || !cam || !o || !b || !rgb_out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (o->mode != SWR_MODE_REFERENCE)
    return set_error(SWR_ERR_INVALID, "swr: the bidirectional tracer renders SWR_MODE_REFERENCE");
  if (o->width == 0 || o->height == 0 || o->spp == 0)
    return set_error(SWR_ERR_INVALID, "swr: zero image size or samples");
  if (o->max_depth == 0 || o->max_depth > (uint32_t)kBdptMax || b->light_jumps > (uint32_t)kBdptMax)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: the bidirectional tracer supports 1..16 vision and 0..16 light jumps");
  if (b->max_depth == 0) return set_error(SWR_ERR_INVALID, "swr: bidirectional maxDepth must be positive");
  {
    ImagePart part;
    const int prc = image_part(o, false, false, &part, "swr_render_bdpt");
    if (prc) return prc;
  }
  if ((uint64_t)o->width * o->height >= (1ull << 32)) return set_error(SWR_ERR_INVALID, "swr: image too large");
  if (o->refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  if ((b->shade_batch & 0xFFu) > 32 || ((b->shade_batch >> 8) & 0xFFu) > 32 || (b->shade_batch >> 16))
    return set_error(SWR_ERR_INVALID, "swr: shade_batch fields must be 0..32");
  if (b->blocks_per_sm != 0 && b->blocks_per_sm != 5 && b->blocks_per_sm != 6 && b->blocks_per_sm != 8)
    return set_error(SWR_ERR_INVALID, "swr: blocks_per_sm must be 0, 5, 6 or 8");
  if (s->dev.num_lights == 0)
    return set_error(SWR_ERR_INVALID, "swr: the bidirectional tracer needs a light source in the scene");
  const bool want_samples = (o->flags & SWR_RENDER_SAMPLES_OUT) != 0;
  if (want_samples && !samples_out)
    return set_error(SWR_ERR_INVALID, "swr: SWR_RENDER_SAMPLES_OUT without a samples buffer");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  RenderWorkspace* ws = workspace_of(s);
  if (!ws) return set_error(SWR_ERR_ALLOC, "swr: workspace");
  const uint64_t npix_total = (uint64_t)o->width * o->height;
  // samples per chunk: by default as many as keep the vertex tables (48 B per vertex slot and
  // sample) within 2 GB. Measured on the Cornell BDPT image (1 M samples, 10 slots): chunks of
  // 2^16 / 2^18 / 2^19 / 2^20 samples -> 6.85 / 3.40 / 2.95 / 2.71 ms; tables small enough for L2
  // do not pay for the per-chunk launches and synchronisation.
  const uint64_t slots = (uint64_t)o->max_depth + std::max<uint32_t>(b->light_jumps, 1u);
  const uint64_t chunk = o->wave_size ? (uint64_t)o->wave_size
                                      : std::max<uint64_t>(1u << 14, kBdptTableBytes / (48 * slots));
  const uint64_t px_per_chunk = std::max<uint64_t>(1, std::min<uint64_t>(npix_total, chunk / o->spp));
  int rc;
  if ((rc = ensure(&ws->cam, ws->cam_px, px_per_chunk, 2 * sizeof(float4)))) return rc;
  if ((rc = ensure(&ws->contrib, ws->contrib_n, px_per_chunk * o->spp, sizeof(float4)))) return rc;
  if ((rc = ensure(&ws->bd_vtx, ws->bd_vtx_n, px_per_chunk * o->spp * 3 * slots, sizeof(float4)))) return rc;
  if ((rc = ensure(&ws->bd_head, ws->bd_head_n, px_per_chunk * o->spp, sizeof(uint4)))) return rc;
  if (!ws->ctrl) {
    SWR_CUDA(cudaMalloc(&ws->ctrl, 4 * sizeof(Ctrl)));
    SWR_CUDA(cudaMallocHost(&ws->host_ctrl, 4 * sizeof(Ctrl)));
  }
  float* img = rgb_out;
  const bool host_img = is_host_pointer(rgb_out);
  if (host_img) {
    if ((rc = ensure(&ws->stage, ws->stage_n, npix_total * 3, sizeof(float)))) return rc;
    img = (float*)ws->stage;
  }
  const bool host_samples = want_samples && is_host_pointer(samples_out);
  Frame F;
  std::memset(&F, 0, sizeof(F));
  std::memcpy(F.vi, cam->view_inv, sizeof(F.vi));
  std::memcpy(F.pi, cam->proj_inv, sizeof(F.pi));
  std::memcpy(F.org, cam->origin, sizeof(F.org));
  F.W = o->width;
  F.H = o->height;
  F.spp = o->spp;
  F.sample0 = 0;
  F.spp_scale = o->spp;
  F.out0 = 0;
  F.depth = o->max_depth;
  F.mode = 0;
  F.rr_q = 1.0f;
  F.seed = o->seed;
  F.refill = o->refill ? o->refill : 4;
  F.cam = (float4*)ws->cam;
  F.contrib = (float4*)ws->contrib;
  BdptArgs B;
  B.vj = o->max_depth;
  B.lj = b->light_jumps;
  B.md = b->max_depth;
  B.batch = (b->shade_batch & 0xFFu) ? (b->shade_batch & 0xFFu) : kBdptBatch;
  B.cbatch = ((b->shade_batch >> 8) & 0xFFu) ? ((b->shade_batch >> 8) & 0xFFu) : kConnectBatch;
  B.vtx = (float4*)ws->bd_vtx;
  B.head = (uint4*)ws->bd_head;
  auto kern = k_bdpt_paths<0>;
  auto kconn = k_bdpt_connect<0>;
  if (b->blocks_per_sm == 5) kern = k_bdpt_paths<5>, kconn = k_bdpt_connect<5>;
  else if (b->blocks_per_sm == 6) kern = k_bdpt_paths<6>, kconn = k_bdpt_connect<6>;
  else if (b->blocks_per_sm == 8) kern = k_bdpt_paths<8>, kconn = k_bdpt_connect<8>;
  int per_sm = 0, per_sm_c = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kTraceBlock, 0));
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_c, kconn, kTraceBlock, 0));
  const unsigned grid = (unsigned)(s->num_sms * std::max(per_sm, 1));
  const unsigned grid_c = (unsigned)(s->num_sms * std::max(per_sm_c, 1));
  for (uint64_t p0 = 0; p0 < npix_total; p0 += px_per_chunk) {
    const uint32_t np = (uint32_t)std::min<uint64_t>(px_per_chunk, npix_total - p0);
    F.pixel0 = (uint32_t)p0;
    F.npix = np;
    Ctrl init;
    std::memset(&init, 0, sizeof(init));
    init.total = (uint64_t)np * o->spp;
    SWR_CUDA(cudaStreamSynchronize(stream));  // the pinned control block may still be in flight
    *ws->host_ctrl = init;
    SWR_CUDA(cudaMemcpyAsync(ws->ctrl, ws->host_ctrl, sizeof(Ctrl), cudaMemcpyHostToDevice, stream));
    k_camera<<<camera_grid(s, np), kTraceBlock, 0, stream>>>(s->dev, F, ws->ctrl);
    B.nsamp = np * o->spp;
    kern<<<grid, kTraceBlock, 0, stream>>>(s->dev, F, ws->ctrl, B);
    kconn<<<grid_c, kTraceBlock, 0, stream>>>(s->dev, F, ws->ctrl, B);
    k_resolve<<<(np + 255) / 256, 256, 0, stream>>>(F, img);
    SWR_CUDA(cudaGetLastError());
    if (want_samples)
      SWR_CUDA(cudaMemcpyAsync(samples_out + (size_t)p0 * o->spp * 4, F.contrib, (size_t)np * o->spp * sizeof(float4),
                               host_samples ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, stream));
  }
  if (host_img)
    SWR_CUDA(cudaMemcpyAsync(rgb_out, img, npix_total * 3 * sizeof(float), cudaMemcpyDeviceToHost, stream));
  if (host_img || host_samples) SWR_CUDA(cudaStreamSynchronize(stream));
  return SWR_OK;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free render (swr_render_noalloc).
//
// Some callers cannot let a library allocate device memory while they run: applications that
// hand all device memory to their own pool up front and forbid allocation by plug-ins, and
// latency-sensitive loops that must not pay for cudaMalloc/cudaFree, which can synchronise the
// whole device. For them the wavefront's scratch (path queues, per-pixel camera records,
// per-sample slots and the control block) lives in one file-scope device array of fixed size,
// loaded with the library and held by every device that loads it until the process exits.
// Every call uses the same array: calls that overlap on the GPU (different streams or threads)
// race on it and must be serialised by the caller. Nothing in the array needs to start at zero:
// each chunk overwrites the control block from the host and writes every camera record and
// sample slot it later reads.
constexpr size_t kNoAllocBytes = 64ull << 20;           // 64 MiB of device scratch
constexpr uint32_t kNoAllocCap = 1u << 16;              // paths in flight
constexpr uint64_t kNoAllocChunkSamples = 1ull << 21;   // samples per chunk
constexpr uint64_t kNoAllocChunkPixels = 1ull << 18;    // pixels per chunk
constexpr size_t kNoAllocQueueBytes = (size_t)kNoAllocCap * (4 * sizeof(float4) + sizeof(uint2));
constexpr size_t kNoAllocCamOffset = 256 + 2 * kNoAllocQueueBytes;  // the control block takes the first 256 bytes
static_assert(sizeof(Ctrl) <= 256, "the allocation-free render keeps its control block in 256 bytes");
constexpr size_t kNoAllocContribOffset = kNoAllocCamOffset + kNoAllocChunkPixels * 2 * sizeof(float4);
static_assert(kNoAllocContribOffset + kNoAllocChunkSamples * sizeof(float4) <= kNoAllocBytes,
              "no-allocation scratch layout exceeds its array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch on the current device. In host code the array's name is
// only a stand-in for the symbol, never a device address. The address is looked up on every call
// rather than cached: the lookup allocates nothing once the module is loaded, and a cached address
// would go stale if the host application reset the device (cudaDeviceReset reloads the module,
// possibly elsewhere). The first call on a device may load the module (lazy loading), so that
// call should come before any stream capture.
static int noalloc_scratch(char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
  *out = (char*)p;
  return SWR_OK;
}

int render_noalloc_impl(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, float* rgb_out,
                        float* samples_out, void* stream_) {
  if (!s || !cam || !o || !rgb_out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (o->width == 0 || o->height == 0 || o->spp == 0)
    return set_error(SWR_ERR_INVALID, "swr: zero image size or samples");
  if (o->max_depth == 0 || o->max_depth > 31)
    return set_error(SWR_ERR_INVALID, "swr: max_depth must be 1..31");
  if (o->mode > 1) return set_error(SWR_ERR_INVALID, "swr: unknown mode");
  if (o->mode == 1 && o->rr_depth != 0 && !(o->rr_survive > 0.0f && o->rr_survive <= 1.0f))
    return set_error(SWR_ERR_INVALID, "swr: rr_survive must be in (0, 1]");
  if ((uint64_t)o->width * o->height >= (1ull << 32))
    return set_error(SWR_ERR_INVALID, "swr: image too large");
  if (o->flags & ~SWR_RENDER_SAMPLES_OUT)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: swr_render_noalloc accepts only SWR_RENDER_SAMPLES_OUT");
  {
    ImagePart part;
    const int prc = image_part(o, false, false, &part, "swr_render_noalloc");
    if (prc) return prc;
  }
  const bool want_samples = (o->flags & SWR_RENDER_SAMPLES_OUT) != 0;
  if (want_samples && !samples_out)
    return set_error(SWR_ERR_INVALID, "swr: SWR_RENDER_SAMPLES_OUT without a samples buffer");
  if (o->spp > kNoAllocChunkSamples)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: swr_render_noalloc handles at most 2097152 samples per pixel "
                                          "(its fixed scratch holds 2^21 sample slots)");
  if (o->wave_size > kNoAllocCap)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: swr_render_noalloc keeps at most 65536 paths in flight");
  if (o->refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  if (o->block_size && o->block_size != 256)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: swr_render_noalloc shades with 256-thread blocks");
  if (o->trace_blocks) return set_error(SWR_ERR_UNSUPPORTED, "swr: swr_render_noalloc uses trace_blocks 0");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  if (is_host_pointer(rgb_out) || (want_samples && is_host_pointer(samples_out)))
    return set_error(SWR_ERR_INVALID, "swr: swr_render_noalloc needs device output buffers (staging host "
                                      "memory would need a device allocation)");
  char* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;

  const uint64_t npix_total = (uint64_t)o->width * o->height;
  const uint64_t px_per_chunk =
      std::max<uint64_t>(1, std::min<uint64_t>(std::min<uint64_t>(npix_total, kNoAllocChunkSamples / o->spp),
                                                kNoAllocChunkPixels));
  uint32_t cap = o->wave_size ? o->wave_size : kNoAllocCap;
  cap = (uint32_t)std::min<uint64_t>(cap, px_per_chunk * o->spp);
  cap = std::min<uint32_t>(kNoAllocCap, std::max<uint32_t>(32, (cap + 255u) & ~255u));

  Ctrl* ctrl = (Ctrl*)base;
  Queue Q[2];
  {
    char* b = base + 256;
    for (int p = 0; p < 2; ++p) {
      Q[p].o = (float4*)b; b += (size_t)kNoAllocCap * sizeof(float4);
      Q[p].d = (float4*)b; b += (size_t)kNoAllocCap * sizeof(float4);
      Q[p].c = (float4*)b; b += (size_t)kNoAllocCap * sizeof(float4);
      Q[p].l = (float4*)b; b += (size_t)kNoAllocCap * sizeof(float4);
      Q[p].hit = (uint2*)b; b += (size_t)kNoAllocCap * sizeof(uint2);
    }
  }
  Frame F;
  std::memset(&F, 0, sizeof(F));  // every byte, padding included, is part of the round-loop graph's key
  std::memcpy(F.vi, cam->view_inv, sizeof(F.vi));
  std::memcpy(F.pi, cam->proj_inv, sizeof(F.pi));
  std::memcpy(F.org, cam->origin, sizeof(F.org));
  F.W = o->width;
  F.H = o->height;
  F.spp = o->spp;
  F.sample0 = 0;
  F.spp_scale = o->spp;
  F.out0 = 0;
  F.depth = o->max_depth;
  F.mode = o->mode;
  F.rr_depth = (o->mode == 1) ? o->rr_depth : 0;
  F.rr_q = (o->mode == 1 && o->rr_depth) ? o->rr_survive : 1.0f;
  F.seed = o->seed;
  F.capacity = cap;
  F.refill = o->refill ? o->refill : 8;
  F.cam = (float4*)(base + kNoAllocCamOffset);
  F.contrib = (float4*)(base + kNoAllocContribOffset);

  int trace_per_sm = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&trace_per_sm, k_trace_dyn<false, 0, false>,
                                                         kTraceBlock, 0));
  const unsigned trace_grid = (unsigned)(s->num_sms * std::max(trace_per_sm, 1));
  const unsigned shade_grid = (cap + 255) / 256;
  for (uint64_t p0 = 0; p0 < npix_total; p0 += px_per_chunk) {
    const uint32_t np = (uint32_t)std::min<uint64_t>(px_per_chunk, npix_total - p0);
    F.pixel0 = (uint32_t)p0;
    F.npix = np;
    const uint64_t total = (uint64_t)np * o->spp;
    Ctrl init;
    std::memset(&init, 0, sizeof(init));
    init.total = total;
    init.inj_n[0] = (unsigned)std::min<uint64_t>(cap, total);
    init.injected = init.inj_n[0];
    init.pixel0 = (uint32_t)p0;
    // pageable source: the copy has been taken when the call returns
    SWR_CUDA(cudaMemcpyAsync(ctrl, &init, sizeof(Ctrl), cudaMemcpyHostToDevice, stream));
    k_camera<<<camera_grid(s, np), kTraceBlock, 0, stream>>>(s->dev, F, ctrl);
    SWR_CUDA(cudaGetLastError());
    uint64_t k = 0;
    const uint64_t max_rounds = (total / cap + 2) * (uint64_t)(o->max_depth + 2) + 64;
    for (;;) {
      if (k > max_rounds) return set_error(SWR_ERR_TIMEOUT, "swr: wavefront did not drain");
      for (int c = 0; c < 8; ++c, ++k) {
        const int p = (int)(k & 1);
        k_shade<256><<<shade_grid, 256, 0, stream>>>(s->dev, F, ctrl, Q[p], Q[p ^ 1], p);
        k_trace_dyn<false, 0, false><<<trace_grid, kTraceBlock, 0, stream>>>(s->dev, F, ctrl, Q[p ^ 1], p);
      }
      SWR_CUDA(cudaGetLastError());
      Ctrl h;
      SWR_CUDA(cudaMemcpyAsync(&h, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, stream));
      SWR_CUDA(cudaStreamSynchronize(stream));
      const int np_ = (int)(k & 1);
      if (h.count[np_] == 0 && h.inj_n[np_] == 0 && h.injected == h.total) break;
    }
    k_resolve<<<(np + 255) / 256, 256, 0, stream>>>(F, rgb_out);
    SWR_CUDA(cudaGetLastError());
    if (want_samples)
      SWR_CUDA(cudaMemcpyAsync(samples_out + (size_t)p0 * o->spp * 4, F.contrib, (size_t)np * o->spp * sizeof(float4),
                               cudaMemcpyDeviceToDevice, stream));
  }
  return SWR_OK;
}

}  // namespace swr

extern "C" {

int swr_render(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, float* rgb_out,
               float* samples_out, void* stream) {
  return swr::render_impl(s, cam, o, rgb_out, samples_out, stream, nullptr);
}

int swr_render_profiled(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, float* rgb_out,
                        float* samples_out, void* stream, swr_render_profile* prof) {
  return swr::render_impl(s, cam, o, rgb_out, samples_out, stream, prof);
}

int swr_render_adjoint(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, const float* dl_dimage,
                       float* dl_dalbedo, float* dl_demission, void* stream) {
  return swr::render_adjoint_impl(s, cam, o, dl_dimage, dl_dalbedo, dl_demission, stream, nullptr);
}

int swr_render_bdpt(swr_scene* s, const swr_camera* cam, const swr_render_opts* opts, const swr_bdpt_opts* bdpt,
                    float* rgb_out, float* samples_out, void* stream) {
  return swr::render_bdpt_impl(s, cam, opts, bdpt, rgb_out, samples_out, stream);
}

int swr_render_adjoint_timed(swr_scene* s, const swr_camera* cam, const swr_render_opts* o,
                             const float* dl_dimage, float* dl_dalbedo, float* dl_demission, void* stream,
                             double* device_ms) {
  return swr::render_adjoint_impl(s, cam, o, dl_dimage, dl_dalbedo, dl_demission, stream, device_ms);
}

int swr_render_noalloc(swr_scene* s, const swr_camera* cam, const swr_render_opts* o, float* rgb_out,
                       float* samples_out, void* stream) {
  return swr::render_noalloc_impl(s, cam, o, rgb_out, samples_out, stream);
}

}  // extern "C"
