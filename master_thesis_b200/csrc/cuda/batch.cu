// Batched rendering of many independent scenes in one wavefront (C ABI: swr_batch_create /
// swr_batch_destroy / swr_render_batch).
//
// All jobs share one path queue. A job = (scene, camera, image size, samples, depth, mode, seed,
// output). Global sample indices run over the jobs back to back (prefix sums in the job table);
// injection finds a sample's job by binary search, every path carries its job id, and the
// traversal reads that job's scene. Samples use the same random-number keys as a single-scene
// render of the job (pixel index within the job's image, sample index), so each job's paths are
// exactly those of swr_render for it. Radiance is summed per pixel in 64-bit fixed point with
// integer atomics (scale 2^32): order-independent, hence deterministic, and it needs 24 bytes per
// pixel instead of 16 bytes per sample (a 256-scene batch has ~2e9 samples). The final per-pixel
// scale is the single-scene one. The shade/trace rounds are captured once into a CUDA graph: a
// conditional WHILE node whose body runs eight rounds and then k_bcheck, which ends the loop on
// the device when the queue has drained (or, as a guard against a logic error, after a proven
// bound on the rounds, recording a timeout). The host waits once per batch.
#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "shading.cuh"
#include "swr_internal.cuh"

namespace swr {
namespace {

using swrx::f3;
using swrx::mk;

constexpr uint32_t kDead = 0xFFFFFFFFu;
constexpr int kTB = 128;
constexpr double kFix = 4294967296.0;  // 2^32
// batches of at least this many samples run as kBatchSubWaves concurrent sub-wavefronts
constexpr uint64_t kBatchTwoWaveSamples = 1ull << 20;
constexpr int kBatchSubWaves = 2;

struct BJob {
  float vi[16], pi[16];
  float org[3];
  uint32_t W, H, spp, depth, mode, rr_depth;
  float rr_q;
  uint32_t scene;
  uint64_t seed;
  uint64_t sample_base;  // first global sample index of the job
  uint64_t pixel_base;   // first global pixel index of the job
  float* out;            // [H*W*3] device (primal)
  const float* dl;       // [H*W*3] device dLoss/dImage (adjoint)
  float* g_alb;          // [triangles*3] device (adjoint)
  float* g_em;           // [objects*3] device (adjoint)
};

struct BCtrl {
  unsigned int count[2];
  unsigned int cursor[2];
  unsigned int inj_n[2];
  unsigned int status;  // 1: the device-side round loop hit max_rounds without draining
  unsigned int pad;
  unsigned long long inj_base[2];
  unsigned long long injected;
  unsigned long long total;
  unsigned long long rays;
  unsigned long long rounds;      // shade/trace rounds run by the device-side loop
  unsigned long long max_rounds;  // its bound (every path ends within depth rounds of injection)
  unsigned long long cam_cursor;  // next pixel of the persistent camera-prefix kernel
};

struct BQueue {
  float4* o;  // origin | pixel (within the job)
  float4* d;  // direction | sample
  float4* c;  // throughput | job << 16 | i << 8 | v
  float4* l;  // physical radiance so far
  uint2* hit;
};

struct BArgs {
  const BJob* jobs;
  const DevScene* scenes;
  uint32_t njobs;
  uint64_t npix;  // total pixels
  uint32_t capacity, refill;
  uint32_t batch;               // adjoint: lanes with a finished trace that shade together
  float4* cam;                  // [npix*2]
  unsigned long long* accum;    // [npix*3] fixed point
};

__device__ __forceinline__ unsigned lane() { return threadIdx.x & 31u; }

// index of the job whose [base, next base) range holds v (bases ascending, first is 0)
__device__ __forceinline__ uint32_t find_job(const BJob* jobs, uint32_t n, uint64_t v, bool by_pixel) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    const uint64_t b = by_pixel ? jobs[mid].pixel_base : jobs[mid].sample_base;
    if (b <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Camera prefix of every pixel of every job, persistent as the single-scene k_camera: idle lanes
// take the next pixels from ctrl->cam_cursor (refill), find their job by binary search and trace
// the pixel-centre ray; a back-facing first hit restarts the lane's traversal past it (using up a
// depth slot), so lanes do not wait for the warp's slowest pixel.
__global__ void __launch_bounds__(kTB) k_bcamera(BArgs A, BCtrl* __restrict__ ctrl) {
  __shared__ uint2 stack[swrx::kStackShared * kTB];
  const unsigned ln = lane();
  const unsigned lt = (1u << ln) - 1u;
  const unsigned refill = A.refill ? A.refill : 8u;
  swrx::Traversal tr;
  const DevScene* sc = nullptr;
  bool active = false, exhausted = false;
  uint64_t p = 0;
  uint32_t i = 0, depth = 0;
  f3 d = mk(0.0f, 0.0f, 0.0f);
  unsigned traced = 0;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= refill) {
      unsigned long long base = 0;
      if (ln == 0) base = atomicAdd(&ctrl->cam_cursor, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= A.npix) exhausted = true;
      if (!active) {
        const uint64_t q = base + (unsigned)__popc(idle & lt);
        if (q < A.npix) {
          p = q;
          i = 0;
          const uint32_t j = find_job(A.jobs, A.njobs, p, true);
          const BJob& J = A.jobs[j];
          sc = &A.scenes[J.scene];
          depth = J.depth;
          const uint32_t pix = (uint32_t)(p - J.pixel_base);
          d = swrx::primary_dir(J.vi, J.pi, pix % J.W, pix / J.W, J.W, J.H);
          tr.init(mk(J.org[0], J.org[1], J.org[2]), d, stack + threadIdx.x, kTB);
          ++traced;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tr.step<false>(sc->nodes, sc->tris, sc->tri_boxes, sc->obj_boxes, nullptr)) {
      // depth slot i traced: a miss ends the prefix, a back face uses up the slot
      float4 r0 = make_float4(0, 0, 0, 0), r1 = make_float4(0, 0, 0, __uint_as_float(kDead));
      bool done = true;
      if (tr.hit.slot != 0xFFFFFFFFu) {
        const f3 o = tr.o;
        const f3 hp = swrx::hit_point(o, d, tr.hit.t);
        const f3 n = swrx::shading_normal(sc->tris, sc->shade, tr.hit.slot, hp);
        if (swrx::vdot(n, d) > 0.0f) {
          if (i + 1 < depth) {
            tr.init(swrx::vadd(hp, swrx::vscale(0.01f, d)), d, stack + threadIdx.x, kTB);
            ++i;
            ++traced;
            done = false;
          }
        } else {
          r0 = make_float4(o.x, o.y, o.z, tr.hit.t);
          r1 = make_float4(d.x, d.y, d.z, __uint_as_float(tr.hit.slot | (i << 27)));
        }
      }
      if (done) {
        A.cam[2 * p] = r0;
        A.cam[2 * p + 1] = r1;
        active = false;
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) traced += __shfl_down_sync(0xffffffffu, traced, off);
  if (ln == 0 && traced) atomicAdd(&ctrl->rays, (unsigned long long)traced);
}

// persistent grid of the batch's camera-prefix kernel for np pixels
static unsigned bcamera_grid(int num_sms, uint64_t np) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bcamera, kTB, 0) != cudaSuccess) {
    cudaGetLastError();
    per_sm = 1;
  }
  const uint64_t need = (np + kTB - 1) / kTB;
  return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)num_sms * std::max(per_sm, 1)));
}

__device__ __forceinline__ void accumulate(unsigned long long* acc, float r, float g, float b) {
  atomicAdd(acc + 0, (unsigned long long)__double2ll_rn((double)r * kFix));
  atomicAdd(acc + 1, (unsigned long long)__double2ll_rn((double)g * kFix));
  atomicAdd(acc + 2, (unsigned long long)__double2ll_rn((double)b * kFix));
}

// Shading round of the batch (as the single-scene k_shade): entries without a hit end at once; a
// persistent grid's warps walk chunks of 32 entries, list the rest (entry, job) in their own
// shared-memory lists and shade them 32 at a time.
__global__ void __launch_bounds__(256) k_bshade(BArgs A, BCtrl* __restrict__ ctrl, BQueue in, BQueue out,
                                                int parity) {
  __shared__ uint2 pending[8][64];
  const uint32_t n_in = ctrl->count[parity];
  const uint32_t n_inj = ctrl->inj_n[parity];
  const unsigned long long inj_base = ctrl->inj_base[parity];
  if (blockIdx.x == 0 && threadIdx.x == 0) ctrl->cursor[parity ^ 1] = 0u;
  const uint64_t total = (uint64_t)n_in + n_inj;
  const uint32_t ln = lane();
  const uint32_t lt = (1u << ln) - 1u;
  uint2* list = pending[threadIdx.x >> 5];
  const uint64_t stride = (uint64_t)gridDim.x * 256;
  uint32_t npend = 0;  // entries in the warp's list (the same in every lane)
  for (uint64_t base = (uint64_t)blockIdx.x * 256 + (threadIdx.x & ~31u);; base += stride) {
    const bool more = base < total;
    if (more) {
      const uint64_t i = base + ln;
      bool has_hit = false;
      uint32_t job = 0;
      if (i < n_in) {
        const uint2 h = in.hit[i];
        const uint32_t meta = __float_as_uint(in.c[i].w);
        job = meta >> 16;
        if (h.x != kDead) {
          has_hit = true;
        } else {
          const BJob& J = A.jobs[job];
          if (J.mode != 0) {  // physical mode: the path ends with the radiance it gathered
            const uint32_t pixel = __float_as_uint(in.o[i].w);
            const float4 ql = in.l[i];
            accumulate(A.accum + 3 * (J.pixel_base + pixel), ql.x, ql.y, ql.z);
          }
        }
      } else if (i < total) {
        const unsigned long long g = inj_base + (i - n_in);
        job = find_job(A.jobs, A.njobs, g, false);
        const BJob& J = A.jobs[job];
        const uint64_t p = J.pixel_base + (g - J.sample_base) / J.spp;
        has_hit = __float_as_uint(A.cam[2 * p + 1].w) != kDead;  // else: a background pixel, nothing gathered
      }
      const unsigned m = __ballot_sync(0xffffffffu, has_hit);
      if (has_hit) list[npend + __popc(m & lt)] = make_uint2((uint32_t)i, job);
      npend += (uint32_t)__popc(m);
      __syncwarp();
    }
    while (npend >= 32u || (!more && npend > 0u)) {
      const uint32_t cnt = npend < 32u ? npend : 32u;
      npend -= cnt;
      bool live = false;
      swrx::PathState st;
      uint32_t pixel = 0, sample = 0, slot = kDead, job = 0;
      float t = 0.0f;
      if (ln < cnt) {
        const uint2 w = list[npend + ln];
        const uint32_t e = w.x;
        job = w.y;
        const BJob& J = A.jobs[job];
        if (e < n_in) {
          const float4 qo = in.o[e], qd = in.d[e], qc = in.c[e];
          const uint2 h = in.hit[e];
          pixel = __float_as_uint(qo.w);
          sample = __float_as_uint(qd.w);
          const uint32_t meta = __float_as_uint(qc.w);
          st.o = mk(qo.x, qo.y, qo.z);
          st.d = mk(qd.x, qd.y, qd.z);
          st.c = mk(qc.x, qc.y, qc.z);
          st.i = (meta >> 8) & 0xFFu;
          st.v = meta & 0xFFu;
          const float4 ql = in.l[e];
          st.L = mk(ql.x, ql.y, ql.z);
          slot = h.x;
          t = __uint_as_float(h.y);
        } else {
          const unsigned long long g = inj_base + (e - n_in);
          const uint64_t local = g - J.sample_base;
          pixel = (uint32_t)(local / J.spp);
          sample = (uint32_t)(local % J.spp);
          const uint64_t p = J.pixel_base + pixel;
          const float4 r0 = A.cam[2 * p], r1 = A.cam[2 * p + 1];
          const uint32_t bits = __float_as_uint(r1.w);
          st.c = mk(1.0f, 1.0f, 1.0f);
          st.L = mk(0.0f, 0.0f, 0.0f);
          st.v = 0;
          st.o = mk(r0.x, r0.y, r0.z);
          st.d = mk(r1.x, r1.y, r1.z);
          st.i = bits >> 27;
          slot = bits & 0x07FFFFFFu;
          t = r0.w;
        }
        const DevScene& sc = A.scenes[J.scene];
        swrx::ShadeParams P;
        P.seed = J.seed;
        P.pixel = pixel;
        P.sample = sample;
        P.depth = J.depth;
        P.mode = J.mode;
        P.rr_depth = J.rr_depth;
        P.rr_q = J.rr_q;
        const uint32_t outcome = swrx::shade_vertex(sc.tris, sc.shade, sc.mats, sc.albedo, slot, t, P, st);
        if (outcome == swrx::kContinue) {
          live = true;
        } else {
          unsigned long long* acc = A.accum + 3 * (J.pixel_base + pixel);
          if (J.mode == 0) {
            if (outcome == swrx::kEndLight) accumulate(acc, st.c.x, st.c.y, st.c.z);
          } else {
            accumulate(acc, st.L.x, st.L.y, st.L.z);
          }
        }
      }
      __syncwarp();  // the list slots just read may be refilled by the next chunk
      const unsigned mask = __ballot_sync(0xffffffffu, live);
      if (mask != 0u) {
        unsigned obase = 0;
        const unsigned leader = __ffs(mask) - 1;
        if (ln == leader) obase = atomicAdd(&ctrl->count[parity ^ 1], (unsigned)__popc(mask));
        obase = __shfl_sync(0xffffffffu, obase, leader);
        if (live) {
          const unsigned j = obase + __popc(mask & lt);
          out.o[j] = make_float4(st.o.x, st.o.y, st.o.z, __uint_as_float(pixel));
          out.d[j] = make_float4(st.d.x, st.d.y, st.d.z, __uint_as_float(sample));
          out.c[j] = make_float4(st.c.x, st.c.y, st.c.z, __uint_as_float((job << 16) | (st.i << 8) | st.v));
          out.l[j] = make_float4(st.L.x, st.L.y, st.L.z, 0.0f);
        }
      }
    }
    if (!more) break;
  }
}

// bounce traversal over the shared queue, refilling idle lanes (as the single-scene kernel)
__global__ void __launch_bounds__(kTB) k_btrace(BArgs A, BCtrl* __restrict__ ctrl, BQueue q, int parity) {
  __shared__ uint2 stack[swrx::kStackShared * kTB];
  const int qp = parity ^ 1;
  const unsigned n = ctrl->count[qp];
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long rem = ctrl->total - ctrl->injected;
    const unsigned long long room = (unsigned long long)A.capacity - n;
    const unsigned long long m = rem < room ? rem : room;
    ctrl->inj_base[qp] = ctrl->injected;
    ctrl->inj_n[qp] = (unsigned)m;
    ctrl->injected += m;
    ctrl->count[parity] = 0u;
    ctrl->rays += n;
  }
  const unsigned ln = lane();
  const unsigned lt = (1u << ln) - 1u;
  swrx::Traversal tr;
  const DevScene* sc = nullptr;
  bool active = false, exhausted = false;
  unsigned ray = 0;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= A.refill) {
      unsigned base = 0;
      if (ln == 0) base = atomicAdd(&ctrl->cursor[qp], (unsigned)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= n) exhausted = true;
      if (!active) {
        const unsigned j = base + __popc(idle & lt);
        if (j < n) {
          const float4 o = q.o[j], d = q.d[j];
          const uint32_t job = __float_as_uint(q.c[j].w) >> 16;
          sc = &A.scenes[A.jobs[job].scene];
          tr.init(mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), stack + threadIdx.x, kTB);
          ray = j;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tr.step<false, false>(sc->nodes, sc->tris, sc->tri_boxes, sc->obj_boxes, nullptr)) {
      q.hit[ray] = make_uint2(tr.hit.slot, __float_as_uint(tr.hit.t));
      active = false;
    }
  }
}

// Batched path-replay adjoint: the single-scene adjoint replay (render.cu, k_adjoint) over the
// batch's global sample range. One persistent launch covers every job: lanes take the next
// global samples (refilling idle lanes), find their job by binary search, start from the job's
// per-pixel camera record and replay the path with the job's scene, seed and Russian roulette,
// then sweep it into the job's gradient buffers. ctrl->injected is the sample cursor.
__global__ void __launch_bounds__(kTB) k_badjoint(BArgs A, BCtrl* __restrict__ ctrl) {
  __shared__ uint2 stack[swrx::kStackShared * kTB];
  const unsigned ln = lane();
  const unsigned lt = (1u << ln) - 1u;
  const unsigned long long total = ctrl->total;
  swrx::Traversal tr;
  swrx::PathState st;
  swrx::AdjointTape tape;
  tape.reset();
  const BJob* J = nullptr;
  const DevScene* sc = nullptr;
  uint32_t pixel = 0, sample = 0, pend_slot = 0;
  float pend_t = 0.0f;
  bool active = false, tracing = false, exhausted = false;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= A.refill) {
      unsigned long long base = 0;
      if (ln == 0) base = atomicAdd(&ctrl->injected, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) exhausted = true;
      if (!active) {
        const unsigned long long g = base + __popc(idle & lt);
        if (g < total) {
          J = &A.jobs[find_job(A.jobs, A.njobs, g, false)];
          const uint64_t local = g - J->sample_base;
          pixel = (uint32_t)(local / J->spp);
          sample = (uint32_t)(local % J->spp);
          const uint64_t p = J->pixel_base + pixel;
          const float4 r0 = A.cam[2 * p], r1 = A.cam[2 * p + 1];
          const uint32_t bits = __float_as_uint(r1.w);
          if (bits != kDead) {
            sc = &A.scenes[J->scene];
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
    if (active && tracing && tr.step<false, false>(sc->nodes, sc->tris, sc->tri_boxes, sc->obj_boxes, nullptr)) {
      tracing = false;
      if (tr.hit.slot == 0xFFFFFFFFu) {  // the path left the scene: no emitter, no gradient
        active = false;
      } else {
        pend_slot = tr.hit.slot;
        pend_t = tr.hit.t;
      }
    }
    // lanes with a pending hit wait until A.batch of them (or every active lane) shade together
    const unsigned waiting = __ballot_sync(0xffffffffu, active && !tracing);
    const unsigned inflight = __ballot_sync(0xffffffffu, active && tracing);
    if (waiting == 0u || ((unsigned)__popc(waiting) < A.batch && inflight != 0u)) continue;
    if (!active || tracing) continue;
    swrx::ShadeParams P;
    P.seed = J->seed;
    P.pixel = pixel;
    P.sample = sample;
    P.depth = J->depth;
    P.mode = 1;
    P.rr_depth = J->rr_depth;
    P.rr_q = J->rr_q;
    const f3 c_before = st.c;
    swrx::AdjVertex av;
    const uint32_t outcome =
        swrx::shade_physical_adj(sc->tris, sc->shade, sc->mats, sc->albedo, pend_slot, pend_t, P, st, av);
    if (outcome == swrx::kContinue) {
      tape.push(pend_slot, c_before, av);
      tr.init(st.o, st.d, stack + threadIdx.x, kTB);
      tracing = true;
      continue;
    }
    if (av.emit_front) {
      const float inv_spp = 1.0f / (float)J->spp;
      const float* dlp = J->dl + (size_t)pixel * 3;
      tape.sweep(sc->tris, sc->mats, sc->albedo, av.obj, c_before,
                 mk(dlp[0] * inv_spp, dlp[1] * inv_spp, dlp[2] * inv_spp), J->g_alb, J->g_em);
    }
    active = false;
  }
}

// End of one iteration of the graph's round loop (eight shade/trace rounds, after which the
// next shade reads parity 0): continue while paths are queued or samples wait for injection; stop
// with status 1 once the proven bound on rounds is exceeded (never reached unless the wavefront
// logic is broken), so the loop always ends.
__global__ void k_bcheck(BCtrl* __restrict__ ctrl, cudaGraphConditionalHandle loop) {
  BCtrl& c = *ctrl;
  c.rounds += 8;
  const bool drained = c.count[0] == 0u && c.inj_n[0] == 0u && c.injected == c.total;
  unsigned go = drained ? 0u : 1u;
  if (!drained && c.rounds > c.max_rounds) {
    c.status = 1u;
    go = 0u;
  }
  cudaGraphSetConditional(loop, go);
}

__global__ void k_bresolve(BArgs A) {
  const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.npix) return;
  const uint32_t j = find_job(A.jobs, A.njobs, p, true);
  const BJob& J = A.jobs[j];
  const float inv = __fdiv_rn(1.0f, (float)J.spp);
  const double s = (J.mode == 0) ? __dmul_rn(6.283185307179586, (double)inv) : (double)inv;
  const unsigned long long* acc = A.accum + 3 * p;
  float* o = J.out + (size_t)(p - J.pixel_base) * 3;
  for (int k = 0; k < 3; ++k)
    o[k] = __double2float_rn((double)(long long)acc[k] / kFix * s);
}

int ensure_bytes(void** p, size_t& have, size_t want) {
  if (have >= want && *p) return SWR_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  have = 0;
  cudaError_t e = cudaMalloc(p, std::max<size_t>(want, 256));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(SWR_ERR_ALLOC, "CUDA: batch workspace allocation of " + std::to_string(want) + " bytes failed");
  }
  have = want;
  return SWR_OK;
}

}  // namespace
}  // namespace swr

struct swr_batch {
  void *qbuf = nullptr, *cam = nullptr, *accum = nullptr, *jobs = nullptr, *scenes = nullptr, *ctrl = nullptr;
  size_t qbytes = 0, cambytes = 0, accbytes = 0, jobbytes = 0, scenebytes = 0, ctrlbytes = 0;
  swr::BCtrl* host_ctrl = nullptr;                                  // [4] pinned control blocks
  cudaGraphExec_t graph[4] = {nullptr, nullptr, nullptr, nullptr};  // round loop per sub-wavefront
  std::vector<char> graph_key[4];
  cudaStream_t side[3] = {nullptr, nullptr, nullptr};  // streams of sub-wavefronts 1..3
  cudaEvent_t fork = nullptr, join[3] = {nullptr, nullptr, nullptr};
  int device = -1;
};

using swr::set_error;

namespace swr {
namespace {

// Appends one job to the table (validating what the primal and the adjoint both need); uniq / hs
// collect the distinct scenes, samples / pixels the running prefix sums.
int add_job(int device, const swr_scene* scene, const swr_camera& cam, const swr_render_opts& o, BJob& d,
            std::vector<const swr_scene*>& uniq, std::vector<DevScene>& hs, uint64_t& samples, uint64_t& pixels) {
  if (!scene) return set_error(SWR_ERR_INVALID, "swr: batch job without scene");
  if (scene->device != device) return set_error(SWR_ERR_INVALID, "swr: batch jobs on another device");
  if (o.width == 0 || o.height == 0 || o.spp == 0) return set_error(SWR_ERR_INVALID, "swr: zero image size");
  if ((uint64_t)o.width * o.height >= (1ull << 32)) return set_error(SWR_ERR_INVALID, "swr: image too large");
  if (o.max_depth == 0 || o.max_depth > 31) return set_error(SWR_ERR_INVALID, "swr: max_depth must be 1..31");
  if (o.mode > 1) return set_error(SWR_ERR_INVALID, "swr: unknown mode");
  if (o.mode == 1 && o.rr_depth && !(o.rr_survive > 0.0f && o.rr_survive <= 1.0f))
    return set_error(SWR_ERR_INVALID, "swr: rr_survive must be in (0, 1]");
  if (o.sample_begin || o.spp_total || o.pixel_begin || o.pixel_count)
    return set_error(SWR_ERR_UNSUPPORTED, "swr: batch jobs render whole images (the range fields must be 0)");
  uint32_t si = 0;
  while (si < uniq.size() && uniq[si] != scene) ++si;
  if (si == uniq.size()) {
    uniq.push_back(scene);
    hs.push_back(scene->dev);
  }
  std::memset(&d, 0, sizeof(d));
  std::memcpy(d.vi, cam.view_inv, sizeof(d.vi));
  std::memcpy(d.pi, cam.proj_inv, sizeof(d.pi));
  std::memcpy(d.org, cam.origin, sizeof(d.org));
  d.W = o.width;
  d.H = o.height;
  d.spp = o.spp;
  d.depth = o.max_depth;
  d.mode = o.mode;
  d.rr_depth = o.mode == 1 ? o.rr_depth : 0;
  d.rr_q = (o.mode == 1 && o.rr_depth) ? o.rr_survive : 1.0f;
  d.scene = si;
  d.seed = o.seed;
  d.sample_base = samples;
  d.pixel_base = pixels;
  const uint64_t np = (uint64_t)o.width * o.height;
  pixels += np;
  samples += np * o.spp;
  return SWR_OK;
}

}  // namespace
}  // namespace swr

extern "C" {

int swr_batch_create(swr_batch** out) {
  if (!out) return set_error(SWR_ERR_INVALID, "swr: null output handle");
  std::unique_ptr<swr_batch> b(new swr_batch());
  SWR_CUDA(cudaGetDevice(&b->device));
  SWR_CUDA(cudaMallocHost(&b->host_ctrl, 4 * sizeof(swr::BCtrl)));
  *out = b.release();
  return SWR_OK;
}

void swr_batch_destroy(swr_batch* b) {
  if (!b) return;
  for (int h = 0; h < 4; ++h)
    if (b->graph[h]) cudaGraphExecDestroy(b->graph[h]);
  for (int h = 0; h < 3; ++h) {
    if (b->side[h]) cudaStreamDestroy(b->side[h]);
    if (b->join[h]) cudaEventDestroy(b->join[h]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  for (void* p : {b->qbuf, b->cam, b->accum, b->jobs, b->scenes, b->ctrl})
    if (p) cudaFree(p);
  if (b->host_ctrl) cudaFreeHost(b->host_ctrl);
  delete b;
}

int swr_render_batch(swr_batch* b, const swr_batch_job* jobs, uint32_t n, const swr_batch_opts* bo,
                     void* stream_) {
  using namespace swr;
  if (!b || !jobs || n == 0) return set_error(SWR_ERR_INVALID, "swr: empty batch");
  if (n > 65535) return set_error(SWR_ERR_UNSUPPORTED, "swr: at most 65535 jobs per batch");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(b->device));
  std::vector<BJob> hj(n);
  std::vector<DevScene> hs;
  std::vector<const swr_scene*> uniq;
  uint64_t samples = 0, pixels = 0;
  int num_sms = 0;
  int rc;
  for (uint32_t k = 0; k < n; ++k) {
    const swr_batch_job& J = jobs[k];
    if (!J.rgb_out) return set_error(SWR_ERR_INVALID, "swr: batch job without output");
    if ((rc = add_job(b->device, J.scene, J.cam, J.opts, hj[k], uniq, hs, samples, pixels))) return rc;
    if (is_host_pointer(J.rgb_out)) return set_error(SWR_ERR_INVALID, "swr: batch outputs must be device memory");
    hj[k].out = J.rgb_out;
    num_sms = J.scene->num_sms;
  }
  uint32_t cap = (bo && bo->wave_size) ? bo->wave_size : (1u << 23);
  cap = (uint32_t)std::min<uint64_t>(cap, samples);
  cap = std::max<uint32_t>(32, (cap + 255u) & ~255u);
  const uint32_t refill = (bo && bo->refill) ? bo->refill : 8;
  if (refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  if ((rc = ensure_bytes(&b->qbuf, b->qbytes, (size_t)cap * (4 * sizeof(float4) + sizeof(uint2)) * 2))) return rc;
  if ((rc = ensure_bytes(&b->cam, b->cambytes, pixels * 2 * sizeof(float4)))) return rc;
  if ((rc = ensure_bytes(&b->accum, b->accbytes, pixels * 3 * sizeof(unsigned long long)))) return rc;
  if ((rc = ensure_bytes(&b->jobs, b->jobbytes, n * sizeof(BJob)))) return rc;
  if ((rc = ensure_bytes(&b->scenes, b->scenebytes, hs.size() * sizeof(DevScene)))) return rc;
  if ((rc = ensure_bytes(&b->ctrl, b->ctrlbytes, 4 * sizeof(BCtrl)))) return rc;
  SWR_CUDA(cudaMemcpyAsync(b->jobs, hj.data(), n * sizeof(BJob), cudaMemcpyHostToDevice, stream));
  SWR_CUDA(cudaMemcpyAsync(b->scenes, hs.data(), hs.size() * sizeof(DevScene), cudaMemcpyHostToDevice, stream));
  SWR_CUDA(cudaMemsetAsync(b->accum, 0, pixels * 3 * sizeof(unsigned long long), stream));
  // zero-filled first: the struct's bytes, padding included, are the graph cache's key
  BArgs A;
  std::memset(&A, 0, sizeof(A));
  A.jobs = (const BJob*)b->jobs;
  A.scenes = (const DevScene*)b->scenes;
  A.njobs = n;
  A.npix = pixels;
  A.capacity = cap;
  A.refill = refill;
  A.cam = (float4*)b->cam;
  A.accum = (unsigned long long*)b->accum;
  uint32_t maxdepth = 0;
  for (uint32_t k = 0; k < n; ++k) maxdepth = std::max(maxdepth, jobs[k].opts.max_depth);
  const bool use_graph = !(bo && (bo->flags & SWR_BATCH_NO_GRAPH));
  // With the graph, large batches run as kBatchSubWaves sub-wavefronts over consecutive ranges of
  // the global sample index (a share of the paths in flight each) on as many streams, so that the
  // SMs one leaves idle at the end of a traversal launch take another's work; the per-pixel sums
  // are order-independent fixed point, so the images do not depend on it.
  const int nsub = (use_graph && samples >= kBatchTwoWaveSamples && cap >= 256u * kBatchSubWaves) ? kBatchSubWaves : 1;
  const uint32_t capw = nsub > 1 ? (cap / nsub) & ~255u : cap;
  A.capacity = capw;  // each sub-wavefront's queue
  BCtrl* dctrl = (BCtrl*)b->ctrl;
  SWR_CUDA(cudaStreamSynchronize(stream));  // the pinned control blocks may still be in flight
  for (int h = 0; h < nsub; ++h) {
    const uint64_t s0 = samples * h / nsub, s1 = samples * (h + 1) / nsub;
    BCtrl init;
    std::memset(&init, 0, sizeof(init));
    init.total = s1;  // the sub-wavefront's end in the global sample index
    init.inj_base[0] = s0;
    init.inj_n[0] = (unsigned)std::min<uint64_t>(capw, s1 - s0);
    init.injected = s0 + init.inj_n[0];
    // every path ends within max_depth rounds of its injection and each round injects up to the
    // queue capacity, so this many rounds always suffice; more means a logic error
    init.max_rounds = ((s1 - s0) / capw + 2) * (uint64_t)(maxdepth + 2) + 64;
    b->host_ctrl[h] = init;
  }
  SWR_CUDA(cudaMemcpyAsync(dctrl, b->host_ctrl, nsub * sizeof(BCtrl), cudaMemcpyHostToDevice, stream));
  k_bcamera<<<bcamera_grid(num_sms, pixels), kTB, 0, stream>>>(A, dctrl);
  SWR_CUDA(cudaGetLastError());
  int per_sm = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_btrace, kTB, 0));
  const unsigned tgrid = (unsigned)(num_sms * std::max(per_sm, 1));
  int shade_per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shade_per_sm, k_bshade, 256, 0) != cudaSuccess) {
    cudaGetLastError();
    shade_per_sm = 1;
  }
  // persistent shading grid (its warps stride over the queue)
  const unsigned sgrid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((capw + 255) / 256, (uint64_t)num_sms * std::max(shade_per_sm, 1)));
  auto queues = [&](int h, BQueue* Qh) {
    char* p = (char*)b->qbuf + (size_t)h * ((size_t)capw * (4 * sizeof(float4) + sizeof(uint2)) * 2);
    for (int k = 0; k < 2; ++k) {
      Qh[k].o = (float4*)p; p += (size_t)capw * sizeof(float4);
      Qh[k].d = (float4*)p; p += (size_t)capw * sizeof(float4);
      Qh[k].c = (float4*)p; p += (size_t)capw * sizeof(float4);
      Qh[k].l = (float4*)p; p += (size_t)capw * sizeof(float4);
      Qh[k].hit = (uint2*)p; p += (size_t)capw * sizeof(uint2);
    }
  };
  auto enqueue_rounds = [&](cudaStream_t st, BCtrl* ctrl, const BQueue* Qh) {
    for (int k = 0; k < 8; ++k) {
      const int p = k & 1;
      k_bshade<<<sgrid, 256, 0, st>>>(A, ctrl, Qh[p], Qh[p ^ 1], p);
      k_btrace<<<tgrid, kTB, 0, st>>>(A, ctrl, Qh[p ^ 1], p);
    }
  };
  if (use_graph) {
    if (nsub > 1 && !b->fork) {
      SWR_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
      for (int h = 0; h < 3; ++h) {
        SWR_CUDA(cudaStreamCreateWithFlags(&b->side[h], cudaStreamNonBlocking));
        SWR_CUDA(cudaEventCreateWithFlags(&b->join[h], cudaEventDisableTiming));
      }
    }
    if (nsub > 1) SWR_CUDA(cudaEventRecord(b->fork, stream));
    for (int h = 0; h < nsub; ++h) {
      BQueue Qh[2];
      queues(h, Qh);
      BCtrl* ctrl = dctrl + h;
      // the whole round loop as one graph (a WHILE node over eight rounds and k_bcheck), rebuilt
      // whenever an argument baked into it changes
      std::vector<char> key(sizeof(A) + sizeof(Qh) + 3 * sizeof(void*));
      {
        char* k = key.data();
        std::memset(k, 0, key.size());
        std::memcpy(k, &A, sizeof(A));
        std::memcpy(k + sizeof(A), Qh, sizeof(Qh));
        const void* extra[3] = {ctrl, (void*)(uintptr_t)sgrid, (void*)(uintptr_t)tgrid};
        std::memcpy(k + sizeof(A) + sizeof(Qh), extra, sizeof(extra));
      }
      if (!b->graph[h] || key != b->graph_key[h]) {
        if (b->graph[h]) cudaGraphExecDestroy(b->graph[h]);
        b->graph[h] = nullptr;
        b->graph_key[h].clear();
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
          enqueue_rounds(cs, ctrl, Qh);
          k_bcheck<<<1, 1, 0, cs>>>(ctrl, loop);
          cudaGraph_t captured = nullptr;
          SWR_CUDA(cudaStreamEndCapture(cs, &captured));
          SWR_CUDA(cudaGraphInstantiate(&b->graph[h], g, 0));
          return SWR_OK;
        };
        const int brc = build();
        if (cs) cudaStreamDestroy(cs);
        if (g) cudaGraphDestroy(g);
        if (brc) {
          if (b->graph[h]) cudaGraphExecDestroy(b->graph[h]);
          b->graph[h] = nullptr;
          return brc;
        }
        b->graph_key[h] = key;
      }
      cudaStream_t st = h ? b->side[h - 1] : stream;
      if (h) SWR_CUDA(cudaStreamWaitEvent(st, b->fork, 0));
      SWR_CUDA(cudaGraphLaunch(b->graph[h], st));
      SWR_CUDA(cudaGetLastError());
      if (h) SWR_CUDA(cudaEventRecord(b->join[h - 1], st));
    }
    for (int h = 1; h < nsub; ++h) SWR_CUDA(cudaStreamWaitEvent(stream, b->join[h - 1], 0));
  } else {
    // without a graph the host runs the loop: eight rounds, then a look at the control block
    BQueue Q0[2];
    queues(0, Q0);
    uint64_t rounds = 0;
    for (;;) {
      if (rounds > b->host_ctrl[0].max_rounds) return set_error(SWR_ERR_TIMEOUT, "swr: batch wavefront did not drain");
      enqueue_rounds(stream, dctrl, Q0);
      rounds += 8;
      SWR_CUDA(cudaGetLastError());
      SWR_CUDA(cudaMemcpyAsync(b->host_ctrl, dctrl, sizeof(BCtrl), cudaMemcpyDeviceToHost, stream));
      SWR_CUDA(cudaStreamSynchronize(stream));
      const BCtrl& h = *b->host_ctrl;
      // after an even number of rounds the next shade reads parity 0
      if (h.count[0] == 0 && h.inj_n[0] == 0 && h.injected == h.total) break;
    }
  }
  k_bresolve<<<(unsigned)((pixels + 255) / 256), 256, 0, stream>>>(A);
  SWR_CUDA(cudaGetLastError());
  if (use_graph) {
    // the one wait of the call: the device-side loops' status
    SWR_CUDA(cudaMemcpyAsync(b->host_ctrl, dctrl, nsub * sizeof(BCtrl), cudaMemcpyDeviceToHost, stream));
    SWR_CUDA(cudaStreamSynchronize(stream));
    for (int h = 0; h < nsub; ++h)
      if (b->host_ctrl[h].status) return set_error(SWR_ERR_TIMEOUT, "swr: batch wavefront did not drain");
  }
  return SWR_OK;
}

int swr_render_adjoint_batch(swr_batch* b, const swr_adjoint_job* jobs, uint32_t n, const swr_batch_opts* bo,
                             void* stream_) {
  using namespace swr;
  if (!b || !jobs || n == 0) return set_error(SWR_ERR_INVALID, "swr: empty batch");
  if (n > 65535) return set_error(SWR_ERR_UNSUPPORTED, "swr: at most 65535 jobs per batch");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(b->device));
  std::vector<BJob> hj(n);
  std::vector<DevScene> hs;
  std::vector<const swr_scene*> uniq;
  uint64_t samples = 0, pixels = 0;
  int num_sms = 0;
  int rc;
  // distinct gradient buffers and their sizes in bytes (zeroed once each; jobs that share a
  // buffer add into it)
  std::vector<std::pair<float*, size_t>> zero;
  auto note = [&](float* p, size_t bytes) -> int {
    for (auto& z : zero)
      if (z.first == p) {
        if (z.second != bytes) return set_error(SWR_ERR_INVALID, "swr: a gradient buffer is shared by scenes of "
                                                                 "different sizes");
        return SWR_OK;
      }
    zero.emplace_back(p, bytes);
    return SWR_OK;
  };
  for (uint32_t k = 0; k < n; ++k) {
    const swr_adjoint_job& J = jobs[k];
    if (!J.dl_dimage || !J.dl_dalbedo || !J.dl_demission) return set_error(SWR_ERR_INVALID, "swr: null argument");
    if (J.opts.mode != SWR_MODE_PHYSICAL)
      return set_error(SWR_ERR_INVALID, "swr: the adjoint is defined for SWR_MODE_PHYSICAL");
    if (J.opts.max_depth > (uint32_t)swrx::kAdjMaxDepth)
      return set_error(SWR_ERR_UNSUPPORTED, "swr: the adjoint supports max_depth 1..16");
    if ((rc = add_job(b->device, J.scene, J.cam, J.opts, hj[k], uniq, hs, samples, pixels))) return rc;
    if (is_host_pointer(J.dl_dimage) || is_host_pointer(J.dl_dalbedo) || is_host_pointer(J.dl_demission))
      return set_error(SWR_ERR_INVALID, "swr: the adjoint takes device buffers");
    hj[k].dl = J.dl_dimage;
    hj[k].g_alb = J.dl_dalbedo;
    hj[k].g_em = J.dl_demission;
    if ((rc = note(J.dl_dalbedo, (size_t)J.scene->dev.num_tris * 3 * sizeof(float)))) return rc;
    if ((rc = note(J.dl_demission, (size_t)J.scene->dev.num_objects * 3 * sizeof(float)))) return rc;
    num_sms = J.scene->num_sms;
  }
  const uint32_t refill = (bo && bo->refill) ? bo->refill : 8;
  if (refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  const uint32_t batch = (bo && bo->shade_batch) ? bo->shade_batch : swrx::kAdjointBatch;
  if (batch > 32) return set_error(SWR_ERR_INVALID, "swr: shade_batch must be 0..32");
  if ((rc = ensure_bytes(&b->cam, b->cambytes, pixels * 2 * sizeof(float4)))) return rc;
  if ((rc = ensure_bytes(&b->jobs, b->jobbytes, n * sizeof(BJob)))) return rc;
  if ((rc = ensure_bytes(&b->scenes, b->scenebytes, hs.size() * sizeof(DevScene)))) return rc;
  if ((rc = ensure_bytes(&b->ctrl, b->ctrlbytes, 4 * sizeof(BCtrl)))) return rc;
  SWR_CUDA(cudaMemcpyAsync(b->jobs, hj.data(), n * sizeof(BJob), cudaMemcpyHostToDevice, stream));
  SWR_CUDA(cudaMemcpyAsync(b->scenes, hs.data(), hs.size() * sizeof(DevScene), cudaMemcpyHostToDevice, stream));
  for (auto& z : zero) SWR_CUDA(cudaMemsetAsync(z.first, 0, z.second, stream));
  BArgs A;
  std::memset(&A, 0, sizeof(A));
  A.jobs = (const BJob*)b->jobs;
  A.scenes = (const DevScene*)b->scenes;
  A.njobs = n;
  A.npix = pixels;
  A.refill = refill;
  A.batch = batch;
  A.cam = (float4*)b->cam;
  BCtrl init;
  std::memset(&init, 0, sizeof(init));
  init.total = samples;
  SWR_CUDA(cudaStreamSynchronize(stream));  // the pinned control block may still be in flight
  *b->host_ctrl = init;
  SWR_CUDA(cudaMemcpyAsync(b->ctrl, b->host_ctrl, sizeof(BCtrl), cudaMemcpyHostToDevice, stream));
  k_bcamera<<<bcamera_grid(num_sms, pixels), kTB, 0, stream>>>(A, (BCtrl*)b->ctrl);
  SWR_CUDA(cudaGetLastError());
  int per_sm = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_badjoint, kTB, 0));
  k_badjoint<<<(unsigned)(num_sms * std::max(per_sm, 1)), kTB, 0, stream>>>(A, (BCtrl*)b->ctrl);
  SWR_CUDA(cudaGetLastError());
  return SWR_OK;
}

}  // extern "C"
