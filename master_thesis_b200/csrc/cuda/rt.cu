// The Vulkan application's PathTracer and its two denoisers as CUDA kernels over the library's
// scene (C ABI: swr_rt_render, swr_rt_render_frame, swr_rt_denoise_gauss, swr_rt_denoise_median).
//
// The reference runs these as ray tracing pipeline and compute shaders (RayTrace program,
// src/main.cpp:58-76; res/shader/path_tracer_vision_raygen.rgen:8-60, denoise_gauss_comp.comp,
// denoise_median_comp.comp). Here traceRay is the wide-BVH traversal with the ray-query hit rule
// (swr_bvh.cuh, kRuleRayQuery) and the shader arithmetic is rt_shading.cuh.
//
//   k_rt_path    persistent: one lane per pixel runs the raygen shader for its pixel (the LCG
//                state is per pixel and carried from sample to sample, so a pixel's samples are
//                sequential). Every traceRay is the resumable Traversal, so lanes of a warp trace
//                independently; lanes whose ray is finished wait until `shade_batch` of them can
//                run the shading code together (then issue their next rays), and a warp with
//                `refill` idle lanes takes that many new pixels with one atomic. Measured on
//                1920x1080 frames (13 paths per pixel): shading each finished ray at once ran the
//                shading code for one or two lanes at a time (7.2 of 32 lanes per instruction);
//                batching 12-16 lanes made the Cornell frame 1.9x and the terrain frame 1.2x
//                faster.
//   k_rt_gauss   one thread per pixel: the (2*off+1)^2 weighted taps in the shader's order, from
//                a shared-memory tile of converted texels.
//   k_rt_median  one thread per pixel: per-channel median of the 3x3 neighbourhood, from a
//                shared-memory tile.
#include <algorithm>
#include <cstring>

#include "rt_shading.cuh"
#include "swr_internal.cuh"

namespace swr {
namespace {

using swrx::f3;
using swrx::mk;
namespace rt = swrx::rt;

constexpr int kBlock = 128;
constexpr uint32_t kMiss = 0xFFFFFFFFu;
constexpr uint32_t kMaxJumps = 1u << 16;
constexpr uint32_t kMaxSpp = 1u << 24;
constexpr uint32_t kMaxGauss = 19;  // GAUSS_ARRAY_MAX_SIZE 20 holds the odd sizes up to 19

struct RtFrame {
  float vi[16], pi[16];
  uint32_t W, H, vj, spp;
  uint32_t refill;
  uint32_t shade_batch;  // lanes of a warp whose ray finished that trigger a shading pass
  float scale;      // (2 * PI) / float(spp)
  float* rgb;       // [W*H*3] finalColor, or null
  uchar4* rgba;     // [W*H] the stored rgba8 pixel, or null
};

enum RtStage : uint32_t { kPrimary = 0, kSampleStart = 1, kJump = 2, kJumpResult = 3 };

__device__ __forceinline__ void store_pixel(const RtFrame& F, uint32_t p, f3 c) {
  if (F.rgb) {
    F.rgb[3 * (size_t)p + 0] = c.x;
    F.rgb[3 * (size_t)p + 1] = c.y;
    F.rgb[3 * (size_t)p + 2] = c.z;
  }
  if (F.rgba) F.rgba[p] = make_uchar4(rt::unorm8(c.x), rt::unorm8(c.y), rt::unorm8(c.z), 0);
}

// The first hit's payload of each lane's pixel (the raygen's defaultRayPayload), read back at the
// start of every sample: kept in shared memory, one column per thread, instead of 12 registers.
struct DefPayload {
  float v[12][kBlock];
  __device__ void put(const rt::Payload& P) {
    const float a[12] = {P.pos.x, P.pos.y, P.pos.z, P.n.x, P.n.y, P.n.z, P.color.x, P.color.y, P.color.z,
                         P.dT, P.rT, P.tT};
#pragma unroll
    for (int k = 0; k < 12; ++k) v[k][threadIdx.x] = a[k];
  }
  __device__ rt::Payload get(float eta) const {
    rt::Payload P;
    const unsigned t = threadIdx.x;
    P.pos = mk(v[0][t], v[1][t], v[2][t]);
    P.n = mk(v[3][t], v[4][t], v[5][t]);
    P.color = mk(v[6][t], v[7][t], v[8][t]);
    P.dT = v[9][t];
    P.rT = v[10][t];
    P.tT = v[11][t];
    P.eta = eta;
    P.light = 0u;  // a first hit on a light ends the pixel before any sample
    return P;
  }
};

// kMinBlocks: resident blocks per SM the register budget targets (0 = the compiler's choice)
template <int kMinBlocks>
__global__ void __launch_bounds__(kBlock, kMinBlocks)
    k_rt_path(DevScene sc, RtFrame F, unsigned long long* __restrict__ cursor) {
  __shared__ uint2 stack[swrx::kStackShared * kBlock];
  __shared__ DefPayload defs;
  const unsigned lane = threadIdx.x & 31u;
  const unsigned lt = (1u << lane) - 1u;
  const unsigned long long total = (unsigned long long)F.W * F.H;
  swrx::Traversal tr;
  rt::Payload cur;
  float def_eta = 0.0f;
  uint32_t pixel = 0, rng = 0, s = 0, i = 0, cull = 0, stage = kPrimary;
  bool active = false, tracing = false, exhausted = false;
  f3 o = mk(0, 0, 0), d = mk(0, 0, 0), sdir = mk(0, 0, 0), col = mk(0, 0, 0), fin = mk(0, 0, 0);
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !active);
    if (!exhausted && (unsigned)__popc(idle) >= F.refill) {
      unsigned long long base = 0;
      if (lane == 0) base = atomicAdd(cursor, (unsigned long long)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base >= total) exhausted = true;
      if (!active) {
        const unsigned long long g = base + __popc(idle & lt);
        if (g < total) {
          pixel = (uint32_t)g;
          const uint32_t x = pixel % F.W, y = pixel / F.W;
          rng = rt::lcg_init(x, y, 0u);
          rt::vision_ray(F.vi, F.pi, x, y, F.W, F.H, o, d);
          sdir = d;
          cull = 0;
          fin = mk(0.0f, 0.0f, 0.0f);
          stage = kPrimary;
          tr.init(o, d, stack + threadIdx.x, kBlock);
          tracing = true;
          active = true;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) {
      if (exhausted) break;
      continue;
    }
    if (active && tracing &&
        tr.step<false, false, swrx::kRuleRayQuery>(sc.nodes, sc.tris, sc.tri_boxes, sc.obj_boxes, nullptr))
      tracing = false;
    // Lanes whose ray is finished wait until shade_batch of them (or every active lane) can shade
    // together: the shading code then runs once for many lanes instead of once per finished ray.
    const unsigned waiting = __ballot_sync(0xffffffffu, active && !tracing);
    const unsigned inflight = __ballot_sync(0xffffffffu, active && tracing);
    if (waiting == 0u || ((unsigned)__popc(waiting) < F.shade_batch && inflight != 0u)) continue;
    if (!active || tracing) continue;
    const uint32_t hs = tr.hit.slot;
    if (stage == kPrimary) {
      // traceRay with back-face culling: up to four traces, each retry from the culled hit
      if (hs == kMiss) {
        store_pixel(F, pixel, mk(0.0f, 0.0f, 0.0f));
        active = false;
        continue;
      }
      const rt::Payload P = rt::hit_payload(sc.tris, sc.shade, sc.mats, hs, o, d);
      if (swrx::vdot(P.n, d) > 0.0f && cull < 3) {
        o = P.pos;
        ++cull;
        tr.init(o, d, stack + threadIdx.x, kBlock);
        tracing = true;
        continue;
      }
      if (P.light) {  // a light seen directly: its color * lightStrength, unscaled
        store_pixel(F, pixel, P.color);
        active = false;
        continue;
      }
      defs.put(P);
      def_eta = P.eta;
      s = 0;
      stage = kSampleStart;
    } else {  // kJumpResult
      if (hs == kMiss) {  // color = 0: the sample adds nothing
        ++s;
        stage = kSampleStart;
      } else {
        const rt::Payload P = rt::hit_payload(sc.tris, sc.shade, sc.mats, hs, o, d);
        if (P.light && swrx::vdot(d, P.n) <= 0.0f) {
          col = swrx::vmul(col, P.color);
          fin = swrx::vadd(fin, col);
          ++s;
          stage = kSampleStart;
        } else {
          cur = P;
          ++i;
          stage = kJump;
        }
      }
    }
    // run the raygen loops until the next traceRay or the end of the pixel
    while (!tracing) {
      if (stage == kSampleStart) {
        if (s >= F.spp) {
          store_pixel(F, pixel, swrx::vscale(F.scale, fin));
          active = false;
          break;
        }
        cur = defs.get(def_eta);
        d = sdir;
        col = mk(1.0f, 1.0f, 1.0f);
        i = 1;
        stage = kJump;
      }
      if (i >= F.vj) {  // the jumps ran out before a light was hit
        ++s;
        stage = kSampleStart;
        continue;
      }
      if (rt::handle_hit(cur, rng, o, d)) {
        const float cs = swrx::vdot(d, cur.n);
        col = swrx::vmul(col, mk(swrx::fmul(cur.color.x, cs), swrx::fmul(cur.color.y, cs),
                                 swrx::fmul(cur.color.z, cs)));
      }
      tr.init(o, d, stack + threadIdx.x, kBlock);
      tracing = true;
      stage = kJumpResult;
    }
  }
}

struct GaussArgs {
  float g[kMaxGauss + 1];
  int off;
  uint32_t W, H;
};

// Denoiser blocks: 32 x 8 threads, one output texel each. A block first stages the texels its
// outputs read (the halo of the largest kernel, 19 taps, included) in shared memory, converted
// once per block; texels outside the image are stored as zeros, which add +0 to a tap sum that
// never holds -0, so the sum is the shader's sum over the in-image taps alone.
constexpr int kDx = 32, kDy = 8;
constexpr int kGaussTile = (kDx + 2 * (kMaxGauss / 2)) * (kDy + 2 * (kMaxGauss / 2));

__global__ void __launch_bounds__(kDx * kDy) k_rt_gauss(const uchar4* __restrict__ in, uchar4* __restrict__ out,
                                                        GaussArgs A) {
  __shared__ float lut[256];
  __shared__ float g[kMaxGauss + 1];
  __shared__ float4 tile[kGaussTile];
  const int tid = (int)(threadIdx.y * kDx + threadIdx.x);
  // imageLoad of an rgba8 texel: byte / 255 as an IEEE float quotient
  lut[tid] = __fdiv_rn((float)tid, 255.0f);
  if (tid <= kMaxGauss) g[tid] = A.g[tid];
  __syncthreads();
  const int W = (int)A.W, H = (int)A.H, off = A.off;
  const int tw = kDx + 2 * off, th = kDy + 2 * off;
  const int x0 = (int)blockIdx.x * kDx - off, y0 = (int)blockIdx.y * kDy - off;
  for (int k = tid; k < tw * th; k += kDx * kDy) {
    const int ty = k / tw, tx = k - ty * tw;
    const int px = x0 + tx, py = y0 + ty;
    float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (px >= 0 && px < W && py >= 0 && py < H) {
      const uchar4 b = __ldg(in + (size_t)py * W + px);
      v = make_float4(lut[b.x], lut[b.y], lut[b.z], lut[b.w]);
    }
    tile[k] = v;
  }
  __syncthreads();
  const int x = (int)(blockIdx.x * kDx + threadIdx.x), y = (int)(blockIdx.y * kDy + threadIdx.y);
  if (x >= W || y >= H) return;
  float4 c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int dx = 0; dx <= 2 * off; ++dx) {  // x offset outer, y offset inner, as the shader loops
    const float gx = g[dx];
    const float4* col = tile + (int)threadIdx.y * tw + (int)threadIdx.x + dx;
    for (int dy = 0; dy <= 2 * off; ++dy) {
      const float gy = g[dy];
      const float4 v = col[dy * tw];
      c.x = __fadd_rn(c.x, __fmul_rn(__fmul_rn(v.x, gx), gy));
      c.y = __fadd_rn(c.y, __fmul_rn(__fmul_rn(v.y, gx), gy));
      c.z = __fadd_rn(c.z, __fmul_rn(__fmul_rn(v.z, gx), gy));
      c.w = __fadd_rn(c.w, __fmul_rn(__fmul_rn(v.w, gx), gy));
    }
  }
  out[(size_t)y * W + x] = make_uchar4(rt::unorm8(c.x), rt::unorm8(c.y), rt::unorm8(c.z), rt::unorm8(c.w));
}

// Median of nine per byte lane: sort each row of three, then the median of (largest row
// minimum, median of the row medians, smallest row maximum). Selecting among the loaded texels
// and storing the selected one back is exact, so the work stays on the packed bytes.
__device__ __forceinline__ void ex(uint32_t& a, uint32_t& b) {
  const uint32_t lo = __vminu4(a, b);
  b = __vmaxu4(a, b);
  a = lo;
}
__device__ __forceinline__ uint32_t med3(uint32_t a, uint32_t b, uint32_t c) {
  return __vmaxu4(__vminu4(a, b), __vminu4(__vmaxu4(a, b), c));
}

__global__ void __launch_bounds__(kDx * kDy) k_rt_median(const uint32_t* __restrict__ in,
                                                         uint32_t* __restrict__ out, uint32_t W, uint32_t H) {
  constexpr int tw = kDx + 2, th = kDy + 2;
  __shared__ uint32_t tile[tw * th];
  const int tid = (int)(threadIdx.y * kDx + threadIdx.x);
  const int x0 = (int)blockIdx.x * kDx - 1, y0 = (int)blockIdx.y * kDy - 1;
  for (int k = tid; k < tw * th; k += kDx * kDy) {
    const int ty = k / tw, tx = k - ty * tw;
    const int px = x0 + tx, py = y0 + ty;
    // texels outside the image are undefined in the shader; they count as 0 here
    tile[k] = (px >= 0 && px < (int)W && py >= 0 && py < (int)H) ? __ldg(in + (size_t)py * W + px) : 0u;
  }
  __syncthreads();
  const int x = (int)(blockIdx.x * kDx + threadIdx.x), y = (int)(blockIdx.y * kDy + threadIdx.y);
  if (x >= (int)W || y >= (int)H) return;
  uint32_t v[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int k = 0; k < 3; ++k) v[3 * r + k] = tile[((int)threadIdx.y + r) * tw + (int)threadIdx.x + k];
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    ex(v[3 * r], v[3 * r + 1]);
    ex(v[3 * r + 1], v[3 * r + 2]);
    ex(v[3 * r], v[3 * r + 1]);
  }
  const uint32_t lo = __vmaxu4(__vmaxu4(v[0], v[3]), v[6]);
  const uint32_t hi = __vminu4(__vminu4(v[2], v[5]), v[8]);
  const uint32_t mid = med3(v[1], v[4], v[7]);
  out[(size_t)y * W + x] = med3(lo, mid, hi);
}

int check_image(uint32_t W, uint32_t H) {
  if (W == 0 || H == 0) return set_error(SWR_ERR_INVALID, "swr: image size must be positive");
  if ((uint64_t)W * H > (1ull << 31)) return set_error(SWR_ERR_INVALID, "swr: image too large");
  return SWR_OK;
}

// Device view of a caller buffer: the buffer itself, or a stream-ordered temporary when it is host
// memory (copied in when `in`, copied back by finish()).
struct Staged {
  void* user = nullptr;
  void* dev = nullptr;
  size_t bytes = 0;
  bool host = false;
};

int stage(void* user, size_t bytes, bool in, cudaStream_t stream, Staged& st) {
  st.user = user;
  st.bytes = bytes;
  st.dev = user;
  st.host = user && is_host_pointer(user);
  if (!st.host) return SWR_OK;
  SWR_CUDA(cudaMallocAsync(&st.dev, bytes, stream));
  if (in) SWR_CUDA(cudaMemcpyAsync(st.dev, user, bytes, cudaMemcpyHostToDevice, stream));
  return SWR_OK;
}

void release(Staged& st, cudaStream_t stream) {
  if (st.host && st.dev) cudaFreeAsync(st.dev, stream);
  st.dev = nullptr;
}

// The scene's RayTrace buffer, at least `need` bytes (grown on demand; growing waits for the
// stream, whose earlier frames may still read the old buffer). Frames into host memory and frames
// with denoisers then allocate nothing per call.
int rt_buffer(swr_scene* s, size_t need, cudaStream_t stream, char** out) {
  if (need > s->rt_buf_bytes) {
    SWR_CUDA(cudaStreamSynchronize(stream));
    if (s->rt_buf) SWR_CUDA(cudaFree(s->rt_buf));
    s->rt_buf = nullptr;
    s->rt_buf_bytes = 0;
    SWR_CUDA(cudaMalloc(&s->rt_buf, need));
    s->rt_buf_bytes = need;
  }
  *out = (char*)s->rt_buf;
  return SWR_OK;
}

// Device view of an output buffer from the scene's RayTrace buffer at `*at` (advanced past it)
// when it is host memory.
void stage_out(void* user, size_t bytes, char* buf, size_t* at, Staged& st) {
  st.user = user;
  st.bytes = bytes;
  st.dev = user;
  st.host = user && is_host_pointer(user);
  if (!st.host) return;
  st.dev = buf + *at;
  *at += (bytes + 255) & ~(size_t)255;
}

int copy_back(Staged& st, cudaStream_t stream) {
  if (st.host) SWR_CUDA(cudaMemcpyAsync(st.user, st.dev, st.bytes, cudaMemcpyDeviceToHost, stream));
  return SWR_OK;
}

int render_impl(swr_scene* s, const swr_camera* cam, const swr_rt_opts* opts, float* rgb, uchar4* rgba,
                cudaStream_t stream) {
  RtFrame F;
  std::memcpy(F.vi, cam->view_inv, sizeof(F.vi));
  std::memcpy(F.pi, cam->proj_inv, sizeof(F.pi));
  F.W = opts->width;
  F.H = opts->height;
  F.vj = opts->vision_jumps;
  F.spp = opts->spp;
  F.refill = opts->refill ? opts->refill : 4u;
  F.shade_batch = opts->shade_batch ? opts->shade_batch : 12u;
  F.scale = (2.0f * rt::kPi) / (float)opts->spp;
  F.rgb = rgb;
  F.rgba = rgba;
  unsigned long long* cursor = (unsigned long long*)s->d_scratch;
  SWR_CUDA(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), stream));
  auto kern = k_rt_path<0>;
  if (opts->blocks_per_sm == 5) kern = k_rt_path<5>;
  else if (opts->blocks_per_sm == 6) kern = k_rt_path<6>;
  int per_sm = 0;
  SWR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, 0));
  per_sm = std::max(per_sm, 1);
  const uint64_t npix = (uint64_t)F.W * F.H;
  const uint64_t need = (npix + kBlock - 1) / kBlock;
  const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)s->num_sms * per_sm, need));
  kern<<<grid, kBlock, 0, stream>>>(s->dev, F, cursor);
  SWR_CUDA(cudaGetLastError());
  return SWR_OK;
}

int check_render_args(const swr_scene* s, const swr_camera* cam, const swr_rt_opts* opts) {
  if (!s || !cam || !opts) return set_error(SWR_ERR_INVALID, "swr: null argument");
  int rc = check_image(opts->width, opts->height);
  if (rc) return rc;
  if (opts->spp == 0 || opts->spp > kMaxSpp)
    return set_error(SWR_ERR_INVALID, "swr: visionRayPerPixelCount must be in 1..2^24");
  if (opts->vision_jumps > kMaxJumps) return set_error(SWR_ERR_INVALID, "swr: visionJumpCount above 65536");
  if (opts->refill > 32) return set_error(SWR_ERR_INVALID, "swr: refill must be 0..32");
  if (opts->shade_batch > 32) return set_error(SWR_ERR_INVALID, "swr: shade_batch must be 0..32");
  if (opts->blocks_per_sm != 0 && opts->blocks_per_sm != 5 && opts->blocks_per_sm != 6)
    return set_error(SWR_ERR_INVALID, "swr: blocks_per_sm must be 0, 5 or 6");
  return SWR_OK;
}

int gauss_args(uint32_t W, uint32_t H, uint32_t k, float sigma, GaussArgs& A) {
  std::memset(&A, 0, sizeof(A));
  int rc = swr_rt_gauss_weights(k, sigma, A.g);
  if (rc) return rc;
  A.off = (int)(k / 2);
  A.W = W;
  A.H = H;
  return SWR_OK;
}

void launch_gauss(const uchar4* in, uchar4* out, const GaussArgs& A, cudaStream_t stream) {
  const dim3 blk(kDx, kDy), grd((A.W + kDx - 1) / kDx, (A.H + kDy - 1) / kDy);
  k_rt_gauss<<<grd, blk, 0, stream>>>(in, out, A);
}

void launch_median(const uchar4* in, uchar4* out, uint32_t W, uint32_t H, cudaStream_t stream) {
  const dim3 blk(kDx, kDy), grd((W + kDx - 1) / kDx, (H + kDy - 1) / kDy);
  k_rt_median<<<grd, blk, 0, stream>>>((const uint32_t*)in, (uint32_t*)out, W, H);
}

int check_denoiser(const swr_rt_denoiser& dn) {
  if (dn.kind == SWR_DENOISER_MEDIAN) return SWR_OK;
  if (dn.kind != SWR_DENOISER_GAUSS) return set_error(SWR_ERR_INVALID, "swr: unknown denoiser kind");
  float g[kMaxGauss + 1];
  return swr_rt_gauss_weights(dn.kernel_size, dn.sigma, g);
}

}  // namespace
}  // namespace swr

using swr::set_error;

extern "C" {

int swr_rt_render(swr_scene* s, const swr_camera* cam, const swr_rt_opts* opts, float* rgb_out,
                  uint8_t* rgba8_out, void* stream_) {
  int rc = swr::check_render_args(s, cam, opts);
  if (rc) return rc;
  if (!rgb_out && !rgba8_out) return set_error(SWR_ERR_INVALID, "swr: no output buffer");
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  const size_t npix = (size_t)opts->width * opts->height;
  const size_t need = (rgb_out && swr::is_host_pointer(rgb_out) ? ((npix * 12 + 255) & ~(size_t)255) : 0) +
                      (rgba8_out && swr::is_host_pointer(rgba8_out) ? ((npix * 4 + 255) & ~(size_t)255) : 0);
  char* buf = nullptr;
  if (need && (rc = swr::rt_buffer(s, need, stream, &buf))) return rc;
  swr::Staged a, b;
  size_t at = 0;
  swr::stage_out(rgb_out, npix * 12, buf, &at, a);
  swr::stage_out(rgba8_out, npix * 4, buf, &at, b);
  rc = swr::render_impl(s, cam, opts, (float*)a.dev, (uchar4*)b.dev, stream);
  if (!rc) rc = swr::copy_back(a, stream);
  if (!rc) rc = swr::copy_back(b, stream);
  if (!rc && (a.host || b.host)) SWR_CUDA(cudaStreamSynchronize(stream));
  return rc;
}

int swr_rt_denoise_gauss(const uint8_t* in, uint8_t* out, uint32_t W, uint32_t H, uint32_t kernel_size,
                         float sigma, void* stream_) {
  if (!in || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (in == out) return set_error(SWR_ERR_INVALID, "swr: the denoisers read and write separate images");
  int rc = swr::check_image(W, H);
  if (rc) return rc;
  swr::GaussArgs A;
  if ((rc = swr::gauss_args(W, H, kernel_size, sigma, A))) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  const size_t bytes = (size_t)W * H * 4;
  swr::Staged si, so;
  if ((rc = swr::stage((void*)in, bytes, true, stream, si))) return rc;
  if ((rc = swr::stage(out, bytes, false, stream, so))) {
    swr::release(si, stream);
    return rc;
  }
  swr::launch_gauss((const uchar4*)si.dev, (uchar4*)so.dev, A, stream);
  cudaError_t e = cudaGetLastError();
  rc = e != cudaSuccess ? swr::cuda_fail(e, "k_rt_gauss") : swr::copy_back(so, stream);
  swr::release(si, stream);
  swr::release(so, stream);
  if (!rc && (si.host || so.host)) SWR_CUDA(cudaStreamSynchronize(stream));
  return rc;
}

int swr_rt_denoise_median(const uint8_t* in, uint8_t* out, uint32_t W, uint32_t H, void* stream_) {
  if (!in || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (in == out) return set_error(SWR_ERR_INVALID, "swr: the denoisers read and write separate images");
  int rc = swr::check_image(W, H);
  if (rc) return rc;
  if (((uintptr_t)in | (uintptr_t)out) & 3) return set_error(SWR_ERR_INVALID, "swr: images must be 4-byte aligned");
  cudaStream_t stream = (cudaStream_t)stream_;
  const size_t bytes = (size_t)W * H * 4;
  swr::Staged si, so;
  if ((rc = swr::stage((void*)in, bytes, true, stream, si))) return rc;
  if ((rc = swr::stage(out, bytes, false, stream, so))) {
    swr::release(si, stream);
    return rc;
  }
  swr::launch_median((const uchar4*)si.dev, (uchar4*)so.dev, W, H, stream);
  cudaError_t e = cudaGetLastError();
  rc = e != cudaSuccess ? swr::cuda_fail(e, "k_rt_median") : swr::copy_back(so, stream);
  swr::release(si, stream);
  swr::release(so, stream);
  if (!rc && (si.host || so.host)) SWR_CUDA(cudaStreamSynchronize(stream));
  return rc;
}

int swr_rt_render_frame(swr_scene* s, const swr_camera* cam, const swr_rt_opts* opts,
                        const swr_rt_denoiser* denoisers, uint32_t num_denoisers, uint8_t* rgba8_out,
                        void* stream_) {
  int rc = swr::check_render_args(s, cam, opts);
  if (rc) return rc;
  if (!rgba8_out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (num_denoisers > SWR_RT_MAX_DENOISERS) return set_error(SWR_ERR_INVALID, "swr: too many denoisers");
  if (num_denoisers && !denoisers) return set_error(SWR_ERR_INVALID, "swr: null denoiser list");
  for (uint32_t k = 0; k < num_denoisers; ++k)
    if ((rc = swr::check_denoiser(denoisers[k]))) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  SWR_CUDA(cudaSetDevice(s->device));
  const uint32_t W = opts->width, H = opts->height;
  const size_t bytes = (size_t)W * H * 4;
  const size_t slot = (bytes + 255) & ~(size_t)255;
  // ping-pong images: the renderer writes the first denoiser's input, the last denoiser the output
  const int ntmp = num_denoisers == 0 ? 0 : (num_denoisers == 1 ? 1 : 2);
  const size_t need = (size_t)ntmp * slot + (swr::is_host_pointer(rgba8_out) ? slot : 0);
  char* buf = nullptr;
  if (need && (rc = swr::rt_buffer(s, need, stream, &buf))) return rc;
  void* tmp[2] = {nullptr, nullptr};
  for (int k = 0; k < ntmp; ++k) tmp[k] = buf + (size_t)k * slot;
  swr::Staged so;
  size_t at = (size_t)ntmp * slot;
  swr::stage_out(rgba8_out, bytes, buf, &at, so);
  uchar4* cur = num_denoisers ? (uchar4*)tmp[0] : (uchar4*)so.dev;
  if (!rc) rc = swr::render_impl(s, cam, opts, nullptr, cur, stream);
  for (uint32_t k = 0; k < num_denoisers && !rc; ++k) {
    uchar4* dst = (k + 1 == num_denoisers) ? (uchar4*)so.dev : (uchar4*)tmp[(k + 1) & 1];
    if (denoisers[k].kind == SWR_DENOISER_GAUSS) {
      swr::GaussArgs A;
      rc = swr::gauss_args(W, H, denoisers[k].kernel_size, denoisers[k].sigma, A);
      if (!rc) swr::launch_gauss(cur, dst, A, stream);
    } else {
      swr::launch_median(cur, dst, W, H, stream);
    }
    cudaError_t e = cudaGetLastError();
    if (!rc && e != cudaSuccess) rc = swr::cuda_fail(e, "denoiser launch");
    cur = dst;
  }
  if (!rc) rc = swr::copy_back(so, stream);
  if (!rc && so.host) SWR_CUDA(cudaStreamSynchronize(stream));
  return rc;
}

}  // extern "C"
