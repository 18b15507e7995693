// Exact-rounding arithmetic shared by the CUDA kernels and their host-side twins.
//
// The parity claims (bit-exact closest-hit ids, matching radiance) rest on every float operation
// of the reference's intersection and shading path being performed once, in the same order, with
// round-to-nearest and no multiply-add fusion. On the device that is what the __f*_rn / __d*_rn
// intrinsics guarantee (they are never contracted into FMAs); on the host the same functions
// compile to plain SSE operations, which requires building host code with -ffp-contract=off.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#if defined(__CUDACC__)
#define SWR_HD __host__ __device__ __forceinline__
#else
#define SWR_HD inline
#endif

namespace swrx {

#if defined(__CUDA_ARCH__)
SWR_HD float fmul(float a, float b) { return __fmul_rn(a, b); }
SWR_HD float fadd(float a, float b) { return __fadd_rn(a, b); }
SWR_HD float fsub(float a, float b) { return __fsub_rn(a, b); }
SWR_HD float fdiv(float a, float b) { return __fdiv_rn(a, b); }
SWR_HD float frcp(float a) { return __frcp_rn(a); }
SWR_HD double dmul(double a, double b) { return __dmul_rn(a, b); }
SWR_HD double dadd(double a, double b) { return __dadd_rn(a, b); }
SWR_HD double dsub(double a, double b) { return __dsub_rn(a, b); }
SWR_HD double ddiv(double a, double b) { return __ddiv_rn(a, b); }
SWR_HD double dsqrt(double a) { return __dsqrt_rn(a); }
SWR_HD float d2f(double a) { return __double2float_rn(a); }
SWR_HD float fsqrt(float a) { return __fsqrt_rn(a); }
SWR_HD int popc(uint32_t x) { return __popc(x); }
SWR_HD int ffs(uint32_t x) { return __ffs(x); }
SWR_HD uint32_t umulhi(uint32_t a, uint32_t b) { return __umulhi(a, b); }
SWR_HD float bits2f(uint32_t x) { return __uint_as_float(x); }
SWR_HD uint32_t f2bits(float x) { return __float_as_uint(x); }
#else
SWR_HD float fmul(float a, float b) { return a * b; }
SWR_HD float fadd(float a, float b) { return a + b; }
SWR_HD float fsub(float a, float b) { return a - b; }
SWR_HD float fdiv(float a, float b) { return a / b; }
SWR_HD float frcp(float a) { return 1.0f / a; }
SWR_HD double dmul(double a, double b) { return a * b; }
SWR_HD double dadd(double a, double b) { return a + b; }
SWR_HD double dsub(double a, double b) { return a - b; }
SWR_HD double ddiv(double a, double b) { return a / b; }
SWR_HD double dsqrt(double a) { return std::sqrt(a); }
SWR_HD float d2f(double a) { return (float)a; }
SWR_HD float fsqrt(float a) { return std::sqrt(a); }
SWR_HD int popc(uint32_t x) { return __builtin_popcount(x); }
SWR_HD int ffs(uint32_t x) { return __builtin_ffs((int)x); }
SWR_HD uint32_t umulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }
SWR_HD float bits2f(uint32_t x) {
  float f;
  __builtin_memcpy(&f, &x, 4);
  return f;
}
SWR_HD uint32_t f2bits(float x) {
  uint32_t u;
  __builtin_memcpy(&u, &x, 4);
  return u;
}
#endif

struct f3 {
  float x, y, z;
};
SWR_HD f3 mk(float x, float y, float z) { return f3{x, y, z}; }
SWR_HD f3 vadd(f3 a, f3 b) { return mk(fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)); }
SWR_HD f3 vsub(f3 a, f3 b) { return mk(fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)); }
SWR_HD f3 vmul(f3 a, f3 b) { return mk(fmul(a.x, b.x), fmul(a.y, b.y), fmul(a.z, b.z)); }
SWR_HD f3 vscale(float s, f3 a) { return mk(fmul(s, a.x), fmul(s, a.y), fmul(s, a.z)); }
// 0 + x0*y0 + x1*y1 + x2*y2, left to right (vector.h:235-241). The leading 0 + only turns a
// -0 first product into +0, which no caller can observe, so it is folded away.
SWR_HD float vdot(f3 a, f3 b) { return fadd(fadd(fmul(a.x, b.x), fmul(a.y, b.y)), fmul(a.z, b.z)); }
SWR_HD f3 vcross(f3 a, f3 b) {
  return mk(fsub(fmul(a.y, b.z), fmul(a.z, b.y)), fsub(fmul(a.z, b.x), fmul(a.x, b.z)),
            fsub(fmul(a.x, b.y), fmul(a.y, b.x)));
}
// normalize with double magnitude and factor (vector.h:210-225)
SWR_HD f3 vnormalize(f3 a) {
  double m = dsqrt((double)vdot(a, a));
  if (m != 0.0) {
    double f = ddiv(1.0, m);
    a.x = d2f(dmul((double)a.x, f));
    a.y = d2f(dmul((double)a.y, f));
    a.z = d2f(dmul((double)a.z, f));
  }
  return a;
}
// 1.0f / direction, component-wise IEEE division (ray.cpp:4-5)
SWR_HD f3 vinv(f3 d) { return mk(frcp(d.x), frcp(d.y), frcp(d.z)); }

// Slab test of the reference (aabb.cpp:39-53): t in [0, inf), std::min/std::max select semantics
// (the second argument never wins on NaN), hit iff tmin < tmax.
SWR_HD bool ref_slab(const float lo[3], const float hi[3], f3 o, f3 inv) {
  const float ov[3] = {o.x, o.y, o.z};
  const float iv[3] = {inv.x, inv.y, inv.z};
  float tmin = 0.0f, tmax = INFINITY;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    float t1 = fmul(fsub(lo[i], ov[i]), iv[i]);
    float t2 = fmul(fsub(hi[i], ov[i]), iv[i]);
    float mn = (t2 < t1) ? t2 : t1;
    float mx = (t1 < t2) ? t2 : t1;
    tmin = (tmin < mn) ? mn : tmin;
    tmax = (mx < tmax) ? mx : tmax;
  }
  return tmin < tmax;
}

// Moller-Trumbore of the reference (triangle.cpp:21-45) with its EPS = 1e-7 and its order of
// operations. On a hit returns t and the squared distance from the ray origin to the hit point
// computed as ray.origin.distanceSquared(origin + t*dir) (graphics_object.cpp:77).
SWR_HD bool ref_intersect(f3 o, f3 d, f3 v0, f3 e0, f3 e1, float& t_out, float& d2_out) {
  const float EPS = 0.0000001f;
  f3 h = vcross(d, e1);
  float a = vdot(e0, h);
  if (a > -EPS && a < EPS) return false;
  float f = frcp(a);
  f3 s = vsub(o, v0);
  float u = fmul(f, vdot(s, h));
  if (u < 0.0f || u > 1.0f) return false;
  f3 q = vcross(s, e0);
  float v = fmul(f, vdot(d, q));
  if (v < 0.0f || fadd(u, v) > 1.0f) return false;
  float t = fmul(f, vdot(e1, q));
  if (!(t > EPS)) return false;
  f3 p = vadd(o, vscale(t, d));
  f3 w = vsub(o, p);
  t_out = t;
  d2_out = vdot(w, w);
  return true;
}

// The barycentric weights (u of v1, v of v2) that ref_intersect computes for the same ray and
// triangle, with the same operations.
SWR_HD void ref_uv(f3 o, f3 d, f3 v0, f3 e0, f3 e1, float& u, float& v) {
  f3 h = vcross(d, e1);
  float f = frcp(vdot(e0, h));
  f3 s = vsub(o, v0);
  u = fmul(f, vdot(s, h));
  f3 q = vcross(s, e0);
  v = fmul(f, vdot(d, q));
}

// hit position as Triangle::rayIntersects computes it
SWR_HD f3 hit_point(f3 o, f3 d, float t) { return vadd(o, vscale(t, d)); }

// Barycentric coordinates (triangle.cpp:47-55)
SWR_HD f3 barycentric(f3 p, f3 v0, f3 e0, f3 e1, float d00, float d01, float d11, float denom) {
  f3 e2 = vsub(p, v0);
  float d20 = vdot(e2, e0);
  float d21 = vdot(e2, e1);
  float v = fdiv(fsub(fmul(d11, d20), fmul(d01, d21)), denom);
  float w = fdiv(fsub(fmul(d00, d21), fmul(d01, d20)), denom);
  return mk(fsub(fsub(1.0f, v), w), v, w);
}

// ------------------------------------------------------------------------------------------
// Philox-4x32-10 (Salmon et al., SC'11). Counter = (pixel, sample, vertex, stream), key = seed.
SWR_HD void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                   uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}
// top 24 bits times 2^-24: exact, in [0, 1)
SWR_HD float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

struct Uniforms {
  float u[4];
};
SWR_HD Uniforms vertex_uniforms(uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t vertex,
                                uint32_t stream) {
  uint32_t o[4];
  philox(pixel, sample, vertex, stream, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  Uniforms r;
  for (int i = 0; i < 4; ++i) r.u[i] = u01(o[i]);
  return r;
}

}  // namespace swrx
