// Shader arithmetic of the Vulkan application's PathTracer, restated for the CUDA kernels in
// rt.cu: the LCG random numbers (res/shader/helper.glsl:11-23), randomNormalDirection
// (helper.glsl:25-41), customRefract (helper.glsl:43-57), getVisionRay (v1.glsl:130-142), the
// closest-hit payload (v1_closesthit.rchit:9-41) and handleHit (v1.glsl:163-188).
//
// GLSL leaves the precision of division, sqrt, sin, cos, acos and normalize to the
// implementation and may fuse multiply-adds. This restatement fixes one choice, used by the CPU
// oracle as well:
//   x / y, sqrt(x)      IEEE float, round to nearest
//   sin, cos, acos      the double-precision function of the widened argument, rounded to float
//   normalize(v)        v / sqrt(dot(v, v)), each component divided
//   dot(a, b)           (a.x*b.x + a.y*b.y) + a.z*b.z
//   mat4 * vec4         column 0 * v.x + column 1 * v.y + column 2 * v.z + column 3 * v.w
// and every operation rounds once (no multiply-add fusion), in the order the shader writes it.
#pragma once

#include "shading.cuh"

namespace swrx {
namespace rt {

constexpr float kPi = 3.1415926538f;     // helper.glsl:1, a float literal
constexpr float kNormalOffset = 0.001f;  // RAY_NORMAL_OFFSET, v1.glsl:11
constexpr uint32_t kLcgA = 6237u, kLcgC = 10697u, kLcgM = 21023u;  // initRNG, helper.glsl:11-18

// initRNG(gl_LaunchIDEXT): uint arithmetic wraps modulo 2^32 as in GLSL.
SWR_HD uint32_t lcg_init(uint32_t x, uint32_t y, uint32_t z) {
  return (625u + x * 7444u + y * 1045u + z * 13336u) % kLcgM;
}
// rand(rng): the next state over m, as a float quotient (the state is below 2^24: exact as float)
SWR_HD float lcg_next(uint32_t& state) {
  state = (kLcgA * state + kLcgC) % kLcgM;
  return fdiv((float)state, (float)kLcgM);
}

SWR_HD f3 gnormalize(f3 v) {
  const float l = fsqrt(vdot(v, v));
  return mk(fdiv(v.x, l), fdiv(v.y, l), fdiv(v.z, l));
}

// reflect(I, N) = I - 2.0 * dot(N, I) * N
SWR_HD f3 greflect(f3 I, f3 N) {
  const float s = fmul(2.0f, vdot(N, I));
  return mk(fsub(I.x, fmul(s, N.x)), fsub(I.y, fmul(s, N.y)), fsub(I.z, fmul(s, N.z)));
}

// refract(I, N, eta): k = 1 - eta*eta*(1 - dot(N,I)^2); 0 if k < 0, else
// eta*I - (eta*dot(N,I) + sqrt(k))*N
SWR_HD f3 grefract(f3 I, f3 N, float eta) {
  const float ndi = vdot(N, I);
  const float k = fsub(1.0f, fmul(fmul(eta, eta), fsub(1.0f, fmul(ndi, ndi))));
  if (k < 0.0f) return mk(0.0f, 0.0f, 0.0f);
  const float s = fadd(fmul(eta, ndi), fsqrt(k));
  return mk(fsub(fmul(eta, I.x), fmul(s, N.x)), fsub(fmul(eta, I.y), fmul(s, N.y)),
            fsub(fmul(eta, I.z), fmul(s, N.z)));
}

// customRefract (helper.glsl:43-57): leaving the surface flips the normal, entering it divides
// 1 by the index; refract while sin(acos(dot(N, I))) * index lies in (-1, 1), else reflect.
SWR_HD f3 gcustom_refract(f3 d, f3 n, float eta) {
  float ndotd = vdot(n, d);
  if (ndotd > 0.0f) {
    n = mk(-n.x, -n.y, -n.z);
    ndotd = vdot(n, d);
  } else {
    eta = fdiv(1.0f, eta);
  }
  const float ac = d2f(dacos((double)ndotd));
  const float angle = fmul(d2f(dsin((double)ac)), eta);
  if (-1.0f < angle && angle < 1.0f) return grefract(d, n, eta);
  return greflect(d, n);
}

// randomNormal + randomNormalDirection (helper.glsl:25-41): theta = 2*PI*rand, u = 2*rand - 1,
// (sqrt(1-u*u) cos theta, sqrt(1-u*u) sin theta, u), negated when it faces away from n.
SWR_HD f3 grandom_normal_dir(uint32_t& rng, f3 n) {
  const float theta = fmul(fmul(2.0f, kPi), lcg_next(rng));
  const float u = fsub(fmul(2.0f, lcg_next(rng)), 1.0f);
  const float suu = fsqrt(fsub(1.0f, fmul(u, u)));
  double sd, cd;
  dsincos((double)theta, &sd, &cd);
  f3 v = mk(fmul(suu, d2f(cd)), fmul(suu, d2f(sd)), u);
  if (vdot(v, n) < 0.0f) v = mk(-v.x, -v.y, -v.z);
  return v;
}

// getVisionRay (v1.glsl:130-142) for the pixel (x, y) of a W x H launch. The matrices are the
// renderer's viewInverse / projInverse, 16 floats in column order (element [c*4 + r]).
SWR_HD void vision_ray(const float* vi, const float* pi, uint32_t x, uint32_t y, uint32_t W,
                       uint32_t H, f3& o, f3& d) {
  const float ux = fdiv(fadd((float)x, 0.5f), (float)W);
  const float uy = fdiv(fadd((float)y, 0.5f), (float)H);
  const float dx = fsub(fmul(ux, 2.0f), 1.0f), dy = fsub(fmul(uy, 2.0f), 1.0f);
  // viewInverse * vec4(0, 0, 0, 1): the zero columns add signed zeros to column 3
  o = mk(vi[12], vi[13], vi[14]);
  f3 t;
  t.x = fadd(fadd(fadd(fmul(pi[0], dx), fmul(pi[4], dy)), fmul(pi[8], 1.0f)), fmul(pi[12], 1.0f));
  t.y = fadd(fadd(fadd(fmul(pi[1], dx), fmul(pi[5], dy)), fmul(pi[9], 1.0f)), fmul(pi[13], 1.0f));
  t.z = fadd(fadd(fadd(fmul(pi[2], dx), fmul(pi[6], dy)), fmul(pi[10], 1.0f)), fmul(pi[14], 1.0f));
  t = gnormalize(t);
  f3 w;
  w.x = fadd(fadd(fadd(fmul(vi[0], t.x), fmul(vi[4], t.y)), fmul(vi[8], t.z)), fmul(vi[12], 0.0f));
  w.y = fadd(fadd(fadd(fmul(vi[1], t.x), fmul(vi[5], t.y)), fmul(vi[9], t.z)), fmul(vi[13], 0.0f));
  w.z = fadd(fadd(fadd(fmul(vi[2], t.x), fmul(vi[6], t.y)), fmul(vi[10], t.z)), fmul(vi[14], 0.0f));
  d = gnormalize(w);
}

// The closest-hit shader's payload (v1_closesthit.rchit:9-41). The hit point is the barycentric
// combination written with the edges the triangle record holds, v0 + u*e0 + v*e1 (equal to
// b0*v0 + u*v1 + v*v2 in exact arithmetic); the normal interpolates the three corner normals with
// (1 - u - v, u, v) and is normalised; light sources return color * lightStrength.
struct Payload {
  f3 pos, n, color;
  float dT, rT, tT, eta;
  uint32_t light;
};

SWR_HD Payload hit_payload(const float4* tris, const float4* shade, const float4* mats, uint32_t s,
                           f3 o, f3 d) {
  const float4 a = ld4(tris + (size_t)s * 3), b = ld4(tris + (size_t)s * 3 + 1),
               c = ld4(tris + (size_t)s * 3 + 2);
  const f3 v0 = mk(a.x, a.y, a.z), e0 = mk(a.w, b.x, b.y), e1 = mk(b.z, b.w, c.x);
  float u, v;
  ref_uv(o, d, v0, e0, e1, u, v);
  const float b0 = fsub(fsub(1.0f, u), v);
  Payload P;
  P.pos = mk(fadd(fadd(v0.x, fmul(e0.x, u)), fmul(e1.x, v)), fadd(fadd(v0.y, fmul(e0.y, u)), fmul(e1.y, v)),
             fadd(fadd(v0.z, fmul(e0.z, u)), fmul(e1.z, v)));
  const float4 n0 = ld4(shade + (size_t)s * 4 + 1), n1 = ld4(shade + (size_t)s * 4 + 2),
               n2 = ld4(shade + (size_t)s * 4 + 3);
  P.n = gnormalize(mk(fadd(fadd(fmul(n0.x, b0), fmul(n1.x, u)), fmul(n2.x, v)),
                      fadd(fadd(fmul(n0.y, b0), fmul(n1.y, u)), fmul(n2.y, v)),
                      fadd(fadd(fmul(n0.z, b0), fmul(n1.z, u)), fmul(n2.z, v))));
  const Material m = load_material(mats, f2bits(c.w));
  P.light = f2bits(m.m1.w) != 0u ? 1u : 0u;
  P.color = mk(m.m0.x, m.m0.y, m.m0.z);
  if (P.light) P.color = vscale(m.m2.w, P.color);
  P.dT = m.m0.w;
  P.rT = m.m1.x;
  P.tT = m.m1.y;
  P.eta = m.m1.z;
  return P;
}

// handleHit (v1.glsl:163-188): one draw picks diffuse (a new hemisphere direction), reflect or
// refract by the cumulative thresholds; a draw above all three keeps the direction. The new
// origin is the hit point plus direction * RAY_NORMAL_OFFSET. Returns true for DIFFUSE_VALUE,
// which is also the value of the no-branch case.
SWR_HD bool handle_hit(const Payload& P, uint32_t& rng, f3& o, f3& d) {
  const float r = lcg_next(rng);
  bool diffuse = true;
  if (r <= P.dT) {
    d = grandom_normal_dir(rng, P.n);
  } else if (r <= P.rT) {
    d = greflect(d, P.n);
    diffuse = false;
  } else if (r <= P.tT) {
    d = gcustom_refract(d, P.n, P.eta);
    diffuse = false;
  }
  o = vadd(P.pos, mk(fmul(d.x, kNormalOffset), fmul(d.y, kNormalOffset), fmul(d.z, kNormalOffset)));
  return diffuse;
}

// imageStore to an rgba8 (UNORM) image: clamp to [0, 1] (NaN to 0), times 255, round to nearest
// even.
SWR_HD uint32_t unorm8(float x) {
  const float c = fminf(fmaxf(x, 0.0f), 1.0f);
#if defined(__CUDA_ARCH__)
  return __float2uint_rn(__fmul_rn(c, 255.0f));
#else
  return (uint32_t)std::nearbyint(c * 255.0f);
#endif
}

}  // namespace rt
}  // namespace swrx
