// Per-vertex shading of the reference's PathTracer (path_tracer.cpp:42-97) and of the physical
// mode, shared by the wavefront kernels. Host-compilable for the CPU twin used in tests.
#pragma once

#include "../swr_bvh.cuh"

namespace swrx {

SWR_HD float4 ld4(const float4* p) { return ldg4(p); }

// Interpolated, normalised shading normal at hit point p of triangle slot s
// (scene.cpp:43-53: normal = 0 + b0*n0 + b1*n1 + b2*n2, then the double normalize).
SWR_HD f3 shading_normal(const float4* tris, const float4* shade, uint32_t s, f3 p) {
  const float4 a = ld4(tris + (size_t)s * 3), b = ld4(tris + (size_t)s * 3 + 1),
               c = ld4(tris + (size_t)s * 3 + 2);
  const float4 den = ld4(shade + (size_t)s * 4);
  const float4 n0 = ld4(shade + (size_t)s * 4 + 1), n1 = ld4(shade + (size_t)s * 4 + 2),
               n2 = ld4(shade + (size_t)s * 4 + 3);
  const f3 bc = barycentric(p, mk(a.x, a.y, a.z), mk(a.w, b.x, b.y), mk(b.z, b.w, c.x), den.x,
                            den.y, den.z, den.w);
  f3 n;
  n.x = fadd(fadd(fadd(0.0f, fmul(bc.x, n0.x)), fmul(bc.y, n1.x)), fmul(bc.z, n2.x));
  n.y = fadd(fadd(fadd(0.0f, fmul(bc.x, n0.y)), fmul(bc.y, n1.y)), fmul(bc.z, n2.y));
  n.z = fadd(fadd(fadd(0.0f, fmul(bc.x, n0.z)), fmul(bc.y, n1.z)), fmul(bc.z, n2.z));
  return vnormalize(n);
}

#if defined(__CUDA_ARCH__)
SWR_HD void dsincos(double x, double* s, double* c) { sincos(x, s, c); }
SWR_HD double dsin(double x) { return sin(x); }
SWR_HD double dacos(double x) { return acos(x); }
#else
SWR_HD void dsincos(double x, double* s, double* c) {
  *s = std::sin(x);
  *c = std::cos(x);
}
SWR_HD double dsin(double x) { return std::sin(x); }
SWR_HD double dacos(double x) { return std::acos(x); }
#endif

// Uniform direction on the sphere flipped into the hemisphere of n (random.cpp:16-35):
// theta = float(2*pi * u1) in double, u = 2*u2 - 1, sqrtf(1 - u*u), double sin/cos.
SWR_HD f3 hemisphere_dir(f3 n, float u1, float u2) {
  const float theta = d2f(dmul(6.283185307179586, (double)u1));
  const float u = fsub(fmul(2.0f, u2), 1.0f);
  const float suu = fsqrt(fsub(1.0f, fmul(u, u)));
  double sd, cd;
  dsincos((double)theta, &sd, &cd);
  const float st = d2f(sd), ct = d2f(cd);
  f3 v = mk(fmul(suu, ct), fmul(suu, st), u);
  if (vdot(v, n) < 0.0f) v = mk(-v.x, -v.y, -v.z);
  return v;
}

// reflect(I, N) = I - (2.0 * (N.I)) * N with the scalar in double (vector.h:319-322)
SWR_HD f3 reflect_ref(f3 I, f3 N) {
  const double s = dmul(2.0, (double)vdot(N, I));
  return mk(fsub(I.x, d2f(dmul(s, (double)N.x))), fsub(I.y, d2f(dmul(s, (double)N.y))),
            fsub(I.z, d2f(dmul(s, (double)N.z))));
}

// refract(I, N, eta) (vector.h:324-330): k in double then stored to float, sqrt in double
SWR_HD f3 refract_ref(f3 I, f3 N, float eta) {
  const float ndi = vdot(N, I);
  const double inner = dsub(1.0, (double)fmul(ndi, ndi));
  const float k = d2f(dsub(1.0, dmul((double)fmul(eta, eta), inner)));
  if ((double)k < 0.0) return mk(0.0f, 0.0f, 0.0f);
  const double s = dadd((double)fmul(eta, ndi), dsqrt((double)k));
  return mk(fsub(fmul(eta, I.x), d2f(dmul(s, (double)N.x))), fsub(fmul(eta, I.y), d2f(dmul(s, (double)N.y))),
            fsub(fmul(eta, I.z), d2f(dmul(s, (double)N.z))));
}

// customRefract (vector.h:332-345): flip N and keep eta when leaving, else eta = 1/eta (in
// double); angle = sin(acos(N.I)) * eta in double, stored to float; refract when |angle| < 1
SWR_HD f3 custom_refract_ref(f3 I, f3 N, float eta) {
  if ((double)vdot(N, I) > 0.0) {
    N = mk(-N.x, -N.y, -N.z);
  } else {
    eta = d2f(ddiv(1.0, (double)eta));
  }
  const float angle = d2f(dmul(dsin(dacos((double)vdot(N, I))), (double)eta));
  if (-1.0 < (double)angle && (double)angle < 1.0) return refract_ref(I, N, eta);
  return reflect_ref(I, N);
}

// Material record: m0 = (color.rgb, diffuse_t), m1 = (reflect_t, transparent_t, eta, light),
// m2 = (Le.rgb, strength)
struct Material {
  float4 m0, m1, m2;
};
SWR_HD Material load_material(const float4* mats, uint32_t obj) {
  Material m;
  m.m0 = ld4(mats + (size_t)obj * 3);
  m.m1 = ld4(mats + (size_t)obj * 3 + 1);
  m.m2 = ld4(mats + (size_t)obj * 3 + 2);
  return m;
}

struct PathState {
  f3 o, d;     // ray of the segment that produced this hit
  f3 c;        // throughput (reference: the cumulativeColor)
  f3 L;        // physical mode: radiance gathered so far
  uint32_t i;  // loop index of the reference's bounce loop
  uint32_t v;  // scattering vertices so far (RNG vertex counter)
};

enum ShadeOutcome : uint32_t { kContinue = 0, kEndLight = 1, kEndDark = 2 };

struct ShadeParams {
  uint64_t seed;
  uint32_t pixel, sample;
  uint32_t depth;
  uint32_t mode;  // 0 reference, 1 physical
  uint32_t rr_depth;
  float rr_q;
};

// Shades the hit (slot, t) of ray (st.o, st.d); on kContinue st holds the next ray.
// Reference mode: result = st.c on kEndLight. Physical: result = st.L on either end.
SWR_HD uint32_t shade_vertex(const float4* tris, const float4* shade, const float4* mats,
                             const float* albedo, uint32_t slot, float t, const ShadeParams& P,
                             PathState& st) {
  const f3 p = hit_point(st.o, st.d, t);
  const f3 n = shading_normal(tris, shade, slot, p);
  const uint32_t obj = f2bits(ld4(tris + (size_t)slot * 3 + 2).w);
  const Material m = load_material(mats, obj);
  const f3 prev = st.d;
  if (P.mode == 0) {
    const Uniforms U = vertex_uniforms(P.seed, P.pixel, P.sample, st.v, 0);
    const float r = U.u[0];
    f3 nd = st.d;
    if (r <= m.m0.w) nd = hemisphere_dir(n, U.u[1], U.u[2]);
    else if (r <= m.m1.x) nd = reflect_ref(st.d, n);
    else if (r <= m.m1.y) nd = custom_refract_ref(st.d, n, m.m1.z);
    st.o = vadd(p, vscale(0.01f, nd));
    st.d = nd;
    if (r <= m.m0.w) {
      const float cs = vdot(n, nd);
      st.c = vmul(st.c, mk(fmul(m.m0.x, cs), fmul(m.m0.y, cs), fmul(m.m0.z, cs)));
    }
    st.v += 1;
    if (f2bits(m.m1.w) != 0u && vdot(n, prev) <= 0.0f) return kEndLight;
    st.i += 1;
    return (st.i < P.depth) ? kContinue : kEndDark;
  }
  // physical mode
  const bool front = vdot(n, prev) <= 0.0f;
  if (f2bits(m.m1.w) != 0u) {
    if (front) {
      st.L.x += st.c.x * m.m2.x;
      st.L.y += st.c.y * m.m2.y;
      st.L.z += st.c.z * m.m2.z;
    }
    return kEndLight;
  }
  const Uniforms U = vertex_uniforms(P.seed, P.pixel, P.sample, st.v, 0);
  const float r = U.u[0];
  f3 nd = st.d;
  if (r <= m.m0.w) {
    const f3 ns = front ? n : mk(-n.x, -n.y, -n.z);
    nd = hemisphere_dir(ns, U.u[1], U.u[2]);
    const float w = 2.0f * vdot(ns, nd);
    const float* a = albedo + (size_t)slot * 3;
    st.c = mk(st.c.x * a[0] * w, st.c.y * a[1] * w, st.c.z * a[2] * w);
  } else if (r <= m.m1.x) {
    nd = reflect_ref(st.d, n);
  } else if (r <= m.m1.y) {
    nd = custom_refract_ref(st.d, n, m.m1.z);
  }
  st.v += 1;
  if (P.rr_depth != 0 && st.v >= P.rr_depth) {
    if (U.u[3] >= P.rr_q) return kEndDark;
    const float inv = 1.0f / P.rr_q;
    st.c = mk(st.c.x * inv, st.c.y * inv, st.c.z * inv);
  }
  st.o = vadd(p, vscale(0.01f, nd));
  st.d = nd;
  st.i += 1;
  return (st.i < P.depth) ? kContinue : kEndDark;
}

// Physical-mode shading of one vertex for the adjoint replay: the same arithmetic as the
// physical branch of shade_vertex (so the replayed path and throughput are the primal's), plus
// what the backward sweep needs. On return: diffuse tells whether the throughput was multiplied
// by albedo * gq (gq = 2 cos / q), else only by gq (gq = 1 / q); emitter / emit_front describe an
// emitter hit (no scattering then).
struct AdjVertex {
  bool emitter, emit_front, diffuse;
  float gq;
  uint32_t obj;
};

SWR_HD uint32_t shade_physical_adj(const float4* tris, const float4* shade, const float4* mats,
                                   const float* albedo, uint32_t slot, float t, const ShadeParams& P,
                                   PathState& st, AdjVertex& av) {
  const f3 p = hit_point(st.o, st.d, t);
  const f3 n = shading_normal(tris, shade, slot, p);
  const uint32_t obj = f2bits(ld4(tris + (size_t)slot * 3 + 2).w);
  const Material m = load_material(mats, obj);
  av.obj = obj;
  av.diffuse = false;
  av.gq = 1.0f;
  const bool front = vdot(n, st.d) <= 0.0f;
  av.emitter = f2bits(m.m1.w) != 0u;
  av.emit_front = av.emitter && front;
  if (av.emitter) {
    if (front) {
      st.L.x += st.c.x * m.m2.x;
      st.L.y += st.c.y * m.m2.y;
      st.L.z += st.c.z * m.m2.z;
    }
    return kEndLight;
  }
  const Uniforms U = vertex_uniforms(P.seed, P.pixel, P.sample, st.v, 0);
  const float r = U.u[0];
  f3 nd = st.d;
  float w = 1.0f;
  if (r <= m.m0.w) {
    const f3 ns = front ? n : mk(-n.x, -n.y, -n.z);
    nd = hemisphere_dir(ns, U.u[1], U.u[2]);
    w = 2.0f * vdot(ns, nd);
    const float* a = albedo + (size_t)slot * 3;
    st.c = mk(st.c.x * a[0] * w, st.c.y * a[1] * w, st.c.z * a[2] * w);
    av.diffuse = true;
  } else if (r <= m.m1.x) {
    nd = reflect_ref(st.d, n);
  } else if (r <= m.m1.y) {
    nd = custom_refract_ref(st.d, n, m.m1.z);
  }
  st.v += 1;
  float inv = 1.0f;
  if (P.rr_depth != 0 && st.v >= P.rr_depth) {
    if (U.u[3] >= P.rr_q) return kEndDark;
    inv = 1.0f / P.rr_q;
    st.c = mk(st.c.x * inv, st.c.y * inv, st.c.z * inv);
  }
  av.gq = w * inv;
  st.o = vadd(p, vscale(0.01f, nd));
  st.d = nd;
  st.i += 1;
  return (st.i < P.depth) ? kContinue : kEndDark;
}

#ifdef __CUDACC__
// The per-path record of the adjoint replay and its backward sweep. A path that ends on an
// emitter seen from the front contributes L = c_e * Le; sweeping its vertices backwards with
// S = Le, dL/dalbedo(tri_j) = c_j * gq_j * S_{j+1} and S_j = albedo_j * gq_j * S_{j+1}; dL/dLe =
// c_e. Each term is weighted by w = dLoss/dImage(pixel) / spp and added atomically.
constexpr int kAdjMaxDepth = 16;
// Lanes of a warp with a pending hit that shade together in the adjoint kernels (the option
// shade_batch overrides it). Measured on the tessellated Cornell adjoint (512x512x32, depth 6):
// batch 1 / 4 / 8 / 12 / 16 / 24 -> 13.9 / 12.2 / 11.6 / 11.6 / 11.9 / 12.4 ms.
constexpr uint32_t kAdjointBatch = 12;

struct AdjointTape {
  uint32_t slot[kAdjMaxDepth];
  float cx[kAdjMaxDepth], cy[kAdjMaxDepth], cz[kAdjMaxDepth], gq[kAdjMaxDepth];
  uint32_t diff;
  int nv;

  __device__ __forceinline__ void reset() {
    nv = 0;
    diff = 0;
  }
  // a vertex after which the path goes on (c = throughput before the vertex)
  __device__ __forceinline__ void push(uint32_t s, f3 c, const AdjVertex& av) {
    slot[nv] = s;
    cx[nv] = c.x;
    cy[nv] = c.y;
    cz[nv] = c.z;
    gq[nv] = av.gq;
    if (av.diffuse) diff |= 1u << nv;
    ++nv;
  }
  // the path ended on the front of emitter object obj with throughput c before it
  __device__ __forceinline__ void sweep(const float4* __restrict__ tris, const float4* __restrict__ mats,
                                        const float* __restrict__ albedo, uint32_t obj, f3 c, f3 w,
                                        float* __restrict__ g_alb, float* __restrict__ g_em) const {
    atomicAdd(&g_em[3 * (size_t)obj + 0], w.x * c.x);
    atomicAdd(&g_em[3 * (size_t)obj + 1], w.y * c.y);
    atomicAdd(&g_em[3 * (size_t)obj + 2], w.z * c.z);
    const float4 le = __ldg(mats + 3 * (size_t)obj + 2);
    float sx = le.x, sy = le.y, sz = le.z;
    for (int j = nv - 1; j >= 0; --j) {
      const float g = gq[j];
      if (diff & (1u << j)) {
        const uint32_t s = slot[j];
        const uint32_t id = __float_as_uint(__ldg(tris + 3 * (size_t)s + 2).y);
        atomicAdd(&g_alb[3 * (size_t)id + 0], w.x * cx[j] * g * sx);
        atomicAdd(&g_alb[3 * (size_t)id + 1], w.y * cy[j] * g * sy);
        atomicAdd(&g_alb[3 * (size_t)id + 2], w.z * cz[j] * g * sz);
        const float* a = albedo + 3 * (size_t)s;
        sx *= a[0] * g;
        sy *= a[1] * g;
        sz *= a[2] * g;
      } else {
        sx *= g;
        sy *= g;
        sz *= g;
      }
    }
  }
};
#endif

// Primary ray through the pixel centre (path_tracer.cpp:19-23)
SWR_HD f3 primary_dir(const float* vi, const float* pi, uint32_t px, uint32_t py, uint32_t W,
                      uint32_t H) {
  const float cx = fadd((float)px, 0.5f), cy = fadd((float)py, 0.5f);
  const float ux = fdiv(cx, (float)W), uy = fdiv(cy, (float)H);
  const float dx = fsub(fmul(2.0f, ux), 1.0f), dy = fsub(fmul(2.0f, uy), 1.0f);
  // projInverse * (dx, dy, 1, 1), row-vector form ret[j] = sum_i m[i][j] v[i]
  const float v4[4] = {dx, dy, 1.0f, 1.0f};
  float r[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r[j] = fadd(r[j], fmul(pi[i * 4 + j], v4[i]));
  const f3 target = vnormalize(mk(r[0], r[1], r[2]));
  const float w4[4] = {target.x, target.y, target.z, 0.0f};
  float q[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) q[j] = fadd(q[j], fmul(vi[i * 4 + j], w4[i]));
  return vnormalize(mk(q[0], q[1], q[2]));
}

}  // namespace swrx
