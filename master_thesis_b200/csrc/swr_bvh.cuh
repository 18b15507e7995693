// Compressed 8-wide BVH and the closest-hit traversal with the reference's hit semantics.
//
// Node record: 80 bytes = five float4, 16-byte aligned (every node touches exactly three 32-byte
// sectors). Child boxes are quantised to 8 bits per plane on a per-node power-of-two grid
// (after Ylitie, Karras, Laine, "Efficient Incoherent Ray Traversal on GPUs Through Compressed
// Wide BVHs", HPG 2017); the encoding details below are this project's own.
//
//   f4[0] = p.x p.y p.z | ex | ey<<8 | ez<<16 | imask<<24     grid origin, exponents, inner mask
//   f4[1] = child_base | tri_base | meta[0..3] | meta[4..7]    meta = (count<<5)|offset for leaf
//                                                               slots, 0 for inner/empty slots
//   f4[2] = qlo_x[0..7] | qlo_y[0..7]
//   f4[3] = qlo_z[0..7] | qhi_x[0..7]
//   f4[4] = qhi_y[0..7] | qhi_z[0..7]
//
// Inner children of a node are stored contiguously from child_base in increasing slot order;
// triangles of its leaf children contiguously from tri_base (at most 24 per node, at most 3 per
// leaf). The builder places children so that slot s holds the child lying towards octant corner s;
// a ray whose direction has sign bits `oct` visits slots in increasing (s ^ oct), near to far.
//
// Triangle record: 48 bytes = three float4:
//   v0.x v0.y v0.z e0.x | e0.y e0.z e1.x e1.y | e1.z id rank obj
// where e0 = v1 - v0, e1 = v2 - v0 exactly as the reference's Triangle computes them, id is the
// global triangle id, rank its position in the reference's visit order (ties), obj its object.
//
// Hit rule (what makes the result bit-identical to Scene::traceRay, scene.cpp:22-56): the
// reference tests every triangle whose own box and whose object's box pass its slab test, with
// its Moller-Trumbore arithmetic, and keeps the smallest squared distance, the first in its
// visit order on ties. Here candidates come from the wide BVH (boxes conservatively enlarged,
// nodes farther than the current best times (1 + 2^-10) pruned); a candidate that would beat
// the current best by (distance^2, rank) is accepted only if both reference slab tests pass.
#pragma once

#include "swr_exact.cuh"

namespace swrx {

constexpr int kNodeF4 = 5;
constexpr int kTriF4 = 3;
constexpr int kStackShared = 8;   // entries per thread kept in shared memory
constexpr int kStackTotal = 64;   // maximum traversal stack depth (checked at build time)
constexpr float kPruneSlack = 1.0f + 1.0f / 1024.0f;

// Hit rules of Traversal::step.
//   kRuleReference  the software renderer's: smallest (squared distance, visit rank), accepted only
//                   when the reference's slab tests pass (see above).
//   kRuleRayQuery   the closest hit that the Vulkan renderers ask the ray tracing pipeline for
//                   (traceRay, v1.glsl:148-161: opaque geometry, tmin 0.001, tmax 10000): the
//                   smallest t in [kRqTmin, kRqTmax], ties to the lower triangle id, with the same
//                   Moller-Trumbore arithmetic; hit.rank then holds the triangle id and hit.d2 is
//                   left unset.
enum HitRule : int { kRuleReference = 0, kRuleRayQuery = 1 };
constexpr float kRqTmin = 0.001f;
constexpr float kRqTmax = 10000.0f;

struct Hit {
  uint32_t slot;   // index into the triangle records, 0xFFFFFFFF on a miss
  uint32_t id;     // global triangle id
  uint32_t rank;
  uint32_t obj;
  float t;
  float d2;
};

// What the traversal carries while it runs (id and object are read from the record at the end).
struct BestHit {
  uint32_t slot;
  uint32_t rank;
  float t;
  float d2;
};

struct TraceStats {
  uint32_t nodes;
  uint32_t tris;
};

// Stack of groups; the first kStackShared entries live in `shared` with the given stride
// (entry-major, thread-minor layout), the rest in thread-local memory. Node groups and postponed
// triangle groups share it; triangle groups carry kTriGroup in .x.
constexpr uint32_t kTriGroup = 0x80000000u;

struct GroupStack {
#if defined(__CUDA_ARCH__)
  uint32_t sbase;  // shared-memory address of this thread's entry 0
  uint32_t sstride;  // bytes between consecutive entries
#else
  uint2* shared;
  int stride;
#endif
  int sp;
  uint2 local[kStackTotal - kStackShared];
  SWR_HD void bind(uint2* p, int stride_entries) {
#if defined(__CUDA_ARCH__)
    sbase = (uint32_t)__cvta_generic_to_shared(p);
    sstride = (uint32_t)stride_entries * (uint32_t)sizeof(uint2);
#else
    shared = p;
    stride = stride_entries;
#endif
    sp = 0;
  }
  SWR_HD void push(uint2 v) {
    if (sp < kStackShared) {
#if defined(__CUDA_ARCH__)
      asm volatile("st.shared.v2.u32 [%0], {%1, %2};" ::"r"(sbase + (uint32_t)sp * sstride), "r"(v.x), "r"(v.y)
                   : "memory");
#else
      shared[sp * stride] = v;
#endif
    } else {
      local[sp - kStackShared] = v;
    }
    ++sp;
  }
  SWR_HD uint2 pop() {
    --sp;
    if (sp < kStackShared) {
#if defined(__CUDA_ARCH__)
      uint2 v;
      asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "r"(sbase + (uint32_t)sp * sstride)
                   : "memory");
      return v;
#else
      return shared[sp * stride];
#endif
    }
    return local[sp - kStackShared];
  }
};

SWR_HD float4 ldg4(const float4* p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}

// Byte k (0..3) of w as a float, exactly. (Measured on B200: the integer-to-float conversion is
// slightly faster here than building 2^23 + byte with a byte-permute and subtracting 2^23, since
// the traversal keeps the ALU and FMA pipes busier than the conversion pipe.)
SWR_HD float byte_f(uint32_t w, int k) { return (float)((w >> (8 * k)) & 0xFFu); }

// max / min of three floats, NaN operands ignored as by fmaxf / fminf
SWR_HD float fmax3(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fmaxf(fmaxf(a, b), c);
#endif
}
SWR_HD float fmin3(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fminf(fminf(a, b), c);
#endif
}

// All ones when a <= b, else zero (false for NaN operands, as the comparison itself).
SWR_HD uint32_t le_mask(float a, float b) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm("set.le.u32.f32 %0, %1, %2;" : "=r"(r) : "f"(a), "f"(b));
  return r;
#else
  return a <= b ? 0xFFFFFFFFu : 0u;
#endif
}

// `width` one bits starting at bit `pos` (pos < 32, width <= 8 here); zero when width is 0.
SWR_HD uint32_t bit_run(uint32_t pos, uint32_t width) {
#if defined(__CUDA_ARCH__)
  uint32_t r;
  asm("bmsk.clamp.b32 %0, %1, %2;" : "=r"(r) : "r"(pos), "r"(width));
  return r;
#else
  return ((1u << width) - 1u) << pos;
#endif
}

// An 8-bit slot mask moved into visit order: bit s goes to bit s ^ oct.
SWR_HD uint32_t slots_to_visit_order(uint32_t m, uint32_t oct) {
  if (oct & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
  if (oct & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
  if (oct & 4u) m = ((m & 0x0Fu) << 4) | ((m >> 4) & 0x0Fu);
  return m;
}

// Resumable closest-hit traversal of one ray: init() sets the ray up, each step() expands at
// most one wide node and tests the triangles of its hit leaves, and returns true once the ray is
// finished (hit holds the result). The persistent kernels keep one Traversal per lane and refill
// lanes whose ray finished; trace_closest() runs a single ray to completion.
struct Traversal {
  f3 o, d;
  float idx, idy, idz;  // traversal reciprocal (zero components replaced by a tiny value)
  uint32_t oct;
  float tprune;
  uint2 ng;  // node group: x = child_base, y = hits (bits 24..31, visit order) | imask (bits 0..7)
  uint2 tg;  // triangle group: x = base, y = hit bits 0..23
  BestHit hit;
  uint32_t any;  // occlusion query: stop at the first accepted candidate
  GroupStack st;
  uint32_t host_turn;  // host build only: drives the alternating postponing decision

  SWR_HD void init(f3 o_, f3 d_, uint2* stack_shared, int stack_stride) {
    o = o_;
    d = d_;
    host_turn = f2bits(o_.x) ^ f2bits(d_.y);
    const float tiny = 1e-20f;
    const float dx = (fabsf(d.x) < tiny) ? copysignf(tiny, d.x) : d.x;
    const float dy = (fabsf(d.y) < tiny) ? copysignf(tiny, d.y) : d.y;
    const float dz = (fabsf(d.z) < tiny) ? copysignf(tiny, d.z) : d.z;
    idx = 1.0f / dx;
    idy = 1.0f / dy;
    idz = 1.0f / dz;
    oct = (idx < 0.0f ? 1u : 0u) | (idy < 0.0f ? 2u : 0u) | (idz < 0.0f ? 4u : 0u);
    hit.slot = 0xFFFFFFFFu;
    hit.rank = 0xFFFFFFFFu;
    hit.t = INFINITY;
    hit.d2 = INFINITY;
    tprune = INFINITY;
    any = 0u;
    st.bind(stack_shared, stack_stride);
    ng = make_uint2(0u, (1u << (24 + oct)) | 1u);  // the root, as inner slot 0
    tg = make_uint2(0u, 0u);
  }

  // Occlusion query (Scene::isOccluded, scene.cpp:58-83): finished at the first candidate whose
  // squared distance is <= dist2; hit.slot stays 0xFFFFFFFF when there is none. The candidate
  // rule is the closest-hit one started from a best of (dist2, no rank), whose first acceptance is
  // exactly "d2 <= dist2"; nodes beyond sqrt(dist2) (with the pruning slack) are skipped, which
  // keeps every such candidate because d is of unit length.
  SWR_HD void init_occlusion(f3 o_, f3 d_, float dist2, uint2* stack_shared, int stack_stride) {
    init(o_, d_, stack_shared, stack_stride);
    hit.d2 = dist2;
    tprune = sqrtf(dist2) * kPruneSlack;
    any = 1u;
  }

  // The finished ray's hit with its triangle id and object read from the triangle record.
  SWR_HD Hit result(const float4* __restrict__ tris) const {
    Hit h;
    h.slot = hit.slot;
    h.rank = hit.rank;
    h.t = hit.t;
    h.d2 = hit.d2;
    h.id = h.obj = 0xFFFFFFFFu;
    if (h.slot != 0xFFFFFFFFu) {
      const float4 c = ldg4(tris + (size_t)h.slot * kTriF4 + 2);
      h.id = f2bits(c.y);
      h.obj = f2bits(c.w);
    }
    return h;
  }

  // kPostpone: triangle postponing. While fewer than a fifth of the warp's active lanes have
  // triangles to test, a lane that could still expand nodes parks its triangle group on its
  // stack, so the warp runs one phase at a time. Without it a lane with pending triangles tests
  // one of them per step and a lane without expands a node. (The visit order never changes the
  // result: the closest hit is an arg-min over the same candidates.)
  template <bool kStats, bool kPostpone = false, int kRule = kRuleReference>
  SWR_HD bool step(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                   const float* __restrict__ tri_boxes, const float* __restrict__ obj_boxes,
                   TraceStats* stats) {
    const bool has_nodes = (ng.y & 0xFF000000u) != 0;
    bool tri_now = tg.y != 0;
    if (kPostpone) {
#if defined(__CUDA_ARCH__)
      const unsigned act = __activemask();
      const unsigned with_tris = __ballot_sync(act, tg.y != 0);
      tri_now = tri_now && (!has_nodes || __popc(with_tris) * 5 >= __popc(act));
#else
      // host build: alternate the decision deterministically so both paths are exercised
      tri_now = tri_now && (!has_nodes || ((host_turn++ * 2654435761u) >> 31) != 0);
#endif
    }
    if (!tri_now && has_nodes) {
      if (tg.y) {
        st.push(make_uint2(tg.x | kTriGroup, tg.y));
        tg.y = 0;
      }
      const uint32_t k = (uint32_t)ffs(ng.y >> 24) - 1u;
      ng.y &= ~(1u << (24 + k));
      const uint32_t slot = k ^ oct;
      const uint32_t child = ng.x + (uint32_t)popc(ng.y & ((1u << slot) - 1u) & 0xFFu);
      if (ng.y & 0xFF000000u) st.push(ng);
      if (kStats) stats->nodes++;

      const float4* np = nodes + (size_t)child * kNodeF4;
      const float4 n0 = ldg4(np + 0), n1 = ldg4(np + 1), n2 = ldg4(np + 2);
      const float4 n3 = ldg4(np + 3), n4 = ldg4(np + 4);
      const uint32_t hdr = f2bits(n0.w);
      const float ex = bits2f((hdr & 0xFFu) << 23);
      const float ey = bits2f(((hdr >> 8) & 0xFFu) << 23);
      const float ez = bits2f(((hdr >> 16) & 0xFFu) << 23);
      const uint32_t imask = hdr >> 24;
      const float ax = ex * idx, ay = ey * idy, az = ez * idz;
      const float bx = (n0.x - o.x) * idx, by = (n0.y - o.y) * idy, bz = (n0.z - o.z) * idz;
      // near/far plane bytes by direction sign
      const uint32_t lox0 = f2bits(n2.x), lox1 = f2bits(n2.y), loy0 = f2bits(n2.z), loy1 = f2bits(n2.w);
      const uint32_t loz0 = f2bits(n3.x), loz1 = f2bits(n3.y), hix0 = f2bits(n3.z), hix1 = f2bits(n3.w);
      const uint32_t hiy0 = f2bits(n4.x), hiy1 = f2bits(n4.y), hiz0 = f2bits(n4.z), hiz1 = f2bits(n4.w);
      const uint32_t nx0 = (oct & 1u) ? hix0 : lox0, nx1 = (oct & 1u) ? hix1 : lox1;
      const uint32_t fx0 = (oct & 1u) ? lox0 : hix0, fx1 = (oct & 1u) ? lox1 : hix1;
      const uint32_t ny0 = (oct & 2u) ? hiy0 : loy0, ny1 = (oct & 2u) ? hiy1 : loy1;
      const uint32_t fy0 = (oct & 2u) ? loy0 : hiy0, fy1 = (oct & 2u) ? loy1 : hiy1;
      const uint32_t nz0 = (oct & 4u) ? hiz0 : loz0, nz1 = (oct & 4u) ? hiz1 : loz1;
      const uint32_t fz0 = (oct & 4u) ? loz0 : hiz0, fz1 = (oct & 4u) ? loz1 : hiz1;
      const uint32_t meta0 = f2bits(n1.z), meta1 = f2bits(n1.w);
      // Branch-free child loop: each slot's box test gives an all-ones or zero mask that selects
      // its bit in the slot mask and its run of triangle bits (an inner or empty slot's meta byte
      // is 0, so its run is empty). Measured on bounce rays of the terrain scene: 9 % faster than
      // branching per slot, and 56 instead of 64 registers (9 resident blocks per SM instead of 8).
      uint32_t hm = 0, trih = 0;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const uint32_t mw = i < 4 ? meta0 : meta1;
        const uint32_t pos = (mw >> ((i & 3) * 8)) & 31u;
        const uint32_t cnt = (mw >> ((i & 3) * 8 + 5)) & 7u;
        const float qnx = byte_f(i < 4 ? nx0 : nx1, i & 3);
        const float qny = byte_f(i < 4 ? ny0 : ny1, i & 3);
        const float qnz = byte_f(i < 4 ? nz0 : nz1, i & 3);
        const float qfx = byte_f(i < 4 ? fx0 : fx1, i & 3);
        const float qfy = byte_f(i < 4 ? fy0 : fy1, i & 3);
        const float qfz = byte_f(i < 4 ? fz0 : fz1, i & 3);
        const float tnx = fmaf(qnx, ax, bx), tny = fmaf(qny, ay, by), tnz = fmaf(qnz, az, bz);
        const float tfx = fmaf(qfx, ax, bx), tfy = fmaf(qfy, ay, by), tfz = fmaf(qfz, az, bz);
        const float tn = fmax3(tnx, tny, fmaxf(tnz, 0.0f));
        const float tf = fmin3(tfx, tfy, fminf(tfz, tprune));
        const uint32_t ok = le_mask(tn, tf);
        hm |= ok & (1u << i);
        trih |= ok & bit_run(pos, cnt);
      }
      const uint32_t inner = slots_to_visit_order(hm & imask, oct);
      ng = make_uint2(f2bits(n1.x), (inner << 24) | imask);
      tg = make_uint2(f2bits(n1.y), trih);
      if (kPostpone) return false;
      tri_now = true;
    }

    // At most one triangle per step: a lane with many candidate triangles then holds the warp
    // for one test per step while the other lanes go on expanding nodes (measured on the
    // terrain workload: 24.5 ms per image against 28.4 ms when a step tests all of them).
    do {
      if (!(tri_now && tg.y)) break;
      const uint32_t j = (uint32_t)ffs(tg.y) - 1u;
      tg.y &= tg.y - 1u;
      const uint32_t s = tg.x + j;
      if (kStats) stats->tris++;
      const float4* tp = tris + (size_t)s * kTriF4;
      const float4 a = ldg4(tp + 0), b = ldg4(tp + 1), c = ldg4(tp + 2);
      float t, d2;
      if (!ref_intersect(o, d, mk(a.x, a.y, a.z), mk(a.w, b.x, b.y), mk(b.z, b.w, c.x), t, d2)) break;
      if (kRule == kRuleRayQuery) {
        if (!(t >= kRqTmin && t <= kRqTmax)) break;
        const uint32_t id = f2bits(c.y);
        if (!(t < hit.t || (t == hit.t && id < hit.rank))) break;
        hit.slot = s;
        hit.rank = id;
        hit.t = t;
        tprune = t * kPruneSlack;
        break;
      }
      const uint32_t rank = f2bits(c.z);
      if (!(d2 < hit.d2 || (d2 == hit.d2 && rank < hit.rank))) break;
      const uint32_t obj = f2bits(c.w);
      const f3 inv = vinv(d);  // exact reciprocal of the reference's slab tests
      if (!ref_slab(tri_boxes + (size_t)s * 6, tri_boxes + (size_t)s * 6 + 3, o, inv)) break;
      if (!ref_slab(obj_boxes + (size_t)obj * 6, obj_boxes + (size_t)obj * 6 + 3, o, inv)) break;
      hit.slot = s;
      hit.rank = rank;
      hit.t = t;
      hit.d2 = d2;
      tprune = t * kPruneSlack;
      if (any) {  // occluded: drop the remaining work so the pop below ends the query
        ng.y = 0u;
        tg.y = 0u;
        st.sp = 0;
      }
    } while (false);

    if (!(ng.y & 0xFF000000u) && tg.y == 0) {
      if (st.sp == 0) return true;
      const uint2 g = st.pop();
      if (g.x & kTriGroup) tg = make_uint2(g.x & ~kTriGroup, g.y);
      else ng = g;
    }
    return false;
  }
};

// Closest hit of ray (o, d), run to completion. obj_boxes/tri_boxes hold the reference's own
// boxes (lo.xyz, hi.xyz) per object and per triangle record. Returns false on a miss.
template <bool kStats, bool kPostpone = false, int kRule = kRuleReference>
SWR_HD bool trace_closest(const float4* __restrict__ nodes, const float4* __restrict__ tris,
                          const float* __restrict__ tri_boxes, const float* __restrict__ obj_boxes,
                          f3 o, f3 d, uint2* stack_shared, int stack_stride, Hit& hit,
                          TraceStats* stats) {
  Traversal tr;
  tr.init(o, d, stack_shared, stack_stride);
  while (!tr.template step<kStats, kPostpone, kRule>(nodes, tris, tri_boxes, obj_boxes, stats)) {
  }
  hit = tr.result(tris);
  return hit.slot != 0xFFFFFFFFu;
}

}  // namespace swrx
