// TEST ONLY: host build of the very traversal and shading code the CUDA kernels run
// (swr_bvh.cuh, shading.cuh), over the same packed scene records. It lets the CPU test suite check
// the wide-BVH build, the quantised traversal and the shading arithmetic against the oracle
// without a GPU. It is never part of the product library.
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../master_thesis_b200/csrc/cuda/rt_shading.cuh"
#include "../../master_thesis_b200/csrc/host/ref_bvh.h"
#include "../../master_thesis_b200/csrc/host/scene_pack.h"

namespace {

struct Twin {
  swr::PackedScene pk;
};

}  // namespace

extern "C" {

void* twin_create(const swr_scene_desc* d, const swr_build_opts* o) {
  Twin* t = new Twin();
  if (swr::pack_scene(d, o, t->pk) != SWR_OK) {
    delete t;
    return nullptr;
  }
  return t;
}

void twin_destroy(void* t) { delete (Twin*)t; }

// the product's Philox (swr_exact.cuh) for known-answer tests
void twin_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  swrx::philox(ctr[0], ctr[1], ctr[2], ctr[3], key[0], key[1], out);
}

// the product's reproduction of the reference BVH::init, as a preorder token list
// (leaf -> element index, inner node -> 0xFFFFFFFF); returns the token count
uint32_t twin_ref_tree(const float* boxes, uint32_t n, uint32_t* out) {
  std::vector<swr::Box> b(n);
  for (uint32_t i = 0; i < n; ++i) {
    b[i].empty = false;
    for (int k = 0; k < 3; ++k) {
      b[i].lo[k] = boxes[6 * i + k];
      b[i].hi[k] = boxes[6 * i + 3 + k];
    }
  }
  swr::RefTree t;
  swr::ref_bvh_leaf_order(b, &t);
  uint32_t m = 0;
  std::vector<int32_t> st{t.root};
  while (!st.empty()) {
    int32_t v = st.back();
    st.pop_back();
    if (t.left[v] < 0) {
      out[m++] = (uint32_t)v;
    } else {
      out[m++] = 0xFFFFFFFFu;
      st.push_back(t.right[v]);
      st.push_back(t.left[v]);
    }
  }
  return m;
}

// the merge sequence itself: left/right child of every node (2n - 1 entries each, -1 for
// leaves) from the build chosen by mode (0 automatic, 1 flat, 2 kd-tree indexed, 3 kd-tree indexed
// with its first queries on 4 threads)
void twin_ref_merges(const float* boxes, uint32_t n, int mode, int32_t* left, int32_t* right) {
  std::vector<swr::Box> b(n);
  for (uint32_t i = 0; i < n; ++i) {
    b[i].empty = false;
    for (int k = 0; k < 3; ++k) {
      b[i].lo[k] = boxes[6 * i + k];
      b[i].hi[k] = boxes[6 * i + 3 + k];
    }
  }
  swr::RefTree t;
  const swr::RefBuild how = mode == 1 ? swr::RefBuild::kFlat : mode >= 2 ? swr::RefBuild::kIndexed : swr::RefBuild::kAuto;
  swr::ref_bvh_leaf_order(b, &t, how, mode == 3 ? 4 : 1);
  for (size_t i = 0; i < t.left.size(); ++i) {
    left[i] = t.left[i];
    right[i] = t.right[i];
  }
}

// copies the packed wide-BVH node words (20 per node) into out (if not null); returns the count
uint32_t twin_node_words(void* t, uint32_t* out) {
  const auto& w = ((Twin*)t)->pk.nodes;
  if (out) std::memcpy(out, w.data(), w.size() * 4);
  return (uint32_t)w.size();
}

// copies the record slot -> triangle id map into out (if not null); returns the slot count
uint32_t twin_slot_ids(void* t, uint32_t* out) {
  const auto& v = ((Twin*)t)->pk.slot_to_id;
  if (out) std::memcpy(out, v.data(), v.size() * 4);
  return (uint32_t)v.size();
}

uint32_t twin_depth(void* t) { return ((Twin*)t)->pk.depth; }
uint32_t twin_nodes(void* t) { return ((Twin*)t)->pk.num_nodes; }

void twin_trace(void* tw, const float* ro, const float* rd, uint64_t n, uint32_t* tri, float* d2,
                float* tt, uint32_t* counts, int postpone) {
  const swr::PackedScene& p = ((Twin*)tw)->pk;
  uint2 stack[swrx::kStackShared];
  for (uint64_t i = 0; i < n; ++i) {
    swrx::Hit h;
    swrx::TraceStats st{0, 0};
    const swrx::f3 o = swrx::mk(ro[4 * i], ro[4 * i + 1], ro[4 * i + 2]);
    const swrx::f3 d = swrx::mk(rd[4 * i], rd[4 * i + 1], rd[4 * i + 2]);
    if (postpone)
      swrx::trace_closest<true, true>((const float4*)p.nodes.data(), p.tris.data(), p.tri_boxes.data(),
                                      p.obj_boxes.data(), o, d, stack, 1, h, &st);
    else
      swrx::trace_closest<true, false>((const float4*)p.nodes.data(), p.tris.data(), p.tri_boxes.data(),
                                       p.obj_boxes.data(), o, d, stack, 1, h, &st);
    tri[i] = h.id;
    d2[i] = h.d2;
    tt[i] = h.t;
    if (counts) {
      counts[2 * i] = st.nodes;
      counts[2 * i + 1] = st.tris;
    }
  }
}

// Reference- or physical-mode radiance per sample for pixels [p0, p1), walking each path with
// the kernels' code: camera prefix as k_camera does it, then shade_vertex / trace_closest.
void twin_render(void* tw, const swr_camera* cam, uint32_t W, uint32_t H, uint32_t spp, uint32_t depth,
                 uint64_t seed, uint32_t mode, uint32_t rr_depth, float rr_q, uint32_t p0, uint32_t p1,
                 float* per_sample) {
  const swr::PackedScene& p = ((Twin*)tw)->pk;
  const float4* nodes = (const float4*)p.nodes.data();
  uint2 stack[swrx::kStackShared];
  for (uint32_t pix = p0; pix < p1; ++pix) {
    swrx::f3 o = swrx::mk(cam->origin[0], cam->origin[1], cam->origin[2]);
    const swrx::f3 d = swrx::primary_dir(cam->view_inv, cam->proj_inv, pix % W, pix / W, W, H);
    bool alive = false;
    uint32_t first_i = 0, slot = 0;
    float t0 = 0.0f;
    for (uint32_t i = 0; i < depth; ++i) {
      swrx::Hit h;
      if (!swrx::trace_closest<false>(nodes, p.tris.data(), p.tri_boxes.data(), p.obj_boxes.data(), o, d,
                                      stack, 1, h, nullptr))
        break;
      const swrx::f3 hp = swrx::hit_point(o, d, h.t);
      const swrx::f3 n = swrx::shading_normal(p.tris.data(), p.shade.data(), h.slot, hp);
      if (swrx::vdot(n, d) > 0.0f) {
        o = swrx::vadd(hp, swrx::vscale(0.01f, d));
        continue;
      }
      alive = true;
      first_i = i;
      slot = h.slot;
      t0 = h.t;
      break;
    }
    for (uint32_t s = 0; s < spp; ++s) {
      float* out = per_sample + (((size_t)(pix - p0)) * spp + s) * 4;
      out[0] = out[1] = out[2] = 0.0f;
      out[3] = (mode == 1) ? 1.0f : 0.0f;  // physical mode: every sample reports its radiance
      if (!alive) continue;
      swrx::PathState st;
      st.o = o;
      st.d = d;
      st.c = swrx::mk(1.0f, 1.0f, 1.0f);
      st.L = swrx::mk(0.0f, 0.0f, 0.0f);
      st.i = first_i;
      st.v = 0;
      swrx::ShadeParams P{seed, pix, s, depth, mode, rr_depth, rr_q};
      uint32_t sl = slot;
      float t = t0;
      for (;;) {
        uint32_t r = swrx::shade_vertex(p.tris.data(), p.shade.data(), p.mats.data(), p.albedo.data(), sl, t, P, st);
        if (r == swrx::kEndLight) {
          if (mode == 0) {
            out[0] = st.c.x;
            out[1] = st.c.y;
            out[2] = st.c.z;
          } else {
            out[0] = st.L.x;
            out[1] = st.L.y;
            out[2] = st.L.z;
          }
          out[3] = 1.0f;
          break;
        }
        if (r == swrx::kEndDark) {
          if (mode == 1) {
            out[0] = st.L.x;
            out[1] = st.L.y;
            out[2] = st.L.z;
            out[3] = 1.0f;
          }
          break;
        }
        swrx::Hit h;
        if (!swrx::trace_closest<false>(nodes, p.tris.data(), p.tri_boxes.data(), p.obj_boxes.data(), st.o,
                                        st.d, stack, 1, h, nullptr)) {
          if (mode == 1) {
            out[0] = st.L.x;
            out[1] = st.L.y;
            out[2] = st.L.z;
            out[3] = 1.0f;
          }
          break;
        }
        sl = h.slot;
        t = h.t;
      }
    }
  }
}

// traceRay's closest hit (the ray-query rule) with the kernels' traversal code
void twin_rt_trace(void* tw, const float* ro, const float* rd, uint64_t n, uint32_t* tri, float* t) {
  const swr::PackedScene& p = ((Twin*)tw)->pk;
  uint2 stack[swrx::kStackShared];
  for (uint64_t i = 0; i < n; ++i) {
    swrx::Hit h;
    swrx::trace_closest<false, false, swrx::kRuleRayQuery>(
        (const float4*)p.nodes.data(), p.tris.data(), p.tri_boxes.data(), p.obj_boxes.data(),
        swrx::mk(ro[4 * i], ro[4 * i + 1], ro[4 * i + 2]), swrx::mk(rd[4 * i], rd[4 * i + 1], rd[4 * i + 2]), stack, 1,
        h, nullptr);
    tri[i] = h.id;
    t[i] = h.t;
  }
}

// The RayTrace PathTracer's raygen for pixels [p0, p1) with the kernels' shading code
// (rt_shading.cuh) and traversal; the control flow restates k_rt_path per pixel.
void twin_rt_render(void* tw, const swr_camera* cam, uint32_t W, uint32_t H, uint32_t vj, uint32_t spp,
                    uint32_t p0, uint32_t p1, float* rgb) {
  namespace rt = swrx::rt;
  const swr::PackedScene& p = ((Twin*)tw)->pk;
  const float4* nodes = (const float4*)p.nodes.data();
  uint2 stack[swrx::kStackShared];
  auto trace = [&](swrx::f3 o, swrx::f3 d, swrx::Hit& h) {
    return swrx::trace_closest<false, false, swrx::kRuleRayQuery>(nodes, p.tris.data(), p.tri_boxes.data(),
                                                                  p.obj_boxes.data(), o, d, stack, 1, h, nullptr);
  };
  for (uint32_t pix = p0; pix < p1; ++pix) {
    float* out = rgb + 3 * (size_t)(pix - p0);
    uint32_t rng = rt::lcg_init(pix % W, pix / W, 0u);
    swrx::f3 o, sdir;
    rt::vision_ray(cam->view_inv, cam->proj_inv, pix % W, pix / W, W, H, o, sdir);
    swrx::Hit h;
    rt::Payload def;
    bool hit = false;
    for (uint32_t c = 0; c < 4; ++c) {
      hit = trace(o, sdir, h);
      if (!hit) break;
      def = rt::hit_payload(p.tris.data(), p.shade.data(), p.mats.data(), h.slot, o, sdir);
      if (!(swrx::vdot(def.n, sdir) > 0.0f)) break;
      o = def.pos;
    }
    swrx::f3 fin = swrx::mk(0.0f, 0.0f, 0.0f);
    if (hit && def.light) {
      fin = def.color;
    } else if (hit) {
      for (uint32_t s = 0; s < spp; ++s) {
        rt::Payload cur = def;
        swrx::f3 d = sdir, col = swrx::mk(1.0f, 1.0f, 1.0f);
        for (uint32_t i = 1; i < vj; ++i) {
          if (rt::handle_hit(cur, rng, o, d)) {
            const float cs = swrx::vdot(d, cur.n);
            col = swrx::vmul(col, swrx::vscale(cs, cur.color));
          }
          if (!trace(o, d, h)) break;
          cur = rt::hit_payload(p.tris.data(), p.shade.data(), p.mats.data(), h.slot, o, d);
          if (cur.light && swrx::vdot(d, cur.n) <= 0.0f) {
            fin = swrx::vadd(fin, swrx::vmul(col, cur.color));
            break;
          }
        }
      }
      fin = swrx::vscale((2.0f * rt::kPi) / (float)spp, fin);
    }
    out[0] = fin.x;
    out[1] = fin.y;
    out[2] = fin.z;
  }
}

}  // extern "C"
