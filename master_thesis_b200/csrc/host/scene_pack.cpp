// Host assembly of the device scene records (see scene_pack.h).
#include "scene_pack.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>

#include "capi_common.h"
#include "wide_bvh.h"

namespace swr {

static constexpr uint32_t kMaxStack = 64;  // swrx::kStackTotal

static inline float ubits(uint32_t u) {
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

int pack_scene(const swr_scene_desc* d, const swr_build_opts* opts, PackedScene& out, bool host_bvh) {
  int rc = validate_desc(d);
  if (rc) return rc;
  Derived dv;
  derive(*d, dv);
  const uint32_t nt = d->num_triangles, no = d->num_objects;
  // Traversal boxes: the reference triangle boxes enlarged by a margin tied to the scene's
  // extent and coordinate magnitude, so that the rounding of the quantised slab tests never
  // loses a box that the reference's own slab test hits.
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
  std::vector<PrimBox> prims(nt);
  parallel_for(nt, [&](size_t t0, size_t t1) {
    for (size_t t = t0; t < t1; ++t)
      for (int k = 0; k < 3; ++k) {
        prims[t].lo[k] = dv.tri_box[t].lo[k] - eps;
        prims[t].hi[k] = dv.tri_box[t].hi[k] + eps;
      }
  });
  WideBvhOptions wo;
  if (opts) {
    if (opts->sah_bins) wo.sah_bins = opts->sah_bins;
    if (opts->max_leaf) wo.max_leaf = opts->max_leaf;
    wo.threads = opts->threads;
    if (opts->leaf_cost_pct > 400)
      return set_error(SWR_ERR_INVALID, "swr: leaf_cost_pct must be 0..400");
    if (opts->leaf_cost_pct) wo.prim_cost = opts->leaf_cost_pct / 100.0;
    if (opts->width) wo.width = opts->width;
  }
  if (wo.max_leaf > 3) return set_error(SWR_ERR_INVALID, "swr: max_leaf must be 1..3");
  if (wo.width < 2 || wo.width > 8) return set_error(SWR_ERR_INVALID, "swr: width must be 2..8");
  if (opts && opts->radius > 256) return set_error(SWR_ERR_INVALID, "swr: radius must be 0..256");
  WideBvh bvh;
  if (host_bvh) {
    bvh = build_wide_bvh(prims, wo);
    // a traversal keeps at most one node group and one postponed triangle group per level
    if (2 * bvh.depth + 2 > kMaxStack)
      return set_error(SWR_ERR_UNSUPPORTED, "swr: BVH deeper than the traversal stack");
  } else {
    bvh.prim_order.resize(nt);
    for (uint32_t t = 0; t < nt; ++t) bvh.prim_order[t] = t;
    out.prim_boxes.resize((size_t)nt * 6);
    for (uint32_t t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) {
        out.prim_boxes[6 * (size_t)t + k] = prims[t].lo[k];
        out.prim_boxes[6 * (size_t)t + 3 + k] = prims[t].hi[k];
      }
  }

  const uint32_t ns = (uint32_t)bvh.prim_order.size();
  out.nodes = std::move(bvh.words);
  out.num_nodes = bvh.num_nodes;
  out.depth = bvh.depth;
  out.tris.assign((size_t)ns * 3, make_float4(0, 0, 0, 0));
  out.shade.assign((size_t)ns * 4, make_float4(0, 0, 0, 0));
  out.tri_boxes.assign((size_t)ns * 6, 0.0f);
  out.albedo.assign((size_t)ns * 3, 0.0f);
  out.obj_boxes.assign((size_t)no * 6, 0.0f);
  out.mats.assign((size_t)no * 3, make_float4(0, 0, 0, 0));
  out.slot_of.assign(nt, 0u);
  out.slot_to_id.assign(ns, 0u);
  parallel_for(ns, [&](size_t s0, size_t s1) {
    for (uint32_t sl = (uint32_t)s0; sl < (uint32_t)s1; ++sl) {
      const uint32_t t = bvh.prim_order[sl];
      out.slot_of[t] = sl;
      out.slot_to_id[sl] = t;
      const uint32_t obj = d->tri_object[t];
      const uint32_t rank = d->tri_rank ? d->tri_rank[t] : t;
      const V3 &v0 = dv.v0[t], &e0 = dv.e0[t], &e1 = dv.e1[t];
      out.tris[3 * (size_t)sl + 0] = make_float4(v0[0], v0[1], v0[2], e0[0]);
      out.tris[3 * (size_t)sl + 1] = make_float4(e0[1], e0[2], e1[0], e1[1]);
      out.tris[3 * (size_t)sl + 2] = make_float4(e1[2], ubits(t), ubits(rank), ubits(obj));
      out.shade[4 * (size_t)sl] = make_float4(dv.den[t][0], dv.den[t][1], dv.den[t][2], dv.den[t][3]);
      for (int c = 0; c < 3; ++c) {
        const uint32_t vi = d->tri_vertices[3 * (size_t)t + c];
        const float* nv = d->vertex_normal + 3 * (size_t)vi;
        out.shade[4 * (size_t)sl + 1 + c] = make_float4(nv[0], nv[1], nv[2], 0.0f);
      }
      for (int k = 0; k < 3; ++k) {
        out.tri_boxes[6 * (size_t)sl + k] = dv.tri_box[t].lo[k];
        out.tri_boxes[6 * (size_t)sl + 3 + k] = dv.tri_box[t].hi[k];
        out.albedo[3 * (size_t)sl + k] =
            d->tri_albedo ? d->tri_albedo[3 * (size_t)t + k] : d->materials[obj].color[k];
      }
    }
  });
  {
    // triangles of each object are contiguous in id order (tri_object is non-decreasing)
    std::vector<uint32_t> first(no + 1, 0);
    for (uint32_t t = 0; t < nt; ++t) first[d->tri_object[t] + 1]++;
    for (uint32_t o = 0; o < no; ++o) first[o + 1] += first[o];
    for (uint32_t o = 0; o < no; ++o) {
      if (!d->materials[o].light_source) continue;
      const uint32_t n = first[o + 1] - first[o];
      out.lights.insert(out.lights.end(), {(uint32_t)(out.light_tris.size() / 5), n, o, 0u});
      for (uint32_t t = first[o]; t < first[o + 1]; ++t) {
        float w[20] = {0};
        for (int c = 0; c < 3; ++c) {
          const uint32_t vi = d->tri_vertices[3 * (size_t)t + c];
          for (int k = 0; k < 3; ++k) {
            w[3 * c + k] = d->vertex_pos[3 * (size_t)vi + k];
            w[9 + 3 * c + k] = d->vertex_normal[3 * (size_t)vi + k];
          }
        }
        for (int q = 0; q < 5; ++q) out.light_tris.push_back(make_float4(w[4 * q], w[4 * q + 1], w[4 * q + 2], w[4 * q + 3]));
      }
    }
  }
  for (uint32_t o = 0; o < no; ++o) {
    const swr_material& m = d->materials[o];
    for (int k = 0; k < 3; ++k) {
      out.obj_boxes[6 * (size_t)o + k] = dv.obj_box[o].lo[k];
      out.obj_boxes[6 * (size_t)o + 3 + k] = dv.obj_box[o].hi[k];
    }
    out.mats[3 * (size_t)o + 0] = make_float4(m.color[0], m.color[1], m.color[2], m.diffuse_t);
    out.mats[3 * (size_t)o + 1] = make_float4(m.reflect_t, m.transparent_t, m.refraction_index,
                                              ubits(m.light_source ? 1u : 0u));
    out.mats[3 * (size_t)o + 2] =
        make_float4(m.color[0] * m.light_strength, m.color[1] * m.light_strength,
                    m.color[2] * m.light_strength, m.light_strength);
  }
  return SWR_OK;
}

}  // namespace swr
