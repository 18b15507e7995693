// Descriptor validation and the reference-exact per-triangle / per-object derived data.
#include <string>

#include "capi_common.h"

namespace swr {

int validate_desc(const swr_scene_desc* d) {
  if (!d) return set_error(SWR_ERR_INVALID, "swr: null scene descriptor");
  if (d->num_triangles == 0 || d->num_objects == 0 || d->num_vertices == 0)
    return set_error(SWR_ERR_INVALID, "swr: empty scene (no triangles, objects or vertices)");
  if (!d->vertex_pos || !d->vertex_normal || !d->tri_vertices || !d->tri_object ||
      !d->object_first_vertex || !d->materials)
    return set_error(SWR_ERR_INVALID, "swr: scene descriptor has a null array");
  if (d->num_triangles > (1u << 27))
    return set_error(SWR_ERR_UNSUPPORTED, "swr: more than 2^27 triangles");
  if (d->object_first_vertex[0] != 0 || d->object_first_vertex[d->num_objects] != d->num_vertices)
    return set_error(SWR_ERR_INVALID, "swr: object vertex ranges do not cover the vertex array");
  for (uint32_t o = 0; o < d->num_objects; ++o)
    if (d->object_first_vertex[o + 1] <= d->object_first_vertex[o])
      return set_error(SWR_ERR_INVALID, "swr: object " + std::to_string(o) + " has no vertices");
  uint32_t prev = 0;
  for (uint32_t t = 0; t < d->num_triangles; ++t) {
    const uint32_t o = d->tri_object[t];
    if (o >= d->num_objects || o < prev)
      return set_error(SWR_ERR_INVALID, "swr: tri_object must be non-decreasing object indices");
    prev = o;
    for (int k = 0; k < 3; ++k) {
      const uint32_t v = d->tri_vertices[3 * (size_t)t + k];
      if (v < d->object_first_vertex[o] || v >= d->object_first_vertex[o + 1])
        return set_error(SWR_ERR_INVALID,
                         "swr: triangle " + std::to_string(t) + " uses a vertex of another object");
    }
  }
  for (uint32_t o = 0; o < d->num_objects; ++o) {
    const swr_material& m = d->materials[o];
    if (!(m.refraction_index > 0.0f))
      return set_error(SWR_ERR_INVALID, "swr: refraction index must be positive");
  }
  return SWR_OK;
}

void derive(const swr_scene_desc& d, Derived& out) {
  const size_t nt = d.num_triangles, no = d.num_objects;
  auto P = [&](uint32_t v) { return v3(d.vertex_pos[3 * (size_t)v], d.vertex_pos[3 * (size_t)v + 1], d.vertex_pos[3 * (size_t)v + 2]); };
  out.v0.resize(nt);
  out.e0.resize(nt);
  out.e1.resize(nt);
  out.den.resize(nt);
  out.tri_box.assign(nt, Box());
  parallel_for(nt, [&](size_t t0, size_t t1) {
    for (size_t t = t0; t < t1; ++t) {
      const V3 a = P(d.tri_vertices[3 * t]), b = P(d.tri_vertices[3 * t + 1]),
               c = P(d.tri_vertices[3 * t + 2]);
      const V3 e0 = sub(b, a), e1 = sub(c, a);
      const float d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1);
      out.v0[t] = a;
      out.e0[t] = e0;
      out.e1[t] = e1;
      out.den[t] = v4(d00, d01, d11, d00 * d11 - d01 * d01);
      out.tri_box[t].add(a);
      out.tri_box[t].add(b);
      out.tri_box[t].add(c);
    }
  });
  out.obj_box.assign(no, Box());
  parallel_for(no, [&](size_t o0, size_t o1) {
    for (size_t o = o0; o < o1; ++o)
      for (uint32_t v = d.object_first_vertex[o]; v < d.object_first_vertex[o + 1]; ++v)
        out.obj_box[o].add(P(v));
  });
}

}  // namespace swr
