// Host-side half of the C ABI: error reporting, the file surface, derived triangle data and
// image output. No CUDA here.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <string>
#include <vector>

#include "../../../include/swr.h"
#include "capi_common.h"
#include "ref_bvh.h"
#include "surface.h"

namespace swr {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

}  // namespace swr

using swr::set_error;

struct swr_host_scene {
  swr::HostScene s;
  std::vector<swr_material> mats;
  std::vector<uint32_t> obj_first_vertex;
};

extern "C" {

const char* swr_last_error(void) { return swr::g_last_error.c_str(); }

int swr_abi_version(void) { return SWR_ABI_VERSION; }

int swr_host_scene_load(const char* scene_path, const char* basepath, swr_host_scene** out) {
  if (!scene_path || !basepath || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  try {
    std::unique_ptr<swr_host_scene> hs(new swr_host_scene());
    hs->s = swr::load_scene_file(scene_path, basepath);
    for (const auto& o : hs->s.objects) {
      swr_material m;
      for (int k = 0; k < 3; ++k) m.color[k] = o.mat.color[k];
      m.diffuse_t = o.mat.diffuse_t;
      m.reflect_t = o.mat.reflect_t;
      m.transparent_t = o.mat.transparent_t;
      m.refraction_index = o.mat.refraction_index;
      m.light_source = o.mat.light ? 1u : 0u;
      m.light_strength = o.mat.light_strength;
      hs->mats.push_back(m);
      hs->obj_first_vertex.push_back(o.first_vertex);
    }
    hs->obj_first_vertex.push_back((uint32_t)hs->s.vpos.size());
    *out = hs.release();
    return SWR_OK;
  } catch (const swr::SurfaceError& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SWR_ERR_PARSE, std::string("swr: ") + e.what());
  }
}

int swr_host_scene_desc(const swr_host_scene* hs, swr_scene_desc* d) {
  if (!hs || !d) return set_error(SWR_ERR_INVALID, "swr: null argument");
  std::memset(d, 0, sizeof(*d));
  d->num_objects = (uint32_t)hs->s.objects.size();
  d->num_vertices = (uint32_t)hs->s.vpos.size();
  d->num_triangles = (uint32_t)hs->s.num_tris();
  d->vertex_pos = hs->s.vpos.empty() ? nullptr : hs->s.vpos[0].v;
  d->vertex_normal = hs->s.vnrm.empty() ? nullptr : hs->s.vnrm[0].v;
  d->tri_vertices = hs->s.tri.data();
  d->tri_object = hs->s.tri_obj.data();
  d->tri_rank = hs->s.tri_rank.data();
  d->object_first_vertex = hs->obj_first_vertex.data();
  d->materials = hs->mats.data();
  d->tri_albedo = nullptr;
  return SWR_OK;
}

int swr_host_scene_ranks_exact(const swr_host_scene* hs) { return hs && hs->s.ranks_exact ? 1 : 0; }

void swr_host_scene_free(swr_host_scene* hs) { delete hs; }

}  // extern "C"

namespace swr {

static swr_object_transform transform_of(const Object& o) {
  swr_object_transform x;
  for (int k = 0; k < 3; ++k) {
    x.position[k] = o.position[k];
    x.scale[k] = o.scl[k];
  }
  x.rotation[0] = o.rotation.s;
  for (int k = 0; k < 3; ++k) x.rotation[1 + k] = o.rotation.v[k];
  return x;
}

void instance_source(const swr_host_scene* hs, InstanceSource& out) {
  const HostScene& s = hs->s;
  const size_t no = s.objects.size();
  std::vector<uint32_t> mesh_base(s.meshes.size(), 0);
  uint32_t nmv = 0;
  for (size_t m = 0; m < s.meshes.size(); ++m) {
    mesh_base[m] = nmv;
    nmv += (uint32_t)s.meshes[m].pos.size();
  }
  out.mesh_pos.resize((size_t)nmv * 3);
  out.mesh_nrm.resize((size_t)nmv * 3);
  for (size_t m = 0; m < s.meshes.size(); ++m)
    for (size_t i = 0; i < s.meshes[m].pos.size(); ++i)
      for (int k = 0; k < 3; ++k) {
        out.mesh_pos[3 * (mesh_base[m] + i) + k] = s.meshes[m].pos[i][k];
        out.mesh_nrm[3 * (mesh_base[m] + i) + k] = s.meshes[m].nrm[i][k];
      }
  out.vert_src.resize(s.vpos.size());
  out.vert_obj.resize(s.vpos.size());
  out.obj_first_vertex.assign(no + 1, 0);
  out.obj_first_tri.assign(no + 1, 0);
  out.local_rank.assign(s.num_tris(), 0);
  out.xf.resize(no);
  for (size_t o = 0; o < no; ++o) {
    const Object& ob = s.objects[o];
    const Mesh& m = s.meshes[ob.mesh_id];
    for (uint32_t i = 0; i < ob.num_vertices; ++i) {
      out.vert_src[ob.first_vertex + i] = mesh_base[ob.mesh_id] + i;
      out.vert_obj[ob.first_vertex + i] = (uint32_t)o;
    }
    out.obj_first_vertex[o] = ob.first_vertex;
    out.obj_first_tri[o] = ob.first_tri;
    // rank = base of the object in the scene order + position in the mesh's leaf order
    // (SceneBuilder::finish)
    for (uint32_t k = 0; k < ob.num_tris; ++k) out.local_rank[ob.first_tri + (m.dfs.empty() ? k : m.dfs[k])] = k;
    out.xf[o] = transform_of(ob);
  }
  out.obj_first_vertex[no] = (uint32_t)s.vpos.size();
  out.obj_first_tri[no] = (uint32_t)s.num_tris();
  out.scene_order_exact = no <= LoadOptions().max_exact_order;
}

void object_matrix(const swr_object_transform& xf, float out[16]) {
  Rot r;
  r.s = xf.rotation[0];
  r.v = v3(xf.rotation[1], xf.rotation[2], xf.rotation[3]);
  // M = I * S * R * T, each step a full matrix product (graphics_object.cpp:54-62)
  M4 m = M4::identity();
  m = matmul(m, scale_matrix(v3(xf.scale[0], xf.scale[1], xf.scale[2])));
  m = matmul(m, r.matrix());
  m = matmul(m, translation_matrix(v3(xf.position[0], xf.position[1], xf.position[2])));
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) out[4 * i + j] = m.m[i][j];
}

std::vector<uint32_t> object_order(const float* boxes, uint32_t n, bool exact) {
  std::vector<uint32_t> order(n);
  if (!exact) {
    for (uint32_t o = 0; o < n; ++o) order[o] = o;
    return order;
  }
  std::vector<Box> b(n);
  for (uint32_t o = 0; o < n; ++o) {
    b[o].empty = false;
    b[o].lo = v3(boxes[6 * o], boxes[6 * o + 1], boxes[6 * o + 2]);
    b[o].hi = v3(boxes[6 * o + 3], boxes[6 * o + 4], boxes[6 * o + 5]);
  }
  return ref_bvh_leaf_order(b, nullptr, RefBuild::kAuto, 0);
}

}  // namespace swr

extern "C" {

int swr_rotation_from_axis_angle(const float axis[3], float angle, float out[4]) {
  if (!axis || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  const swr::Rot r = swr::Rot::from_axis_angle(swr::v3(axis[0], axis[1], axis[2]), angle);
  out[0] = r.s;
  for (int k = 0; k < 3; ++k) out[1 + k] = r.v[k];
  return SWR_OK;
}

int swr_host_scene_transforms(const swr_host_scene* hs, swr_object_transform* out) {
  if (!hs || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  for (size_t o = 0; o < hs->s.objects.size(); ++o) out[o] = swr::transform_of(hs->s.objects[o]);
  return SWR_OK;
}

int swr_camera_load(const char* camera_path, uint32_t width, uint32_t height, uint32_t use_fov_key,
                    swr_camera* out) {
  if (!camera_path || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (width == 0 || height == 0) return set_error(SWR_ERR_INVALID, "swr: zero image size");
  try {
    swr::CameraParams c = swr::load_camera_file(camera_path);
    swr::CameraFrame f = swr::camera_frame(c, width, height, use_fov_key != 0);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        out->view_inv[i * 4 + j] = f.view_inv.m[i][j];
        out->proj_inv[i * 4 + j] = f.proj_inv.m[i][j];
      }
    for (int k = 0; k < 3; ++k) out->origin[k] = f.origin[k];
    out->reserved = 0.0f;
    return SWR_OK;
  } catch (const swr::SurfaceError& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SWR_ERR_PARSE, std::string("swr: ") + e.what());
  }
}

int swr_camera_make(const float position[3], float angle_theta, float angle_phi, float fov_deg,
                    uint32_t width, uint32_t height, swr_camera* out) {
  if (!position || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (width == 0 || height == 0) return set_error(SWR_ERR_INVALID, "swr: zero image size");
  try {
    // the same entry a .camera file produces: position(x, y, z) angle(theta, phi) [fov(deg)]
    swr::InputEntry e("Camera");
    auto str = [](float v) {
      char b[64];
      std::snprintf(b, sizeof(b), "%.9g", (double)v);
      return std::string(b);
    };
    e.insert("position", {str(position[0]), str(position[1]), str(position[2])});
    e.insert("angle", {str(angle_theta), str(angle_phi)});
    if (fov_deg > 0.0f) e.insert("fov", {str(fov_deg)});
    swr::CameraParams c = swr::parse_camera(e);
    swr::CameraFrame f = swr::camera_frame(c, width, height, fov_deg > 0.0f);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        out->view_inv[i * 4 + j] = f.view_inv.m[i][j];
        out->proj_inv[i * 4 + j] = f.proj_inv.m[i][j];
      }
    for (int k = 0; k < 3; ++k) out->origin[k] = f.origin[k];
    out->reserved = 0.0f;
    return SWR_OK;
  } catch (const std::exception& ex) {
    return set_error(SWR_ERR_INVALID, std::string("swr: ") + ex.what());
  }
}

int swr_renderer_load(const char* renderer_path, uint32_t* max_depth, uint32_t* spp) {
  if (!renderer_path) return set_error(SWR_ERR_INVALID, "swr: null argument");
  try {
    swr::RendererParams r = swr::load_renderer_file(renderer_path, false);
    if (r.name != "PathTracer")
      return set_error(SWR_ERR_UNSUPPORTED, "swr: renderer \"" + r.name + "\" is not provided");
    if (max_depth) *max_depth = r.vision_jump_count;
    if (spp) *spp = r.rays_per_pixel;
    return SWR_OK;
  } catch (const swr::SurfaceError& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SWR_ERR_PARSE, std::string("swr: ") + e.what());
  }
}

int swr_renderer_load_params(const char* renderer_path, swr_renderer_params* out) {
  if (!renderer_path || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  try {
    swr::RendererParams r = swr::load_renderer_file(renderer_path);
    std::memset(out, 0, sizeof(*out));
    out->kind = r.name == "PathTracer" ? SWR_RENDERER_PATH_TRACER : SWR_RENDERER_BIDIRECTIONAL;
    out->vision_jumps = r.vision_jump_count;
    out->light_jumps = r.light_jump_count;
    out->max_depth = r.max_depth;
    out->spp = r.rays_per_pixel;
    return SWR_OK;
  } catch (const swr::SurfaceError& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SWR_ERR_PARSE, std::string("swr: ") + e.what());
  }
}

int swr_rt_renderer_load(const char* renderer_path, swr_rt_renderer_params* out) {
  if (!renderer_path || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  try {
    swr::RtRendererParams r = swr::load_rt_renderer_file(renderer_path);
    if (r.denoisers.size() > SWR_RT_MAX_DENOISERS)
      return set_error(SWR_ERR_UNSUPPORTED, "swr: more than 8 denoisers");
    std::memset(out, 0, sizeof(*out));
    out->vision_jumps = r.vision_jump_count;
    out->spp = r.vision_rays_per_pixel;
    out->num_denoisers = (uint32_t)r.denoisers.size();
    for (size_t k = 0; k < r.denoisers.size(); ++k) {
      const bool gauss = r.denoisers[k].name == "GaussDenoiser";
      out->denoisers[k].kind = gauss ? SWR_DENOISER_GAUSS : SWR_DENOISER_MEDIAN;
      out->denoisers[k].kernel_size = r.denoisers[k].kernel_size;
      out->denoisers[k].sigma = r.denoisers[k].sigma;
    }
    return SWR_OK;
  } catch (const swr::SurfaceError& e) {
    return set_error(e.code, e.what());
  } catch (const std::exception& e) {
    return set_error(SWR_ERR_PARSE, std::string("swr: ") + e.what());
  }
}

// GaussDenoiser::updateUniforms (gauss_denoiser.cpp:31-46), in float with the same order of
// operations; exp is evaluated in double and rounded.
int swr_rt_gauss_weights(uint32_t k, float sigma, float* out) {
  if (!out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (k == 0 || k > 19 || (k & 1u) == 0)
    return set_error(SWR_ERR_INVALID, "swr: GaussDenoiser kernelSize must be odd and in 1..19");
  if (!(sigma > 0.0f) || !std::isfinite(sigma))
    return set_error(SWR_ERR_INVALID, "swr: GaussDenoiser sigma must be positive");
  float sum = 0.0f;
  for (uint32_t i = 0; i < k; ++i) {
    float a = (float)i - ((float)k - 1.0f);
    a = a * a;
    const float b = 2.0f * sigma * sigma;
    const float r = (float)std::exp((double)(-a / b));
    out[i] = r;
    sum += r;
  }
  sum = 1.0f / sum;
  for (uint32_t i = 0; i < k; ++i) out[i] *= sum;
  return SWR_OK;
}

int swr_scene_derive(const swr_scene_desc* d, float* tri_e0, float* tri_e1, float* tri_den,
                     float* tri_box, float* obj_box) {
  int rc = swr::validate_desc(d);
  if (rc) return rc;
  swr::Derived dv;
  swr::derive(*d, dv);
  const size_t nt = d->num_triangles, no = d->num_objects;
  for (size_t t = 0; t < nt; ++t) {
    for (int k = 0; k < 3; ++k) {
      if (tri_e0) tri_e0[3 * t + k] = dv.e0[t][k];
      if (tri_e1) tri_e1[3 * t + k] = dv.e1[t][k];
      if (tri_box) {
        tri_box[6 * t + k] = dv.tri_box[t].lo[k];
        tri_box[6 * t + 3 + k] = dv.tri_box[t].hi[k];
      }
    }
    if (tri_den)
      for (int k = 0; k < 4; ++k) tri_den[4 * t + k] = dv.den[t][k];
  }
  if (obj_box)
    for (size_t o = 0; o < no; ++o)
      for (int k = 0; k < 3; ++k) {
        obj_box[6 * o + k] = dv.obj_box[o].lo[k];
        obj_box[6 * o + 3 + k] = dv.obj_box[o].hi[k];
      }
  return SWR_OK;
}

int swr_quantize_rgb8(const float* rgb, uint32_t width, uint32_t height, uint8_t* out) {
  if (!rgb || !out) return set_error(SWR_ERR_INVALID, "swr: null argument");
  const size_t n = (size_t)width * height * 3;
  for (size_t i = 0; i < n; ++i) {
    // std::clamp(c, 0, 1) then truncation of c * 255.0f to a byte (graphics_engine.cpp:90-95)
    float c = rgb[i];
    c = (c < 0.0f) ? 0.0f : ((1.0f < c) ? 1.0f : c);
    out[i] = (uint8_t)(int)(c * 255.0f);
  }
  return SWR_OK;
}

int swr_write_ppm(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height) {
  if (!path || !rgb8) return set_error(SWR_ERR_INVALID, "swr: null argument");
  std::ofstream f(path, std::ios::out | std::ios::binary);
  if (!f) return set_error(SWR_ERR_IO, std::string("swr: cannot write \"") + path + "\"");
  f << "P6\n" << width << "\n" << height << "\n" << 255u << "\n";
  f.write((const char*)rgb8, (std::streamsize)width * height * 3);
  return f ? SWR_OK : set_error(SWR_ERR_IO, std::string("swr: write failed \"") + path + "\"");
}

}  // extern "C"

namespace {

// CRC-32 (ISO 3309 / ITU-T V.42 polynomial 0xEDB88320, reflected), as PNG chunks use it
uint32_t crc32_png(const uint8_t* p, size_t n, uint32_t c = 0xFFFFFFFFu) {
  static uint32_t table[256];
  static bool init = false;
  if (!init) {
    for (uint32_t i = 0; i < 256; ++i) {
      uint32_t x = i;
      for (int k = 0; k < 8; ++k) x = (x & 1u) ? (0xEDB88320u ^ (x >> 1)) : (x >> 1);
      table[i] = x;
    }
    init = true;
  }
  for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xFFu] ^ (c >> 8);
  return c;
}

void put32(std::vector<uint8_t>& v, uint32_t x) {
  v.push_back((uint8_t)(x >> 24));
  v.push_back((uint8_t)(x >> 16));
  v.push_back((uint8_t)(x >> 8));
  v.push_back((uint8_t)x);
}

void chunk(std::vector<uint8_t>& out, const char* type, const std::vector<uint8_t>& data) {
  put32(out, (uint32_t)data.size());
  const size_t start = out.size();
  out.insert(out.end(), type, type + 4);
  out.insert(out.end(), data.begin(), data.end());
  put32(out, crc32_png(out.data() + start, out.size() - start) ^ 0xFFFFFFFFu);
}

}  // namespace

extern "C" {

// PNG (RFC 2083): 8-bit RGB, filter 0 on every row, the image data as a zlib stream (RFC 1950)
// of stored deflate blocks (RFC 1951 BTYPE 00) with its Adler-32; no compression library needed.
int swr_write_png(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height) {
  if (!path || !rgb8) return set_error(SWR_ERR_INVALID, "swr: null argument");
  if (width == 0 || height == 0 || width > (1u << 24) || height > (1u << 24))
    return set_error(SWR_ERR_INVALID, "swr: bad PNG image size");
  std::vector<uint8_t> raw;
  raw.reserve((size_t)height * (1 + (size_t)width * 3));
  for (uint32_t y = 0; y < height; ++y) {
    raw.push_back(0);  // filter type None
    raw.insert(raw.end(), rgb8 + (size_t)y * width * 3, rgb8 + (size_t)(y + 1) * width * 3);
  }
  std::vector<uint8_t> z{0x78, 0x01};
  for (size_t off = 0; off < raw.size() || off == 0;) {
    const size_t n = std::min<size_t>(65535, raw.size() - off);
    const bool last = off + n >= raw.size();
    z.push_back(last ? 1 : 0);
    z.push_back((uint8_t)n);
    z.push_back((uint8_t)(n >> 8));
    z.push_back((uint8_t)~n);
    z.push_back((uint8_t)(~n >> 8));
    z.insert(z.end(), raw.begin() + off, raw.begin() + off + n);
    off += n;
    if (last) break;
  }
  uint32_t a = 1, b = 0;  // Adler-32
  for (uint8_t c : raw) {
    a = (a + c) % 65521u;
    b = (b + a) % 65521u;
  }
  put32(z, (b << 16) | a);
  std::vector<uint8_t> png{0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
  std::vector<uint8_t> ihdr;
  put32(ihdr, width);
  put32(ihdr, height);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8 bits, RGB, deflate, adaptive filters, no interlace
  chunk(png, "IHDR", ihdr);
  chunk(png, "IDAT", z);
  chunk(png, "IEND", {});
  std::ofstream f(path, std::ios::out | std::ios::binary);
  if (!f) return set_error(SWR_ERR_IO, std::string("swr: cannot write \"") + path + "\"");
  f.write((const char*)png.data(), (std::streamsize)png.size());
  return f ? SWR_OK : set_error(SWR_ERR_IO, std::string("swr: write failed \"") + path + "\"");
}

}  // extern "C"
