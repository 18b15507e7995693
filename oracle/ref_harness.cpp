// TEST INFRASTRUCTURE ONLY. Harness around the reference's own SoftwareRenderer sources, compiled
// from the reference tree by oracle/Makefile into oracle/_ref/. It produces the pinned outputs the
// parity tests compare against:
//
//   ref_harness dump   <basepath> <scene> <camera> <W> <H> <out>
//       world-space vertices/normals/triangles/boxes/materials exactly as GraphicsObject::init
//       computed them, the leaf orders of the reference's BVHs (scene over objects, each mesh
//       over its triangles) and the camera matrices of GraphicsEngine::render.
//   ref_harness trace  <basepath> <scene> <rays> <out>
//       closest hit of Scene::traceRay for each ray (object, triangle, distance^2, hit vertex).
//   ref_harness render <basepath> <scene> <camera> <W> <H> <spp> <depth> <seed> <p0> <p1> <out>
//       PathTracer radiance for pixels [p0, p1) (row-major index), per sample and per pixel,
//       with the Philox shim cursor set to (seed, pixel, sample) before each sample.
//   ref_harness render_bdpt <basepath> <scene> <camera> <W> <H> <spp> <vision> <light> <maxdepth>
//                           <seed> <p0> <p1> <out>
//       BidirectionalPathTracer::renderPixel with one ray per pixel per call, the Philox shim
//       cursor set to (seed, pixel, sample) before each call: per-sample values (with the
//       reference's 2 pi scale for one sample).
//   ref_harness tree   <boxes> <out>
//       the reference BVH::init tree over the given boxes (for builder equivalence tests).
//
// Private members are reached by compiling the reference headers with private mapped to public;
// all standard headers are included first so the mapping only touches the reference's classes.
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <list>
#include <map>
#include <mutex>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#define private public
#include "camera.h"
#include "graphic/graphics_engine.h"
#include "graphic/bidirectional_path_tracer.h"
#include "graphic/graphics_object.h"
#include "graphic/path_tracer.h"
#include "graphic/scene.h"
#include "input_parser.h"
#include "mesh_manager.h"
#undef private

extern "C" void swr_shim_set_cursor(uint64_t seed, uint32_t pixel, uint32_t sample);

namespace {

// ---- simple tagged binary container: repeated {name[32], kind, pad[7], count u64, bytes} ----
struct Writer {
  std::ofstream f;
  explicit Writer(const std::string& p) : f(p, std::ios::binary) {
    if (!f) throw std::runtime_error("cannot write " + p);
    f.write("SWRB0001", 8);
  }
  void put(const std::string& name, char kind, const void* data, uint64_t count, size_t elem) {
    char hdr[48] = {0};
    std::strncpy(hdr, name.c_str(), 31);
    hdr[32] = kind;
    std::memcpy(hdr + 40, &count, 8);
    f.write(hdr, 48);
    f.write((const char*)data, (std::streamsize)(count * elem));
  }
  void f32(const std::string& n, const std::vector<float>& v) { put(n, 'f', v.data(), v.size(), 4); }
  void u32(const std::string& n, const std::vector<uint32_t>& v) { put(n, 'u', v.data(), v.size(), 4); }
};

std::vector<uint8_t> read_file(const std::string& p) {
  std::ifstream f(p, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read " + p);
  return std::vector<uint8_t>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

void push3(std::vector<float>& v, const Vector3f& x) {
  v.push_back(x[0]);
  v.push_back(x[1]);
  v.push_back(x[2]);
}

void leaf_order(const BVH::Node* n, std::vector<uint32_t>& out) {
  if (n->left == nullptr) {
    out.push_back((uint32_t)n->elemIndex);
    return;
  }
  leaf_order(n->left, out);
  leaf_order(n->right, out);
}

// the tree as a preorder token list: leaf -> element index, internal -> 0xFFFFFFFF
void tree_tokens(const BVH::Node* n, std::vector<uint32_t>& out) {
  if (n->left == nullptr) {
    out.push_back((uint32_t)n->elemIndex);
    return;
  }
  out.push_back(0xFFFFFFFFu);
  tree_tokens(n->left, out);
  tree_tokens(n->right, out);
}

struct Loaded {
  MeshManager* mm = nullptr;
  GraphicsEngine* engine = nullptr;
  std::vector<GraphicsObject*> objs;
};

Loaded load(const std::string& basepath, const std::string& scene) {
  Loaded L;
  L.mm = new MeshManager(basepath);
  L.mm->createObjectsFromFile(scene);
  L.engine = new GraphicsEngine();
  L.engine->imageSize = Vector2u({1, 1});
  L.engine->objects = L.mm->getCreatedObjects();
  L.engine->lightSources = L.mm->getCreatedLightSources();
  PathTracer* pt = new PathTracer();
  L.engine->init(pt, 1);
  L.objs = L.engine->objects;
  return L;
}

std::vector<uint32_t> object_tri_offsets(const Loaded& L) {
  std::vector<uint32_t> off;
  uint32_t acc = 0;
  for (auto* o : L.objs) {
    off.push_back(acc);
    acc += (uint32_t)o->triangles.size();
  }
  off.push_back(acc);
  return off;
}

int cmd_dump(char** a) {
  std::string basepath = a[0], scene = a[1], camera = a[2];
  unsigned W = (unsigned)std::atoi(a[3]), H = (unsigned)std::atoi(a[4]);
  Loaded L = load(basepath, scene);
  Writer w(a[5]);
  std::vector<float> vpos, vnrm, tv0, te0, te1, tden, tbox, obox, mat;
  std::vector<uint32_t> tidx, tobj, ofv, oft, onv, ont, olight, obox_empty, tbox_empty;
  std::vector<uint32_t> scene_order, tri_order;
  uint32_t vacc = 0;
  for (size_t oi = 0; oi < L.objs.size(); ++oi) {
    GraphicsObject* o = L.objs[oi];
    ofv.push_back(vacc);
    onv.push_back((uint32_t)o->vertices.size());
    for (auto& v : o->vertices) {
      push3(vpos, v.pos);
      push3(vnrm, v.normal);
    }
    for (auto& t : o->triangles) {
      tidx.push_back(vacc + t.indices[0]);
      tidx.push_back(vacc + t.indices[1]);
      tidx.push_back(vacc + t.indices[2]);
      tobj.push_back((uint32_t)oi);
      push3(tv0, t.v0);
      push3(te0, t.edge0);
      push3(te1, t.edge1);
      tden.push_back(t.d00);
      tden.push_back(t.d01);
      tden.push_back(t.d11);
      tden.push_back(t.denom);
      tbox_empty.push_back(t.aabb.empty ? 1u : 0u);
      push3(tbox, t.aabb.aabbMin);
      push3(tbox, t.aabb.aabbMax);
    }
    oft.push_back(0);
    ont.push_back((uint32_t)o->triangles.size());
    obox_empty.push_back(o->aabb.empty ? 1u : 0u);
    push3(obox, o->aabb.aabbMin);
    push3(obox, o->aabb.aabbMax);
    push3(mat, o->color);
    mat.push_back(o->diffuseThreshold);
    mat.push_back(o->reflectThreshold);
    mat.push_back(o->transparentThreshold);
    mat.push_back(o->refractionIndex);
    mat.push_back(o->lightStrength);
    olight.push_back(o->lightSource ? 1u : 0u);
    // mesh-BVH leaf order of this object's (refit) tree
    std::vector<uint32_t> ord;
    leaf_order(o->bvh.root, ord);
    tri_order.insert(tri_order.end(), ord.begin(), ord.end());
    vacc += (uint32_t)o->vertices.size();
  }
  {
    uint32_t acc = 0;
    for (size_t oi = 0; oi < L.objs.size(); ++oi) {
      oft[oi] = acc;
      acc += ont[oi];
    }
  }
  leaf_order(L.engine->scene.bvh.root, scene_order);

  Camera cam;
  InputParser cp(camera);
  cp.parse();
  cam.parseInput(cp.getInputEntry(0));
  Matrix4f vi = cam.getViewMatrix().inverseMatrix();
  Matrix4f pi = cam.getProjectionMatrix(float(W) / float(H)).inverseMatrix();
  Vector3f origin = cutVector(vi * Vector4f({0.0f, 0.0f, 0.0f, 1.0f}));
  std::vector<float> cam_out;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) cam_out.push_back(vi.m[i][j]);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) cam_out.push_back(pi.m[i][j]);
  push3(cam_out, origin);
  cam_out.push_back(cam.theta);
  cam_out.push_back(cam.phi);

  w.f32("vpos", vpos);
  w.f32("vnrm", vnrm);
  w.u32("tri", tidx);
  w.u32("tri_obj", tobj);
  w.f32("tri_v0", tv0);
  w.f32("tri_e0", te0);
  w.f32("tri_e1", te1);
  w.f32("tri_den", tden);
  w.f32("tri_box", tbox);
  w.u32("tri_box_empty", tbox_empty);
  w.u32("obj_first_vertex", ofv);
  w.u32("obj_num_vertices", onv);
  w.u32("obj_first_tri", oft);
  w.u32("obj_num_tris", ont);
  w.f32("obj_box", obox);
  w.u32("obj_box_empty", obox_empty);
  w.f32("obj_mat", mat);
  w.u32("obj_light", olight);
  w.u32("scene_order", scene_order);
  w.u32("tri_order", tri_order);
  w.f32("camera", cam_out);
  return 0;
}

int cmd_trace(char** a) {
  Loaded L = load(a[0], a[1]);
  std::vector<uint8_t> raw = read_file(a[2]);
  const size_t n = raw.size() / 24;
  const float* r = (const float*)raw.data();
  std::vector<uint32_t> off = object_tri_offsets(L);
  std::unordered_map<const GraphicsObject*, uint32_t> oid;
  for (size_t i = 0; i < L.objs.size(); ++i) oid[L.objs[i]] = (uint32_t)i;
  std::vector<uint32_t> hit_id(n), hit_obj(n);
  std::vector<float> hit_d2(n), hit_pos(3 * n), hit_nrm(3 * n);
  const Scene& scene = L.engine->scene;
  unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<size_t> next(0);
  auto work = [&]() {
    for (;;) {
      size_t i = next.fetch_add(1024);
      if (i >= n) break;
      size_t e = std::min(n, i + 1024);
      for (; i < e; ++i) {
        Ray ray(Vector3f({r[6 * i + 0], r[6 * i + 1], r[6 * i + 2]}),
                Vector3f({r[6 * i + 3], r[6 * i + 4], r[6 * i + 5]}));
        // Scene::traceRay's own loop, keeping the Triangle* that it discards (scene.cpp:22-41)
        std::vector<size_t> elems = scene.bvh.getHits(ray);
        float minDistance = INFINITY;
        const Triangle* tri = nullptr;
        const GraphicsObject* obj = nullptr;
        Vector3f hp;
        for (size_t e2 : elems) {
          const GraphicsObject* o = scene.objs[e2];
          if (o->traceRay(ray, hp, tri, minDistance)) obj = o;
        }
        Mesh::Vertex hv;
        const GraphicsObject* obj2 = nullptr;
        bool hit = scene.traceRay(ray, hv, obj2);
        if (hit != (obj != nullptr) || obj != obj2) {
          std::fprintf(stderr, "harness: inconsistent trace at ray %zu\n", i);
          std::abort();
        }
        if (!obj) {
          hit_id[i] = 0xFFFFFFFFu;
          hit_obj[i] = 0xFFFFFFFFu;
          hit_d2[i] = INFINITY;
          continue;
        }
        uint32_t o_i = oid[obj];
        hit_obj[i] = o_i;
        hit_id[i] = off[o_i] + (uint32_t)(tri - obj->triangles.data());
        hit_d2[i] = minDistance;
        for (int k = 0; k < 3; ++k) {
          hit_pos[3 * i + k] = hv.pos[k];
          hit_nrm[3 * i + k] = hv.normal[k];
        }
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nthreads; ++t) th.emplace_back(work);
  for (auto& t : th) t.join();
  Writer w(a[3]);
  w.u32("hit_id", hit_id);
  w.u32("hit_obj", hit_obj);
  w.f32("hit_d2", hit_d2);
  w.f32("hit_pos", hit_pos);
  w.f32("hit_nrm", hit_nrm);
  return 0;
}

int cmd_render(char** a) {
  std::string basepath = a[0], scene = a[1], camera = a[2];
  unsigned W = (unsigned)std::atoi(a[3]), H = (unsigned)std::atoi(a[4]);
  unsigned spp = (unsigned)std::atoi(a[5]), depth = (unsigned)std::atoi(a[6]);
  uint64_t seed = std::strtoull(a[7], nullptr, 10);
  uint32_t p0 = (uint32_t)std::atoi(a[8]), p1 = (uint32_t)std::atoi(a[9]);
  Loaded L = load(basepath, scene);
  PathTracer* pt = (PathTracer*)L.engine->renderer;
  pt->visionJumpCount = depth;
  pt->raysPerPixel = spp;

  Camera cam;
  InputParser cp(camera);
  cp.parse();
  cam.parseInput(cp.getInputEntry(0));
  Matrix4f vi = cam.getViewMatrix().inverseMatrix();
  Matrix4f pi = cam.getProjectionMatrix(float(W) / float(H)).inverseMatrix();
  Vector3f origin = cutVector(vi * Vector4f({0.0f, 0.0f, 0.0f, 1.0f}));

  const uint32_t np = p1 - p0;
  std::vector<float> per_sample((size_t)np * spp * 4), per_pixel((size_t)np * 3);
  std::vector<float> check((size_t)np * 3);
  unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<uint32_t> next(0);
  auto work = [&]() {
    Renderer::PixelRenderData prd;
    prd.scene = &L.engine->scene;
    prd.objects = &L.engine->objects;
    prd.lightSources = &L.engine->lightSources;
    prd.imageSize = Vector2u({W, H});
    prd.origin = origin;
    prd.viewInverse = vi;
    prd.projInverse = pi;
    std::vector<PathTracer::HitPoint> path(depth);
    for (;;) {
      uint32_t k = next.fetch_add(1);
      if (k >= np) break;
      uint32_t p = p0 + k;
      prd.pixel[0] = p % W;
      prd.pixel[1] = p / W;
      // primary ray of PathTracer::renderPixel (path_tracer.cpp:19-23)
      Vector2f pixelCenter = Vector2f({(float)prd.pixel[0], (float)prd.pixel[1]}) + Vector2f({0.5f, 0.5f});
      Vector2f inUV = Vector2f({pixelCenter[0] / (float)prd.imageSize[0], pixelCenter[1] / (float)prd.imageSize[1]});
      Vector2f d = (2.0f * inUV) - Vector2f({1.0f, 1.0f});
      Vector3f target = cutVector(prd.projInverse * Vector4f({d[0], d[1], 1.0f, 1.0f})).normalize();
      Vector3f direction = cutVector(prd.viewInverse * expandVector(target, 0.0f)).normalize();
      Vector3f finalColor({0.0f, 0.0f, 0.0f});
      Ray start(prd.origin, direction);
      for (unsigned s = 0; s < spp; ++s) {
        swr_shim_set_cursor(seed, p, s);
        size_t dp = pt->traceSinglePath(prd, path, start, 0, depth);
        float* o = &per_sample[((size_t)k * spp + s) * 4];
        o[0] = o[1] = o[2] = o[3] = 0.0f;
        if (dp == 0) continue;
        if (!path[dp - 1].lightHit) continue;
        for (int c = 0; c < 3; ++c) o[c] = path[dp - 1].cumulativeColor[c];
        o[3] = 1.0f;
        finalColor += path[dp - 1].cumulativeColor;
      }
      finalColor *= 2.0f * M_PI * (1.0f / float(spp));
      for (int c = 0; c < 3; ++c) per_pixel[(size_t)k * 3 + c] = finalColor[c];
      // self-check: with one sample, the reference's own renderPixel gives the same value
      if (spp == 1) {
        swr_shim_set_cursor(seed, p, 0);
        Vector3f ref = pt->renderPixel(prd);
        for (int c = 0; c < 3; ++c) check[(size_t)k * 3 + c] = ref[c];
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nthreads; ++t) th.emplace_back(work);
  for (auto& t : th) t.join();
  if (spp == 1 && std::memcmp(check.data(), per_pixel.data(), check.size() * 4) != 0) {
    std::fprintf(stderr, "harness: renderPixel self-check failed\n");
    return 3;
  }
  Writer w(a[10]);
  w.f32("per_sample", per_sample);
  w.f32("per_pixel", per_pixel);
  return 0;
}

int cmd_render_bdpt(char** a) {
  std::string basepath = a[0], scene = a[1], camera = a[2];
  unsigned W = (unsigned)std::atoi(a[3]), H = (unsigned)std::atoi(a[4]);
  unsigned spp = (unsigned)std::atoi(a[5]);
  unsigned vj = (unsigned)std::atoi(a[6]), lj = (unsigned)std::atoi(a[7]), md = (unsigned)std::atoi(a[8]);
  uint64_t seed = std::strtoull(a[9], nullptr, 10);
  uint32_t p0 = (uint32_t)std::atoi(a[10]), p1 = (uint32_t)std::atoi(a[11]);
  Loaded L = load(basepath, scene);
  Camera cam;
  InputParser cp(camera);
  cp.parse();
  cam.parseInput(cp.getInputEntry(0));
  Matrix4f vi = cam.getViewMatrix().inverseMatrix();
  Matrix4f pi = cam.getProjectionMatrix(float(W) / float(H)).inverseMatrix();
  Vector3f origin = cutVector(vi * Vector4f({0.0f, 0.0f, 0.0f, 1.0f}));
  const uint32_t np = p1 - p0;
  std::vector<float> per_sample((size_t)np * spp * 4);
  unsigned nthreads = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<uint32_t> next(0);
  auto work = [&]() {
    BidirectionalPathTracer bd;
    bd.visionJumpCount = vj;
    bd.lightJumpCount = lj;
    bd.maxDepth = md;
    bd.raysPerPixel = 1;
    Renderer::PixelRenderData prd;
    prd.scene = &L.engine->scene;
    prd.objects = &L.engine->objects;
    prd.lightSources = &L.engine->lightSources;
    prd.imageSize = Vector2u({W, H});
    prd.origin = origin;
    prd.viewInverse = vi;
    prd.projInverse = pi;
    for (;;) {
      uint32_t k = next.fetch_add(1);
      if (k >= np) break;
      uint32_t p = p0 + k;
      prd.pixel[0] = p % W;
      prd.pixel[1] = p / W;
      for (unsigned s = 0; s < spp; ++s) {
        swr_shim_set_cursor(seed, p, s);
        Vector3f v = bd.renderPixel(prd);
        float* o = &per_sample[((size_t)k * spp + s) * 4];
        for (int c = 0; c < 3; ++c) o[c] = v[c];
        o[3] = 1.0f;
      }
    }
  };
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nthreads; ++t) th.emplace_back(work);
  for (auto& t : th) t.join();
  Writer w(a[12]);
  w.f32("per_sample", per_sample);
  return 0;
}

int cmd_tree(char** a) {
  std::vector<uint8_t> raw = read_file(a[0]);
  const size_t n = raw.size() / 24;
  const float* b = (const float*)raw.data();
  std::vector<BVH::Data> in;
  for (size_t i = 0; i < n; ++i) {
    AABB box(Vector3f({b[6 * i + 0], b[6 * i + 1], b[6 * i + 2]}),
             Vector3f({b[6 * i + 3], b[6 * i + 4], b[6 * i + 5]}));
    in.push_back({box, i});
  }
  BVH bvh;
  bvh.init(in);
  std::vector<uint32_t> tok;
  tree_tokens(bvh.root, tok);
  Writer w(a[1]);
  w.u32("tree", tok);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_harness dump|trace|render|tree ...\n");
    return 2;
  }
  std::string cmd = argv[1];
  try {
    if (cmd == "dump" && argc == 8) return cmd_dump(argv + 2);
    if (cmd == "trace" && argc == 6) return cmd_trace(argv + 2);
    if (cmd == "render" && argc == 13) return cmd_render(argv + 2);
    if (cmd == "tree" && argc == 4) return cmd_tree(argv + 2);
    if (cmd == "render_bdpt" && argc == 15) return cmd_render_bdpt(argv + 2);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "harness error: %s\n", e.what());
    return 1;
  }
  std::fprintf(stderr, "bad arguments\n");
  return 2;
}
