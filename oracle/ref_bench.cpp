// TEST INFRASTRUCTURE ONLY. Times the reference's own CPU path tracer on a bounded pixel sample.
// Linked against the unmodified reference sources, including its original RandomGenerator
// (mutex-guarded mt19937), so the timed code is exactly the reference's PathTracer::renderPixel ->
// Scene::traceRay -> BVH::getHits -> Triangle::rayIntersects path. The driver loop reproduces
// GraphicsEngine::render's worker (graphics_engine.cpp:59-97): threads pull pixel indices from an
// atomic counter, render, clamp and quantise. The pixel sample is every k-th pixel of the image,
// so it spans the whole frame.
//
//   ref_bench <basepath> <scene> <camera> <W> <H> <spp> <depth> <threads> <max_pixels> [fast]
//             [bdpt <lightJumpCount> <maxDepth>] [passes <timed> <warmup>] [target <seconds>]
//
// With "passes", the scene is loaded once and the same pixel sample is rendered <warmup> untimed
// times and then <timed> timed times (one timed pass = one bench step); the JSON line lists every
// timed pass. Without it there is one timed pass and no warm-up. With "target", max_pixels is
// only an upper bound: an untimed probe over a few pixels per thread measures the rate first, and
// the sample is sized so that one pass takes about <seconds>.
//
// With "bdpt" the timed renderer is the reference's BidirectionalPathTracer (visionJumpCount =
// depth) instead of its PathTracer.
//
// With "fast", scene loading replaces the two BVH::init calls (mesh topology, scene topology) by an
// exact re-implementation of the same agglomerative build (tree-identical, checked by the tests)
// because the reference's own builder is cubic in the number of leaves; everything that is timed
// is unchanged reference code. Prints one JSON line.
#include <algorithm>
#include <atomic>
#include <chrono>
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
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../master_thesis_b200/csrc/host/ref_bvh.h"

#define private public
#include "camera.h"
#include "graphic/graphics_engine.h"
#include "graphic/bidirectional_path_tracer.h"
#include "graphic/graphics_object.h"
#include "graphic/path_tracer.h"
#include "graphic/scene.h"
#include "input_parser.h"
#include "mesh_manager.h"
#include "obj_loader.h"
#include "stl_loader.h"
#undef private

namespace {

swr::Box to_box(const AABB& a) {
  swr::Box b;
  b.empty = a.empty;
  for (int i = 0; i < 3; ++i) {
    b.lo[i] = a.aabbMin[i];
    b.hi[i] = a.aabbMax[i];
  }
  return b;
}

// BVH::Node tree equal to what BVH::init builds over `in`
BVH::Node* fast_tree(const std::vector<BVH::Data>& in) {
  std::vector<swr::Box> boxes;
  for (const auto& d : in) boxes.push_back(to_box(d.aabb));
  swr::RefTree t;
  swr::ref_bvh_leaf_order(boxes, &t);
  const size_t n = in.size();
  std::vector<BVH::Node*> nodes(t.left.size(), nullptr);
  for (size_t i = 0; i < t.left.size(); ++i) {
    BVH::Node* nd = new BVH::Node();
    nd->left = nd->right = nullptr;
    nd->elemIndex = 0;
    if (i < n) {
      nd->aabb = in[i].aabb;
      nd->elemIndex = in[i].elemIndex;
    }
    nodes[i] = nd;
  }
  for (size_t i = n; i < t.left.size(); ++i) {
    nodes[i]->left = nodes[t.left[i]];
    nodes[i]->right = nodes[t.right[i]];
    nodes[i]->aabb = AABB(nodes[i]->left->aabb, nodes[i]->right->aabb);
  }
  return nodes[t.root];
}

bool ends_with(const std::string& v, const std::string& e) {
  return e.size() <= v.size() && std::equal(e.rbegin(), e.rend(), v.rbegin());
}

// MeshManager::createObjectsFromFile (mesh_manager.cpp:30-60) with the mesh BVH from fast_tree
std::vector<GraphicsObject*> load_fast(const std::string& basepath, const std::string& scene,
                                       std::vector<GraphicsObject*>& lights) {
  InputParser parser(scene);
  parser.parse();
  std::unordered_map<std::string, Mesh*> meshes;
  std::vector<GraphicsObject*> objs;
  for (unsigned i = 0; i < parser.size(); ++i) {
    const InputEntry& entry = parser.getInputEntry(i);
    if (entry.name == "Probes") continue;
    Mesh* mesh;
    if (meshes.count(entry.name)) {
      mesh = meshes[entry.name];
    } else {
      if (ends_with(entry.name, ".obj")) {
        ObjLoader l(basepath);
        l.load(entry.name);
        mesh = l.get_mesh();
      } else {
        STLLoader l(basepath);
        l.load(entry.name);
        mesh = l.get_mesh();
      }
      std::vector<BVH::Data> in;
      for (size_t k = 0; k < mesh->indices.size(); k += 3) {
        AABB box;
        box.addPoint(mesh->vertices[mesh->indices[k + 0]].pos);
        box.addPoint(mesh->vertices[mesh->indices[k + 1]].pos);
        box.addPoint(mesh->vertices[mesh->indices[k + 2]].pos);
        in.push_back({box, k / 3});
      }
      mesh->bvh.root = fast_tree(in);
      meshes[entry.name] = mesh;
    }
    Vector3f pos = entry.getVector<3, float>("position");
    GraphicsObject* obj = new GraphicsObject(mesh, pos);
    if (entry.keyExists("color")) obj->color = entry.getVector<3, float>("color");
    if (entry.keyExists("scale")) obj->scale = entry.getVector<3, float>("scale");
    if (entry.keyExists("rotation")) obj->rotation = entry.getRotation("rotation");
    if (entry.keyExists("diffuse")) obj->diffuseWeight = entry.get<float>("diffuse");
    if (entry.keyExists("reflect")) obj->reflectWeight = entry.get<float>("reflect");
    if (entry.keyExists("transparent")) obj->transparentWeight = entry.get<float>("transparent");
    if (entry.keyExists("refractionIndex")) obj->refractionIndex = entry.get<float>("refractionIndex");
    if (entry.keyExists("lightSource")) {
      obj->lightSource = true;
      obj->lightStrength = entry.get<float>("lightSource", 0);
      lights.push_back(obj);
    }
    objs.push_back(obj);
  }
  return objs;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 10) {
    std::fprintf(stderr,
                 "usage: ref_bench basepath scene camera W H spp depth threads max_pixels [fast] [bdpt light maxdepth]\n");
    return 2;
  }
  std::string basepath = argv[1], scenePath = argv[2], cameraPath = argv[3];
  unsigned W = (unsigned)std::atoi(argv[4]), H = (unsigned)std::atoi(argv[5]);
  unsigned spp = (unsigned)std::atoi(argv[6]), depth = (unsigned)std::atoi(argv[7]);
  unsigned threads = (unsigned)std::atoi(argv[8]);
  uint64_t maxPixels = std::strtoull(argv[9], nullptr, 10);
  bool fast = false;
  bool bdpt = false;
  unsigned light_jumps = 0, max_depth = 0;
  unsigned timed_passes = 1, warm_passes = 0;
  double target_s = 0.0;
  for (int a = 10; a < argc; ++a) {
    const std::string k = argv[a];
    if (k == "fast") fast = true;
    if (k == "passes" && a + 2 < argc) {
      timed_passes = std::max(1, std::atoi(argv[a + 1]));
      warm_passes = (unsigned)std::max(0, std::atoi(argv[a + 2]));
      a += 2;
    }
    if (k == "target" && a + 1 < argc) {
      target_s = std::atof(argv[a + 1]);
      a += 1;
    }
    if (k == "bdpt" && a + 2 < argc) {
      bdpt = true;
      light_jumps = (unsigned)std::atoi(argv[a + 1]);
      max_depth = (unsigned)std::atoi(argv[a + 2]);
      a += 2;
    }
  }

  auto t0 = std::chrono::steady_clock::now();
  GraphicsEngine engine;
  engine.imageSize = Vector2u({W, H});
  Renderer* pt;
  if (bdpt) {
    BidirectionalPathTracer* b = new BidirectionalPathTracer();
    b->visionJumpCount = depth;
    b->lightJumpCount = light_jumps;
    b->maxDepth = max_depth;
    b->raysPerPixel = spp;
    pt = b;
  } else {
    PathTracer* p = new PathTracer();
    p->visionJumpCount = depth;
    p->raysPerPixel = spp;
    pt = p;
  }
  MeshManager* mm = nullptr;
  if (fast) {
    std::vector<GraphicsObject*> lights;
    engine.objects = load_fast(basepath, scenePath, lights);
    engine.lightSources = lights;
    engine.renderer = pt;
    engine.threadCount = threads;
    // GraphicsEngine::init (graphics_engine.cpp:20-30) with the scene BVH from fast_tree
    std::vector<BVH::Data> in;
    for (size_t i = 0; i < engine.objects.size(); ++i) {
      engine.objects[i]->init();
      engine.scene.addObject(engine.objects[i]);
      in.push_back({engine.objects[i]->aabb, i});
    }
    engine.scene.bvh.root = fast_tree(in);
    engine.image.resize((size_t)W * H * 3);
  } else {
    mm = new MeshManager(basepath);
    mm->createObjectsFromFile(scenePath);
    engine.objects = mm->getCreatedObjects();
    engine.lightSources = mm->getCreatedLightSources();
    engine.init(pt, threads);
  }
  Camera* cam = new Camera();
  InputParser cp(cameraPath);
  cp.parse();
  cam->parseInput(cp.getInputEntry(0));
  engine.camera = cam;
  auto t1 = std::chrono::steady_clock::now();

  Matrix4f vi = cam->getViewMatrix().inverseMatrix();
  Matrix4f pi = cam->getProjectionMatrix(float(W) / float(H)).inverseMatrix();
  Vector3f origin = cutVector(vi * Vector4f({0.0f, 0.0f, 0.0f, 1.0f}));
  const uint64_t total = (uint64_t)W * H;
  uint64_t npix = std::min<uint64_t>(maxPixels, total);
  uint64_t stride = std::max<uint64_t>(1, total / std::max<uint64_t>(1, npix));
  std::atomic<uint64_t> counter(0);
  auto worker = [&]() {
    Renderer::PixelRenderData prd;
    prd.scene = &engine.scene;
    prd.objects = &engine.objects;
    prd.lightSources = &engine.lightSources;
    prd.imageSize = engine.imageSize;
    prd.origin = origin;
    prd.viewInverse = vi;
    prd.projInverse = pi;
    for (;;) {
      uint64_t k = counter.fetch_add(1);
      if (k >= npix) break;
      uint64_t p = (k * stride) % total;
      prd.pixel[0] = (uint32_t)(p % W);
      prd.pixel[1] = (uint32_t)(p / W);
      Vector3f c = engine.renderer->renderPixel(prd);
      for (unsigned i = 0; i < 3; ++i) c[i] = std::clamp(c[i], 0.0f, 1.0f);
      size_t idx = (prd.pixel[0] + (size_t)prd.pixel[1] * W) * 3;
      for (unsigned i = 0; i < 3; ++i) engine.image[idx + i] = (char)(c[i] * 255.0f);
    }
  };
  // one pass: GraphicsEngine::render's worker threads over the pixel sample
  auto pass = [&]() {
    counter.store(0);
    auto a = std::chrono::steady_clock::now();
    std::vector<std::thread> th;
    for (unsigned t = 0; t < threads; ++t) th.emplace_back(worker);
    for (auto& t : th) t.join();
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
  };
  uint64_t probe_pixels = 0;
  double probe_s = 0.0;
  if (target_s > 0.0) {
    const uint64_t cap = npix;
    npix = std::min<uint64_t>(cap, std::max<uint64_t>(8, 4ull * threads));
    stride = std::max<uint64_t>(1, total / npix);
    probe_pixels = npix;
    probe_s = pass();
    const double rate = (double)npix / std::max(probe_s, 1e-6);
    npix = std::min<uint64_t>(cap, std::max<uint64_t>(2ull * threads, (uint64_t)(rate * target_s)));
    stride = std::max<uint64_t>(1, total / npix);
  }
  for (unsigned w = 0; w < warm_passes; ++w) pass();
  std::vector<double> pass_s;
  double render_s = 0.0;
  for (unsigned r = 0; r < timed_passes; ++r) {
    pass_s.push_back(pass());
    render_s += pass_s.back();
  }
  double load_s = std::chrono::duration<double>(t1 - t0).count();
  double samples = (double)npix * spp * timed_passes;
  std::string passes = "[";
  for (size_t r = 0; r < pass_s.size(); ++r) passes += (r ? ", " : "") + std::to_string(pass_s[r]);
  passes += "]";
  std::printf(
      "{\"pixels\": %llu, \"spp\": %u, \"samples\": %.0f, \"threads\": %u, \"load_s\": %.6f, "
      "\"render_s\": %.6f, \"msamples_per_s\": %.6f, \"fast_build\": %s, \"timed_passes\": %u, "
      "\"warmup_passes\": %u, \"pass_s\": %s, \"probe_pixels\": %llu, \"probe_s\": %.6f}\n",
      (unsigned long long)npix, spp, samples, threads, load_s, render_s,
      samples / render_s / 1e6, fast ? "true" : "false", timed_passes, warm_passes, passes.c_str(),
      (unsigned long long)probe_pixels, probe_s);
  return 0;
}
