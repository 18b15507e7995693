// Scene / camera / renderer / mesh file surface. See surface.h for the reference files each
// part follows. Numeric parsing deliberately goes through the same standard-library routines the
// reference uses (stringstream extraction, std::stof, std::atof, std::atoi), so the parsed floats
// are identical, and all arithmetic goes through rmath.h.
#include "surface.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <map>
#include <sstream>
#include <thread>
#include <unordered_map>

#include "ref_bvh.h"

namespace swr {

static constexpr int kErrIO = 1;
static constexpr int kErrParse = 2;
static constexpr int kErrInvalid = 6;
static constexpr int kErrUnsupported = 7;

// ------------------------------------------------------------------------------------------
// InputEntry

const std::vector<std::string>& InputEntry::values(const std::string& key) const {
  auto it = data_.find(key);
  if (it == data_.end())
    throw SurfaceError(kErrParse, "InputEntry", "entry \"" + name + "\" has no key \"" + key + "\"");
  return it->second;
}

static const std::string& value_at(const InputEntry& e, const std::string& key, size_t index) {
  const auto& v = e.values(key);
  if (index >= v.size())
    throw SurfaceError(kErrParse, "InputEntry",
                       "key \"" + key + "\" of entry \"" + e.name + "\" has too few values");
  return v[index];
}

float InputEntry::get_float(const std::string& key, size_t index) const {
  float value = 0.0f;
  std::stringstream(value_at(*this, key, index)) >> value;
  return value;
}

unsigned InputEntry::get_uint(const std::string& key, size_t index) const {
  unsigned value = 0;
  std::stringstream(value_at(*this, key, index)) >> value;
  return value;
}

V3 InputEntry::get_v3(const std::string& key) const {
  return v3(get_float(key, 0), get_float(key, 1), get_float(key, 2));
}

Rot InputEntry::get_rotation(const std::string& key) const {
  try {
    V3 axis = v3(std::stof(value_at(*this, key, 0)), std::stof(value_at(*this, key, 1)),
                 std::stof(value_at(*this, key, 2)));
    float angle = std::stof(value_at(*this, key, 3));
    return Rot::from_axis_angle(axis, angle);
  } catch (const std::logic_error&) {
    throw SurfaceError(kErrParse, "InputEntry", "bad rotation in entry \"" + name + "\"");
  }
}

// ------------------------------------------------------------------------------------------
// Text format (input_parser.cpp:38-93). The loop drives the stream with the same primitive
// operations, so end-of-file corner cases (a last line without newline, an unterminated value
// list) come out the same.

template <class Stream>
static std::pair<std::string, std::vector<std::string>> read_key_values(Stream& in) {
  std::string key;
  std::getline(in, key, '(');
  std::vector<std::string> vals;
  std::string cur;
  while (in.good()) {
    char c = (char)in.get();
    if (c == ')') {
      in.get();
      break;
    } else if (c == ',') {
      vals.push_back(cur);
      cur.clear();
    } else if (c != ' ') {
      cur += c;
    }
  }
  vals.push_back(cur);
  return {key, vals};
}

template <class Stream>
static std::vector<InputEntry> parse_stream(Stream& in) {
  std::vector<InputEntry> out;
  InputEntry cur("");
  while (in.good()) {
    char c = (char)in.get();
    if (c == '\n') continue;
    if (c == '#') {
      std::string skip;
      std::getline(in, skip);
    } else if (c == '\t') {
      auto kv = read_key_values(in);
      cur.insert(kv.first, kv.second);
    } else if (c != ' ') {
      in.unget();
      if (!cur.name.empty()) out.push_back(cur);
      std::string name;
      std::getline(in, name);
      cur = InputEntry(name);
    }
  }
  if (!cur.name.empty()) out.push_back(cur);
  return out;
}

std::vector<InputEntry> parse_input_file(const std::string& path) {
  std::ifstream in(path);
  if (in.fail()) throw SurfaceError(kErrIO, "InputParser", "failed to open file \"" + path + "\"!");
  return parse_stream(in);
}

std::vector<InputEntry> parse_input_text(const std::string& text) {
  std::istringstream in(text);
  return parse_stream(in);
}

// ------------------------------------------------------------------------------------------
// OBJ (obj_loader.cpp). Vertices are de-duplicated on the (position, texcoord, normal) index
// triple in first-use order; n-gons are fanned from their first vertex.

namespace {
struct ObjCorner {
  unsigned pos, tc, nrm;
  bool operator<(const ObjCorner& o) const {
    if (pos != o.pos) return pos < o.pos;
    if (tc != o.tc) return tc < o.tc;
    return nrm < o.nrm;
  }
};

float atof_f(const std::string& s) { return (float)std::atof(s.c_str()); }

V3 obj_triple(std::istringstream& ls) {
  std::string a, b, c;
  std::getline(ls, a, ' ');
  std::getline(ls, b, ' ');
  std::getline(ls, c);
  return v3(atof_f(a), atof_f(b), atof_f(c));
}

ObjCorner obj_corner(const std::string& tok) {
  std::istringstream fs(tok);
  std::string a, b, c;
  std::getline(fs, a, '/');
  std::getline(fs, b, '/');
  std::getline(fs, c);
  return ObjCorner{(unsigned)std::atoi(a.c_str()), (unsigned)std::atoi(b.c_str()),
                   (unsigned)std::atoi(c.c_str())};
}
}  // namespace

static Mesh obj_from_stream(std::istream& in, const std::string& basepath, const std::string& name,
                            bool allow_mtl) {
  std::vector<V3> points, normals;
  size_t ntex = 0;
  std::vector<std::vector<ObjCorner>> faces;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string mode;
    std::getline(ls, mode, ' ');
    if (mode == "mtllib") {
      std::string mtl;
      std::getline(ls, mtl);
      if (allow_mtl) {
        std::ifstream mf(basepath + "../res/obj/" + mtl);
        if (!mf.is_open())
          throw SurfaceError(kErrIO, "ObjLoader", "Could not load MTL file \"" + mtl + "\"!");
      }
    } else if (mode == "v") {
      points.push_back(obj_triple(ls));
    } else if (mode == "vt") {
      ++ntex;
    } else if (mode == "vn") {
      normals.push_back(obj_triple(ls));
    } else if (mode == "f") {
      std::vector<ObjCorner> f;
      std::string tok;
      while (std::getline(ls, tok, ' ')) f.push_back(obj_corner(tok));
      faces.push_back(f);
    }
  }
  (void)ntex;
  Mesh m;
  std::map<ObjCorner, unsigned> uniq;
  for (const auto& f : faces)
    for (const auto& c : f) {
      if (uniq.count(c)) continue;
      if (c.pos == 0 || c.pos > points.size() || c.nrm == 0 || c.nrm > normals.size())
        throw SurfaceError(kErrParse, "ObjLoader", "face index out of range in \"" + name + "\"");
      m.pos.push_back(points[c.pos - 1]);
      m.nrm.push_back(normals[c.nrm - 1]);
      uniq.insert({c, (unsigned)(m.pos.size() - 1)});
    }
  for (const auto& f : faces)
    for (size_t i = 2; i < f.size(); ++i) {
      m.idx.push_back(uniq.find(f[0])->second);
      m.idx.push_back(uniq.find(f[i - 1])->second);
      m.idx.push_back(uniq.find(f[i])->second);
    }
  return m;
}

Mesh load_obj(const std::string& basepath, const std::string& name) {
  std::ifstream in(basepath + "../res/obj/" + name);
  if (!in.is_open())
    throw SurfaceError(kErrIO, "ObjLoader", "Could not load OBJ file \"" + name + "\"!");
  return obj_from_stream(in, basepath, name, true);
}

Mesh parse_obj_text(const std::string& text) {
  std::istringstream in(text);
  return obj_from_stream(in, "", "<text>", false);
}

// ------------------------------------------------------------------------------------------
// STL (stl_loader.cpp). Positions are grouped by exact value in a std::unordered_map with the
// reference's key hash, then each position group is split into sub-groups of corners whose face
// normals are within 60 degrees of the sub-group's first normal; every sub-group becomes one
// vertex with the mean face normal. The map's iteration order decides the vertex order (and with
// it which vertex pads the object box), so the same container, hash and insertion sequence are
// used here.

namespace {
struct PosKey {
  V3 p;
  bool operator==(const PosKey& o) const {
    return p[0] == o.p[0] && p[1] == o.p[1] && p[2] == o.p[2];
  }
};
struct PosKeyHash {
  size_t operator()(const PosKey& k) const {
    size_t h = ~size_t(0);
    for (size_t i = 0; i < 3; ++i) h ^= std::hash<float>()(k.p[(int)i]) << i;
    return h;
  }
};
struct Corner {
  uint32_t tri;
  uint32_t corner;
};
struct StlTri {
  V3 n;
  V3 v[3];
};

// angle between two vectors in double, as Vector::angle (vector.h:243-245)
bool normals_fit(const V3& a, const V3& b) {
  double c = double(dot(a, b)) / (magnitude(a) * magnitude(b));
  c = std::clamp(c, -1.0, 1.0);
  const float angle = (float)std::acos(c);  // stl_loader.cpp:12 keeps the angle in a float
  return angle < 1.0 / 3.0 * M_PI;
}
}  // namespace

Mesh parse_stl_bytes(const std::vector<uint8_t>& bytes) {
  if (bytes.size() < 84) throw SurfaceError(kErrParse, "STLLoader", "file too short");
  uint32_t count;
  std::memcpy(&count, bytes.data() + 80, 4);
  std::vector<StlTri> tris;
  tris.reserve(count);
  for (uint32_t t = 0; t < count; ++t) {
    size_t off = 84 + (size_t)t * 50;
    float raw[12] = {0};
    if (off + 50 <= bytes.size()) std::memcpy(raw, bytes.data() + off, 48);
    // a short file leaves the rest of the record zeroed, as an ifstream read into a
    // zero-initialised struct would leave it; y and z are swapped on load
    StlTri tr;
    tr.n = v3(raw[0], raw[2], raw[1]);
    for (int i = 0; i < 3; ++i) tr.v[i] = v3(raw[3 + 3 * i], raw[3 + 3 * i + 2], raw[3 + 3 * i + 1]);
    tris.push_back(tr);
  }

  std::unordered_map<PosKey, std::vector<Corner>, PosKeyHash> pre;
  for (uint32_t t = 0; t < tris.size(); ++t)
    for (uint32_t i = 0; i < 3; ++i) {
      PosKey k{tris[t].v[i]};
      if (pre.count(k) == 0) pre.insert({k, {}});
      pre[k].push_back(Corner{t, i});
    }

  std::vector<std::pair<V3, std::vector<Corner>>> groups;
  for (const auto& kv : pre) {
    std::vector<Corner> rest = kv.second;
    std::vector<std::vector<Corner>> sub;
    sub.push_back({rest.back()});
    rest.pop_back();
    for (const Corner& c : rest) {
      bool placed = false;
      for (auto& g : sub) {
        if (normals_fit(tris[g.at(0).tri].n, tris[c.tri].n)) {
          g.push_back(c);
          placed = true;
          break;
        }
      }
      if (!placed) sub.push_back({c});
    }
    for (auto& g : sub) groups.push_back({kv.first.p, g});
  }

  Mesh m;
  std::vector<uint32_t> corner_vertex((size_t)tris.size() * 3, 0);
  uint32_t index = 0;
  for (const auto& g : groups) {
    V3 n = v3(0, 0, 0);
    for (const Corner& c : g.second) n = add(n, tris[c.tri].n);
    const float cnt = (float)g.second.size();
    n = v3(n[0] / cnt, n[1] / cnt, n[2] / cnt);
    m.pos.push_back(g.first);
    m.nrm.push_back(n);
    for (const Corner& c : g.second) corner_vertex[(size_t)c.tri * 3 + c.corner] = index;
    ++index;
  }
  m.idx = corner_vertex;
  return m;
}

Mesh load_stl(const std::string& name) {
  std::ifstream in("../res/stl/" + name, std::ios::in | std::ios::binary);
  if (!in.is_open())
    throw SurfaceError(kErrIO, "STLLoader", "Could not load STL file \"" + name + "\"!");
  std::vector<uint8_t> bytes((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  return parse_stl_bytes(bytes);
}

// ------------------------------------------------------------------------------------------
// Scene assembly (mesh_manager.cpp:30-60, graphics_object.cpp:12-62, mesh.cpp:24-37).

static bool ends_with(const std::string& v, const std::string& e) {
  return e.size() <= v.size() && std::equal(e.rbegin(), e.rend(), v.rbegin());
}

void prepare_mesh(const std::string& name, Mesh& mesh, const LoadOptions& opt) {
  if (mesh.num_tris() == 0)
    throw SurfaceError(kErrInvalid, "MeshManager", "mesh \"" + name + "\" has no triangles");
  for (uint32_t i : mesh.idx)
    if (i >= mesh.pos.size())
      throw SurfaceError(kErrInvalid, "MeshManager", "mesh \"" + name + "\" has a bad index");
  // topology of the reference's object-space BVH over triangle boxes (mesh.cpp:24-37)
  if (mesh.num_tris() <= opt.max_exact_order) {
    std::vector<Box> boxes(mesh.num_tris());
    for (size_t t = 0; t < mesh.num_tris(); ++t) {
      boxes[t].add(mesh.pos[mesh.idx[3 * t + 0]]);
      boxes[t].add(mesh.pos[mesh.idx[3 * t + 1]]);
      boxes[t].add(mesh.pos[mesh.idx[3 * t + 2]]);
    }
    mesh.dfs = ref_bvh_leaf_order(boxes);
  }
}

uint32_t SceneBuilder::add_mesh(const std::string& name, Mesh mesh) {
  auto it = mesh_ids_.find(name);
  if (it != mesh_ids_.end()) return it->second;
  prepare_mesh(name, mesh, opt_);
  return add_prepared_mesh(name, std::move(mesh));
}

uint32_t SceneBuilder::add_prepared_mesh(const std::string& name, Mesh mesh) {
  auto it = mesh_ids_.find(name);
  if (it != mesh_ids_.end()) return it->second;
  uint32_t id = (uint32_t)s_.meshes.size();
  s_.meshes.push_back(std::move(mesh));
  mesh_ids_[name] = id;
  return id;
}

void SceneBuilder::add_object(uint32_t mesh_id, const V3& position, const V3& scl, const Rot& rot,
                              const Material& mat_in) {
  const Mesh& mesh = s_.meshes.at(mesh_id);
  Object o;
  o.mesh_id = mesh_id;
  o.position = position;
  o.scl = scl;
  o.rotation = rot;
  o.mat = mat_in;
  // M = I * S * R * T, each step a full matrix product (graphics_object.cpp:54-62)
  M4 m = M4::identity();
  m = matmul(m, scale_matrix(scl));
  m = matmul(m, rot.matrix());
  m = matmul(m, translation_matrix(position));
  o.first_vertex = (uint32_t)s_.vpos.size();
  o.num_vertices = (uint32_t)mesh.pos.size();
  for (size_t i = 0; i < mesh.pos.size(); ++i) {
    V4 p = xform(m, v4(mesh.pos[i][0], mesh.pos[i][1], mesh.pos[i][2], 1.0f));
    V4 n = xform(m, v4(mesh.nrm[i][0], mesh.nrm[i][1], mesh.nrm[i][2], 0.0f));
    V3 wp = v3(p[0], p[1], p[2]);
    s_.vpos.push_back(wp);
    s_.vnrm.push_back(v3(n[0], n[1], n[2]));
    o.aabb.add(wp);
  }
  o.first_tri = (uint32_t)s_.tri_obj.size();
  o.num_tris = (uint32_t)mesh.num_tris();
  const uint32_t oid = (uint32_t)s_.objects.size();
  for (size_t i = 0; i < mesh.idx.size(); ++i) s_.tri.push_back(o.first_vertex + mesh.idx[i]);
  for (size_t t = 0; t < mesh.num_tris(); ++t) s_.tri_obj.push_back(oid);
  // material thresholds (graphics_object.cpp:48-51)
  Material& mt = o.mat;
  float total = mt.diffuse_w + mt.reflect_w + mt.transparent_w;
  mt.diffuse_t = mt.diffuse_w / total;
  mt.reflect_t = mt.diffuse_t + (mt.reflect_w / total);
  mt.transparent_t = mt.reflect_t + (mt.transparent_w / total);
  s_.objects.push_back(o);
}

Mesh load_mesh_file(const std::string& basepath, const std::string& name) {
  if (ends_with(name, ".obj")) return load_obj(basepath, name);
  if (ends_with(name, ".stl")) return load_stl(name);
  throw SurfaceError(kErrParse, "MeshManager", "unknown mesh type \"" + name + "\"");
}

void SceneBuilder::add_entry(const InputEntry& e, const std::string& basepath) {
  if (e.name == "Probes") return;
  const uint32_t mid = has_mesh(e.name) ? mesh_id(e.name) : add_mesh(e.name, load_mesh_file(basepath, e.name));
  add_entry_object(e, mid);
}

void SceneBuilder::add_entry_object(const InputEntry& e, uint32_t mid) {
  V3 pos = e.get_v3("position");
  V3 scl = v3(1.0f, 1.0f, 1.0f);
  Rot rot;
  Material mat;
  if (e.has("color")) mat.color = e.get_v3("color");
  if (e.has("scale")) scl = e.get_v3("scale");
  if (e.has("rotation")) rot = e.get_rotation("rotation");
  if (e.has("diffuse")) mat.diffuse_w = e.get_float("diffuse");
  if (e.has("reflect")) mat.reflect_w = e.get_float("reflect");
  if (e.has("transparent")) mat.transparent_w = e.get_float("transparent");
  if (e.has("refractionIndex")) mat.refraction_index = e.get_float("refractionIndex");
  if (e.has("lightSource")) {
    mat.light = true;
    mat.light_strength = e.get_float("lightSource", 0);
  }
  add_object(mid, pos, scl, rot, mat);
}

HostScene SceneBuilder::finish() {
  HostScene s = std::move(s_);
  s_ = HostScene();
  mesh_ids_.clear();
  const size_t nobj = s.objects.size();
  s.tri_rank.assign(s.num_tris(), 0);
  s.ranks_exact = true;
  for (const auto& m : s.meshes)
    if (m.dfs.empty()) s.ranks_exact = false;
  if (nobj > 0 && nobj <= opt_.max_exact_order) {
    std::vector<Box> boxes(nobj);
    for (size_t o = 0; o < nobj; ++o) boxes[o] = s.objects[o].aabb;
    s.obj_dfs = ref_bvh_leaf_order(boxes, nullptr, RefBuild::kAuto, 0);
  } else {
    s.obj_dfs.resize(nobj);
    for (size_t o = 0; o < nobj; ++o) s.obj_dfs[o] = (uint32_t)o;
    if (nobj > 0) s.ranks_exact = false;
  }
  // rank = position in the reference's visit order: objects in scene-BVH leaf order, and
  // within an object its triangles in mesh-BVH leaf order (scene.cpp:22-41,
  // graphics_object.cpp:64-87)
  uint32_t base = 0;
  for (uint32_t o : s.obj_dfs) {
    const Object& ob = s.objects[o];
    const Mesh& m = s.meshes[ob.mesh_id];
    for (uint32_t k = 0; k < ob.num_tris; ++k) {
      uint32_t local = m.dfs.empty() ? k : m.dfs[k];
      s.tri_rank[ob.first_tri + local] = base + k;
    }
    base += ob.num_tris;
  }
  return s;
}

// The mesh files named by a scene are read and prepared (parse, checks, reference leaf order)
// concurrently, one mesh per task; objects are then assembled in file order. A failure is
// reported at the first block that uses the failing mesh, in file order, as a sequential load
// (the reference's MeshManager) reports it.
HostScene load_scene_file(const std::string& scene_path, const std::string& basepath,
                          const LoadOptions& opt) {
  std::vector<InputEntry> entries = parse_input_file(scene_path);
  std::vector<std::string> names;
  std::unordered_map<std::string, size_t> index;
  for (const auto& e : entries)
    if (e.name != "Probes" && index.emplace(e.name, names.size()).second) names.push_back(e.name);
  std::vector<Mesh> meshes(names.size());
  std::vector<std::exception_ptr> errors(names.size());
  std::atomic<size_t> next{0};
  auto work = [&]() {
    for (size_t i; (i = next.fetch_add(1)) < names.size();) {
      try {
        Mesh m = load_mesh_file(basepath, names[i]);
        prepare_mesh(names[i], m, opt);
        meshes[i] = std::move(m);
      } catch (...) {
        errors[i] = std::current_exception();
      }
    }
  };
  unsigned nt = opt.threads ? opt.threads : std::max(1u, std::thread::hardware_concurrency());
  nt = (unsigned)std::min<size_t>(nt, names.size());
  std::vector<std::thread> pool;
  for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
  SceneBuilder b(opt);
  for (const auto& e : entries) {
    if (e.name == "Probes") continue;
    const size_t i = index.at(e.name);
    if (!b.has_mesh(e.name)) {
      if (errors[i]) std::rethrow_exception(errors[i]);
      b.add_prepared_mesh(e.name, std::move(meshes[i]));
    }
    b.add_entry_object(e, b.mesh_id(e.name));
  }
  return b.finish();
}

// ------------------------------------------------------------------------------------------
// Camera (camera.cpp:13-51) and per-image matrices (graphics_engine.cpp:42-46)

CameraParams parse_camera(const InputEntry& e) {
  CameraParams c;
  c.position = e.get_v3("position");
  float theta = e.get_float("angle", 0);
  float phi = e.get_float("angle", 1);
  theta = (float)((double)theta * M_PI);
  phi = (float)((double)phi * -M_PI_2 + M_PI_2);
  if (phi < 0.01f) phi = 0.01f;
  if (phi > M_PI - 0.01f) phi = (float)(M_PI - 0.01f);
  if (theta < -M_PI) theta = (float)((double)theta + M_PI * 2.0f);
  if (theta > M_PI) theta = (float)((double)theta - M_PI * 2.0f);
  c.theta = theta;
  c.phi = phi;
  if (e.has("fov")) {
    c.has_fov_key = true;
    c.fov_key_deg = e.get_float("fov");
  }
  return c;
}

CameraParams load_camera_file(const std::string& path) {
  auto entries = parse_input_file(path);
  if (entries.empty()) throw SurfaceError(kErrParse, "Camera", "no entry in \"" + path + "\"");
  return parse_camera(entries[0]);
}

CameraFrame camera_frame(const CameraParams& c, uint32_t width, uint32_t height, bool use_fov_key) {
  float sinPhi = (float)std::sin((double)c.phi);
  float cosPhi = (float)std::cos((double)c.phi);
  float sinTheta = (float)std::sin((double)c.theta);
  float cosTheta = (float)std::cos((double)c.theta);
  V3 look = v3(sinPhi * cosTheta, cosPhi, sinPhi * sinTheta);
  M4 view = look_at(c.position, add(look, c.position), v3(0.0f, 1.0f, 0.0f));
  float fov = c.fov;
  if (use_fov_key && c.has_fov_key) fov = (float)((double)c.fov_key_deg * M_PI / 180.0);
  M4 proj = perspective(float(width) / float(height), fov, c.nearZ, c.farZ, c.invertY);
  CameraFrame f;
  f.view_inv = inverse(view);
  f.proj_inv = inverse(proj);
  V4 o = xform(f.view_inv, v4(0.0f, 0.0f, 0.0f, 1.0f));
  f.origin = v3(o[0], o[1], o[2]);
  return f;
}

RendererParams load_renderer_file(const std::string& path, bool bdpt_keys) {
  auto entries = parse_input_file(path);
  if (entries.empty()) throw SurfaceError(kErrParse, "Renderer", "no entry in \"" + path + "\"");
  RendererParams r;
  r.name = entries[0].name;
  if (r.name != "PathTracer" && r.name != "BidirectionalPathTracer")
    throw SurfaceError(kErrInvalid, "getRenderer not found", r.name);
  if (r.name == "PathTracer") {  // path_tracer.cpp:13-16
    r.vision_jump_count = entries[0].get_uint("visionJumpCount");
    r.rays_per_pixel = entries[0].get_uint("raysPerPixel");
  } else if (bdpt_keys) {  // bidirectional_path_tracer.cpp:13-18
    r.vision_jump_count = entries[0].get_uint("visionJumpCount");
    r.light_jump_count = entries[0].get_uint("lightJumpCount");
    r.max_depth = entries[0].get_uint("maxDepth");
    r.rays_per_pixel = entries[0].get_uint("raysPerPixel");
  }
  return r;
}

RtRendererParams load_rt_renderer_file(const std::string& path) {
  auto entries = parse_input_file(path);
  if (entries.empty()) throw SurfaceError(kErrParse, "Renderer", "no entry in \"" + path + "\"");
  RtRendererParams r;
  r.name = entries[0].name;
  // getRenderer (src/main.cpp:58-71)
  static const char* kOthers[] = {"PhotonMapper", "BidirectionalPathTracer", "ShadowTracer",
                                  "Majercik2019", "Majercik2022", "Majercik2022BidirectionalPathTracer",
                                  "Bitterli2020", "Bitterli2020BidirectionalPathTracer", "MetaRenderer",
                                  "PhongShader"};
  if (r.name != "PathTracer") {
    for (const char* n : kOthers)
      if (r.name == n)
        throw SurfaceError(kErrUnsupported, "getRenderer",
                           r.name + " is a renderer of the RayTrace program that this library does not restate");
    throw SurfaceError(kErrInvalid, "getRenderer not found", r.name);
  }
  r.vision_jump_count = entries[0].get_uint("visionJumpCount");
  r.vision_rays_per_pixel = entries[0].get_uint("visionRayPerPixelCount");
  for (size_t i = 1; i < entries.size(); ++i) {  // getDenoiser (src/main.cpp:73-77)
    RtDenoiserParams d;
    d.name = entries[i].name;
    if (d.name == "GaussDenoiser") {
      d.kernel_size = entries[i].get_uint("kernelSize");
      d.sigma = entries[i].get_float("sigma");
    } else if (d.name != "MedianDenoiser") {
      throw SurfaceError(kErrInvalid, "getDenoiser not found", d.name);
    }
    r.denoisers.push_back(d);
  }
  return r;
}

}  // namespace swr
