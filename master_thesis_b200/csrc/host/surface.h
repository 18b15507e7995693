// Scene / camera / renderer file surface of the path tracer.
//
// These classes accept the same text and mesh files as the reference's SoftwareRenderer and
// turn them into world-space geometry that is bit-identical to what the reference computes in
// GraphicsObject::init. The file formats and their parsing rules follow:
//   software_renderer/input_parser.cpp:38-93   (.scene / .camera / .renderer text format)
//   software_renderer/obj_loader.cpp:19-184    (OBJ, path basepath + "../res/obj/")
//   software_renderer/stl_loader.cpp:18-123    (binary STL, path "../res/stl/" relative to cwd)
//   software_renderer/mesh_manager.cpp:17-60   (scene entries -> objects, mesh cache by name)
//   software_renderer/graphic/graphics_object.cpp:12-62 (S*R*T transform, material thresholds)
//   software_renderer/camera.cpp:13-51, graphic/graphics_engine.cpp:42-46 (camera matrices)
// Errors are reported as SurfaceError (system + message), the counterpart of the reference's
// InitException (init_exception.h:9-19).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "rmath.h"

namespace swr {

struct SurfaceError : public std::runtime_error {
  std::string system;
  int code;
  SurfaceError(int code_, const std::string& sys, const std::string& msg)
      : std::runtime_error("Init exception: " + sys + ": " + msg), system(sys), code(code_) {}
};

// One named block of a text file: "name" followed by tab-indented "key(v1, v2, ...)" lines.
class InputEntry {
 public:
  explicit InputEntry(const std::string& n) : name(n) {}
  bool has(const std::string& key) const { return data_.count(key) > 0; }
  const std::vector<std::string>& values(const std::string& key) const;
  // stringstream extraction, as InputEntry::get<T> (input_parser.h:23-28)
  float get_float(const std::string& key, size_t index = 0) const;
  unsigned get_uint(const std::string& key, size_t index = 0) const;
  V3 get_v3(const std::string& key) const;
  // std::stof of the four values, as InputEntry::getRotation (input_parser.cpp:20-26)
  Rot get_rotation(const std::string& key) const;
  void insert(const std::string& key, const std::vector<std::string>& vals) {
    data_.insert({key, vals});  // first occurrence of a key wins, like unordered_map::insert
  }
  std::string name;

 private:
  std::unordered_map<std::string, std::vector<std::string>> data_;
};

// Parses a whole file; throws SurfaceError(IO) when the file cannot be opened.
std::vector<InputEntry> parse_input_file(const std::string& path);
std::vector<InputEntry> parse_input_text(const std::string& text);

// Object-space mesh: vertices (position, normal) and triangle indices.
struct Mesh {
  std::vector<V3> pos;
  std::vector<V3> nrm;
  std::vector<uint32_t> idx;  // 3 per triangle
  // Leaf order of the reference's BVH over this mesh (left-first DFS of BVH::init's tree,
  // built in object space). Empty when the mesh exceeds the exact-order size limit.
  std::vector<uint32_t> dfs;
  size_t num_tris() const { return idx.size() / 3; }
};

// OBJ loader: full path is basepath + "../res/obj/" + name (obj_loader.cpp:5-6,20).
Mesh load_obj(const std::string& basepath, const std::string& name);
Mesh parse_obj_text(const std::string& text);
// Binary STL loader: path "../res/stl/" + name relative to the working directory.
Mesh load_stl(const std::string& name);
Mesh parse_stl_bytes(const std::vector<uint8_t>& bytes);

struct Material {
  V3 color = v3(1.0f, 1.0f, 1.0f);
  bool light = false;
  float light_strength = 0.0f;
  float diffuse_w = 1.0f, reflect_w = 0.0f, transparent_w = 0.0f;
  float refraction_index = 1.0f;
  float diffuse_t = 1.0f, reflect_t = 1.0f, transparent_t = 1.0f;  // cumulative thresholds
};

struct Object {
  std::string mesh_name;
  uint32_t mesh_id = 0;
  V3 position = v3(0, 0, 0);
  V3 scl = v3(1.0f, 1.0f, 1.0f);
  Rot rotation;
  Material mat;
  uint32_t first_vertex = 0, num_vertices = 0;
  uint32_t first_tri = 0, num_tris = 0;
  Box aabb;  // world box over all vertices, first one padded (graphics_object.cpp:25)
};

// World-space scene: every object transformed, triangles in object-major order, so a triangle's
// global id is (sum of triangle counts of earlier objects) + its index in its object, which is
// the order of GraphicsObject::triangles within MeshManager's object order.
struct HostScene {
  std::vector<Mesh> meshes;
  std::vector<Object> objects;
  std::vector<V3> vpos, vnrm;       // world vertices of all objects, concatenated
  std::vector<uint32_t> tri;        // 3 global vertex indices per triangle
  std::vector<uint32_t> tri_obj;    // owning object per triangle
  std::vector<uint32_t> tri_rank;   // position of the triangle in the reference's visit order
  std::vector<uint32_t> obj_dfs;    // scene-level BVH leaf order of objects (may be empty)
  bool ranks_exact = true;          // false if some mesh or the scene exceeded the size limit
  size_t num_tris() const { return tri_obj.size(); }
};

struct LoadOptions {
  // Meshes / object counts above this size do not get the reference's exact BVH leaf order;
  // ties then go to the lower index. (The reference's own builder is cubic in this size; the
  // exact rebuild here takes about 0.2 s for 32k boxes, 1 s for 131k, 5 s for 524k on one core.)
  uint32_t max_exact_order = 1u << 20;
  uint32_t threads = 0;  // mesh files parsed concurrently by load_scene_file; 0 = all cores
};

// Reads a mesh named in a .scene block: ".obj" from basepath + "../res/obj/", ".stl" from
// "../res/stl/"; any other name is a parse error (mesh_manager.cpp:17-28).
Mesh load_mesh_file(const std::string& basepath, const std::string& name);

// Checks a mesh and computes its reference leaf order (mesh.cpp:24-37); throws SurfaceError.
void prepare_mesh(const std::string& name, Mesh& mesh, const LoadOptions& opt);

// Adds one object (already parsed mesh + entry keys) the way MeshManager + GraphicsObject do.
class SceneBuilder {
 public:
  explicit SceneBuilder(const LoadOptions& opt = LoadOptions()) : opt_(opt) {}
  uint32_t add_mesh(const std::string& name, Mesh mesh);  // returns mesh id (cached by name)
  uint32_t add_prepared_mesh(const std::string& name, Mesh mesh);  // after prepare_mesh
  bool has_mesh(const std::string& name) const { return mesh_ids_.count(name) > 0; }
  uint32_t mesh_id(const std::string& name) const { return mesh_ids_.at(name); }
  void add_object(uint32_t mesh_id, const V3& position, const V3& scl, const Rot& rot,
                  const Material& mat);
  void add_entry(const InputEntry& e, const std::string& basepath);  // a .scene block
  void add_entry_object(const InputEntry& e, uint32_t mesh_id);      // its keys, mesh resolved
  HostScene finish();  // computes reference visit ranks

 private:
  LoadOptions opt_;
  HostScene s_;
  std::unordered_map<std::string, uint32_t> mesh_ids_;
};

HostScene load_scene_file(const std::string& scene_path, const std::string& basepath,
                          const LoadOptions& opt = LoadOptions());

// Camera as parsed from a .camera file (camera.cpp:13-31).
struct CameraParams {
  float theta = (float)M_PI;
  float phi = (float)M_PI_2;
  V3 position = v3(4.0f, 0.0f, 0.0f);
  float fov = (float)M_PI_4;
  float nearZ = 0.01f, farZ = 1000.0f;
  bool invertY = true;
  bool has_fov_key = false;  // extension key fov(degrees); the reference ignores it
  float fov_key_deg = 45.0f;
};
CameraParams parse_camera(const InputEntry& e);
CameraParams load_camera_file(const std::string& path);

// The per-image camera data of GraphicsEngine::render (graphics_engine.cpp:42-46).
struct CameraFrame {
  M4 view_inv, proj_inv;
  V3 origin;
};
CameraFrame camera_frame(const CameraParams& c, uint32_t width, uint32_t height, bool use_fov_key);

// Renderer file: first entry name and its keys (main.cpp:62-66, path_tracer.cpp:13-16).
struct RendererParams {
  std::string name;
  unsigned vision_jump_count = 0;
  unsigned rays_per_pixel = 0;
  unsigned light_jump_count = 0;  // BidirectionalPathTracer only
  unsigned max_depth = 0;         // BidirectionalPathTracer only
};
// Renderer file; the bidirectional tracer's keys are read (and required) only with bdpt_keys.
RendererParams load_renderer_file(const std::string& path, bool bdpt_keys = true);

// Renderer file of the RayTrace program (src/main.cpp:153-168): the renderer entry, then the
// denoiser entries in file order (gauss_denoiser.cpp:51-54; MedianDenoiser has no keys).
struct RtDenoiserParams {
  std::string name;
  unsigned kernel_size = 0;
  float sigma = 0.0f;
};
struct RtRendererParams {
  std::string name;
  unsigned vision_jump_count = 0;
  unsigned vision_rays_per_pixel = 0;
  std::vector<RtDenoiserParams> denoisers;
};
// Accepts the PathTracer (path_tracer.cpp:30-33); the program's other renderers raise
// SWR_ERR_UNSUPPORTED, unknown renderer or denoiser names the getRenderer / getDenoiser errors.
RtRendererParams load_rt_renderer_file(const std::string& path);

}  // namespace swr
