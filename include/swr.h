/* swr.h - C ABI of the B200 path tracer (drop-in for vikkre/master_thesis's SoftwareRenderer
 * PathTracer path).
 *
 * Parts: the file surface (scene, mesh, camera and renderer files), scene creation with a host or
 * device BVH build, closest-hit queries, the PathTracer render (reference and physical modes),
 * the BidirectionalPathTracer, batched and differentiable (adjoint) rendering, moving objects
 * (GPU transforms and BVH refit), the Vulkan program's PathTracer and denoisers restated in
 * CUDA, and PPM/PNG output.
 *
 * Conventions
 *  - Every call returns an int status: SWR_OK (0) or one of the SWR_ERR_* codes. No C++ exception
 *    crosses this boundary. swr_last_error() returns a thread-local "system: message" string for
 *    the last failure on the calling thread, in the spirit of the reference's InitException
 *    (software_renderer/init_exception.h:9-19).
 *  - Pointers are plain C pointers. Arguments documented "device or host" may point to either;
 *    the library inspects the pointer and stages host memory through the device itself.
 *  - Device work is queued on the given CUDA stream (a cudaStream_t passed as void*, NULL = the
 *    legacy default stream) and is asynchronous unless stated; swr_sync waits for it. A scene
 *    handle must not be used by two host threads at the same time; different handles on different
 *    streams may run concurrently.
 */
#ifndef SWR_H
#define SWR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWR_ABI_VERSION 3

enum {
  SWR_OK = 0,
  SWR_ERR_IO = 1,          /* file missing / unreadable (InitException from the loaders) */
  SWR_ERR_PARSE = 2,       /* malformed scene / camera / renderer / mesh file */
  SWR_ERR_ALLOC = 3,       /* device or host allocation failed */
  SWR_ERR_CUDA = 4,        /* a CUDA runtime call failed */
  SWR_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
  SWR_ERR_INVALID = 6,     /* bad argument */
  SWR_ERR_UNSUPPORTED = 7  /* valid request this build does not handle */
};

/* Render semantics.
 * SWR_MODE_REFERENCE: exactly the reference's PathTracer::traceSinglePath (path_tracer.cpp:42-97):
 *   pixel-centre camera rays, the first back-face hits skipped (using up a depth slot), a path
 *   contributes its throughput product only when it hits a light source from the front, no
 *   Russian roulette, image = sum * 2*pi/spp (lightStrength is not used, as in the reference).
 * SWR_MODE_PHYSICAL: the same scenes and random numbers with emission L_e = color * lightStrength
 *   collected at emitters hit from the front (emitters absorb), two-sided Lambertian BRDF with
 *   per-triangle albedo, uniform-hemisphere sampling weight 2*albedo*cos, optional Russian
 *   roulette with a constant survival probability, image = sum / spp. */
enum { SWR_MODE_REFERENCE = 0, SWR_MODE_PHYSICAL = 1 };

typedef struct swr_material {
  float color[3];          /* GraphicsObject::color */
  float diffuse_t;         /* cumulative event thresholds, graphics_object.cpp:48-51 */
  float reflect_t;
  float transparent_t;
  float refraction_index;
  uint32_t light_source;   /* nonzero for lightSource(...) objects */
  float light_strength;
} swr_material;

/* World-space scene. Triangles are numbered in object-major order (the global triangle id of
 * the hit results); objects in scene-file order. */
typedef struct swr_scene_desc {
  uint32_t num_objects;
  uint32_t num_vertices;
  uint32_t num_triangles;
  uint32_t reserved;
  const float* vertex_pos;             /* [num_vertices*3] world positions */
  const float* vertex_normal;          /* [num_vertices*3] world normals as the reference keeps
                                          them (transformed, not renormalised) */
  const uint32_t* tri_vertices;        /* [num_triangles*3] global vertex indices v0 v1 v2 */
  const uint32_t* tri_object;          /* [num_triangles] owning object, non-decreasing */
  const uint32_t* tri_rank;            /* [num_triangles] position in the reference's visit order
                                          (closest-hit ties go to the lower rank); NULL = id order */
  const uint32_t* object_first_vertex; /* [num_objects+1] vertex range of each object; its box is
                                          built over that range in order, first point padded */
  const swr_material* materials;       /* [num_objects] */
  const float* tri_albedo;             /* [num_triangles*3] or NULL (physical mode albedo) */
} swr_scene_desc;

typedef struct swr_build_opts {
  uint32_t sah_bins;       /* host builder: SAH bins, 0 = 64 */
  uint32_t max_leaf;       /* triangles per leaf, 1..3; 0 = 3 */
  uint32_t threads;        /* host builder threads, 0 = all */
  uint32_t leaf_cost_pct;  /* SAH cost of a triangle test relative to a wide-node visit, in
                              percent (1..400); 0 = 80 */
  uint32_t builder;        /* SWR_BUILD_HOST (binned SAH on the host) or SWR_BUILD_DEVICE
                              (clustering and collapse on the GPU); same closest hits either way */
  uint32_t radius;         /* device builder: clustering search radius 1..256, 0 = 16 */
  uint32_t width;          /* children per wide node, 2..8 (nodes keep 8 slots); 0 = 8 */
} swr_build_opts;
enum { SWR_BUILD_HOST = 0, SWR_BUILD_DEVICE = 1 };

/* Camera as GraphicsEngine::render derives it (graphics_engine.cpp:42-46): inverse view and
 * projection matrices (row-major m[row][col], row-vector convention) and the eye position. */
typedef struct swr_camera {
  float view_inv[16];
  float proj_inv[16];
  float origin[3];
  float reserved;
} swr_camera;

typedef struct swr_render_opts {
  uint32_t width, height;  /* image size (argv[3], argv[4] of the reference CLI) */
  uint32_t spp;            /* raysPerPixel */
  uint32_t max_depth;      /* visionJumpCount, 1..31 */
  uint64_t seed;           /* key of the counter-based RNG */
  uint32_t mode;           /* SWR_MODE_* */
  uint32_t rr_depth;       /* physical mode: Russian roulette at path vertices >= rr_depth (0=off) */
  float rr_survive;        /* physical mode: survival probability, (0, 1] */
  uint32_t wave_size;      /* paths in flight, 0 = 2^23 (capped by the samples of a chunk). Each
                              path in flight holds 144 bytes of the scene's queue memory; a large
                              image renders fastest with all of its samples in flight (1920x1080
                              at 64 spp: 2^27 paths, 19.3 GB). The
                              bidirectional tracer: samples per chunk, 0 = as many as keep the
                              chunk's vertex tables within 2 GB */
  uint32_t block_size;     /* threads per block of the shading kernel, 0 = automatic */
  uint32_t flags;          /* SWR_RENDER_* */
  uint32_t refill;         /* bounce traversal: idle lanes (1..32) that trigger a refill, 0 = 8 */
  uint32_t trace_blocks;   /* bounce traversal: resident blocks per SM targeted by the register
                              budget, one of 0 (the library's default, 9), 9, 10 */
  uint32_t shade_batch;    /* adjoint: lanes of a warp with a pending hit that shade together
                              (1..32; fewer when no trace of the warp is in flight), 0 = the
                              library's choice; the wavefront renders ignore it */
  /* Part of an image, for splitting one image over several calls or GPUs (the reference's
   * engine splits one image over host threads by pixel, graphics_engine.cpp:49-56,73-74).
   * Sample range (swr_render, swr_render_profiled, swr_render_adjoint): samples
   * [sample_begin, sample_begin + spp) of every pixel of an image with spp_total samples per
   * pixel; the random numbers are those of the whole image's samples and the output is scaled by
   * the whole image's 1/spp_total (times 2 pi in reference mode), so the outputs of calls over a
   * partition of [0, spp_total) sum to the whole image up to float summation order, and their
   * adjoint gradients sum to the whole image's gradient. spp_total 0 = spp (the whole range).
   * Pixel range (swr_render, swr_render_profiled): pixels [pixel_begin, pixel_begin +
   * pixel_count) of the width x height image in row-major order; rgb_out then holds pixel_count
   * pixels (and samples_out pixel_count * spp samples), bit-identical to those pixels of a whole
   * image. pixel_count 0 = to the end of the image. The other entry points require all four 0. */
  uint32_t sample_begin;
  uint32_t spp_total;
  uint32_t pixel_begin;
  uint32_t pixel_count;
} swr_render_opts;

#define SWR_RENDER_SAMPLES_OUT 1u   /* write per-sample radiance to the samples buffer */

typedef struct swr_hit {
  uint32_t tri;            /* global triangle id, 0xFFFFFFFF on a miss */
  uint32_t obj;            /* object index, 0xFFFFFFFF on a miss */
  float dist2;             /* squared distance origin -> hit point, the reference's comparison key */
  float t;                 /* ray parameter of the hit */
} swr_hit;

typedef struct swr_scene swr_scene;
typedef struct swr_host_scene swr_host_scene;

/* ---------------------------------------------------------------------------------------------
 * Library */
const char* swr_last_error(void);
int swr_abi_version(void);
/* Waits for all work queued on stream. */
int swr_sync(void* stream);

/* ---------------------------------------------------------------------------------------------
 * Host-side file surface (software_renderer/mesh_manager.cpp:30-60 createObjectsFromFile,
 * obj_loader.cpp, stl_loader.cpp, input_parser.cpp, graphic/graphics_object.cpp:12-52 init).
 * OBJ meshes are read from basepath + "../res/obj/", STL meshes from "../res/stl/" relative to
 * the working directory, exactly like the reference. */
int swr_host_scene_load(const char* scene_path, const char* basepath, swr_host_scene** out);
/* Fills a descriptor whose arrays point into the host scene (valid until it is freed). */
int swr_host_scene_desc(const swr_host_scene* hs, swr_scene_desc* out);
/* 1 when every tie rank comes from the reference's exact BVH order, 0 when some mesh was too
 * large for it (then ties inside that mesh go to the lower triangle index). */
int swr_host_scene_ranks_exact(const swr_host_scene* hs);
void swr_host_scene_free(swr_host_scene* hs);

/* Camera file -> per-image matrices (camera.cpp:19-51, graphics_engine.cpp:42-46). With
 * use_fov_key nonzero an optional fov(degrees) key is honoured; otherwise the field of view is the
 * reference's fixed pi/4. */
int swr_camera_load(const char* camera_path, uint32_t width, uint32_t height, uint32_t use_fov_key,
                    swr_camera* out);
/* Camera from values instead of a file: the same result as a .camera file with
 * position(x, y, z) angle(angle_theta, angle_phi) and, when fov_deg > 0, fov(fov_deg) honoured. */
int swr_camera_make(const float position[3], float angle_theta, float angle_phi, float fov_deg,
                    uint32_t width, uint32_t height, swr_camera* out);
/* Renderer file (main.cpp:62-66, path_tracer.cpp:13-16): accepts PathTracer; returns its
 * visionJumpCount and raysPerPixel. */
int swr_renderer_load(const char* renderer_path, uint32_t* max_depth, uint32_t* spp);
/* Renderer file with either renderer of the reference (main.cpp:22-26): PathTracer
 * (path_tracer.cpp:13-16) or BidirectionalPathTracer (bidirectional_path_tracer.cpp:13-18). */
enum { SWR_RENDERER_PATH_TRACER = 0, SWR_RENDERER_BIDIRECTIONAL = 1 };
typedef struct swr_renderer_params {
  uint32_t kind;          /* SWR_RENDERER_* */
  uint32_t vision_jumps;  /* visionJumpCount */
  uint32_t light_jumps;   /* lightJumpCount (bidirectional) */
  uint32_t max_depth;     /* maxDepth (bidirectional) */
  uint32_t spp;           /* raysPerPixel */
  uint32_t reserved[3];
} swr_renderer_params;
int swr_renderer_load_params(const char* renderer_path, swr_renderer_params* out);

/* Derived per-triangle data exactly as the reference's Triangle / GraphicsObject compute them
 * (triangle.cpp:4-17, graphics_object.cpp:25): edges e0 = v1-v0, e1 = v2-v0 [3*ntri each],
 * den = d00 d01 d11 denom [4*ntri], triangle boxes lo.xyz hi.xyz [6*ntri], object boxes
 * [6*nobj]. Any output may be NULL. Host memory. */
int swr_scene_derive(const swr_scene_desc* desc, float* tri_e0, float* tri_e1, float* tri_den,
                     float* tri_box, float* obj_box);

/* ---------------------------------------------------------------------------------------------
 * Device scene (replaces MeshManager + GraphicsEngine::init + Scene::init, scene.cpp:13-20). The
 * library copies what it needs; the caller keeps ownership of the descriptor's arrays. */
int swr_scene_create(const swr_scene_desc* desc, const swr_build_opts* opts, swr_scene** out);
void swr_scene_destroy(swr_scene* scene);
/* Wide-BVH statistics: nodes, depth, bytes of nodes and triangle records. */
int swr_scene_stats(const swr_scene* scene, uint64_t out[8]);

/* Closest hit per ray (replaces Scene::traceRay, scene.cpp:22-56, with its exact semantics:
 * same triangle, same squared distance, ties to the reference's visit order).
 * ray_o, ray_d: [n*4] floats (x y z unused), device or host. out: [n] swr_hit, device or host. */
int swr_trace_closest(swr_scene* scene, const float* ray_o, const float* ray_d, uint64_t n,
                      swr_hit* out, void* stream);

/* As swr_trace_closest, also writing per ray the number of wide-BVH nodes visited and triangles
 * tested (counts: [2*n] uint32, device or host). Instrumentation for the traffic model. */
int swr_trace_closest_stats(swr_scene* scene, const float* ray_o, const float* ray_d, uint64_t n,
                            swr_hit* out, uint32_t* counts, void* stream);

/* Full image (replaces GraphicsEngine::render + PathTracer::renderPixel,
 * graphics_engine.cpp:42-97, path_tracer.cpp:18-40). rgb_out: [height*width*3] floats, row-major
 * (x + y*width)*3 as the reference's image buffer, unclamped radiance, device or host.
 * samples_out (optional, only with SWR_RENDER_SAMPLES_OUT): [height*width*spp*4] floats, per
 * sample r g b and a flag (1 = the path reached a light), device or host. */
int swr_render(swr_scene* scene, const swr_camera* cam, const swr_render_opts* opts, float* rgb_out,
               float* samples_out, void* stream);

#define SWR_RENDER_PROFILE 2u       /* time each kernel kind with CUDA events (see swr_render_profile) */
#define SWR_RENDER_COUNT 4u         /* count wide-BVH node visits and triangle tests of the bounce
                                       traversal kernel (slower; for the traffic model only) */
#define SWR_RENDER_STATIC_FETCH 8u  /* bounce traversal takes rays 32 at a time per warp and runs
                                       them to completion, instead of refilling idle lanes */
#define SWR_RENDER_POSTPONE 16u     /* bounce traversal postpones triangle tests while few lanes of
                                       a warp have any (keeps warps in one phase) */
#define SWR_RENDER_ONE_WAVEFRONT 32u /* run every chunk as one wavefront on the caller's stream. By
                                       default a chunk of 2^20 samples or more of a scene of 2^16
                                       triangles or more runs as two sub-wavefronts (half the pixels and half the paths in flight
                                       each) on the caller's stream and an internal one, so that the
                                       SMs one of them leaves idle at the end of a traversal launch
                                       take the other's work; results are identical either way.
                                       Profiled renders (SWR_RENDER_PROFILE) always use one. */
#define SWR_RENDER_HOST_LOOP 64u    /* the host launches every shade/trace round itself, one
                                       wavefront per chunk (as profiled renders do), instead of
                                       launching a CUDA graph whose round loop ends on the device.
                                       Profilers that capture kernels one launch at a time cannot
                                       capture the kernel nodes of such a graph. Results are
                                       identical; it is slower (a host wait every 8 rounds). */

/* Per-call instrumentation of swr_render_profiled. Times are device milliseconds summed over the
 * launches of each kernel kind (with SWR_RENDER_PROFILE). */
typedef struct swr_render_profile {
  uint64_t rays;            /* rays traced: camera prefix + all bounces */
  uint64_t bounce_rays;     /* rays traced by the bounce traversal kernel */
  uint64_t node_visits;     /* with SWR_RENDER_COUNT: nodes fetched by the bounce traversal */
  uint64_t tri_tests;       /* with SWR_RENDER_COUNT: triangle records tested by it */
  uint64_t iterations;      /* shade/trace rounds */
  uint64_t launches;        /* kernels launched by the call */
  uint64_t trace_launches;  /* launches of the bounce traversal kernel */
  uint64_t first_trace_rays;  /* rays of its first non-empty launch (first chunk) */
  uint64_t h2d_bytes, d2h_bytes;  /* explicit host<->device copies made by the call */
  double trace_ms, shade_ms, camera_ms, resolve_ms;
} swr_render_profile;

/* As swr_render, filling *prof (which may be NULL). */
int swr_render_profiled(swr_scene* scene, const swr_camera* cam, const swr_render_opts* opts,
                        float* rgb_out, float* samples_out, void* stream, swr_render_profile* prof);

/* Bidirectional path tracer (replaces BidirectionalPathTracer, bidirectional_path_tracer.cpp:20-168,
 * with Scene::isOccluded, scene.cpp:58-83, as its occlusion query). opts->max_depth is
 * visionJumpCount (1..16), opts->mode must be SWR_MODE_REFERENCE; bdpt->light_jumps is
 * lightJumpCount (0..16) and bdpt->max_depth the reference's maxDepth (connections with
 * vision index + light index <= maxDepth; the sum is divided by it). The light sources are the
 * scene's light_source objects in object order; the scene needs at least one. samples_out (with
 * SWR_RENDER_SAMPLES_OUT) receives per sample the contribution before the 2*pi/spp scale. */
typedef struct swr_bdpt_opts {
  uint32_t light_jumps;
  uint32_t max_depth;
  uint32_t shade_batch;  /* lanes of a warp with a finished trace that advance together, bits 0-7
                            for the path stages and bits 8-15 for the connection queries (each
                            1..32, 0 = the library's choice) */
  uint32_t blocks_per_sm;  /* resident blocks per SM targeted by the register budget: 0 (compiler's
                              choice), 5, 6 or 8 */
} swr_bdpt_opts;
int swr_render_bdpt(swr_scene* scene, const swr_camera* cam, const swr_render_opts* opts,
                    const swr_bdpt_opts* bdpt, float* rgb_out, float* samples_out, void* stream);

/* Batched rendering: many independent jobs (scene, camera, options, output) in one shared
 * wavefront, so that small images do not leave the GPU idle (no counterpart in the reference,
 * which renders one image per process). Per-job results match swr_render's for the same job up to
 * the order of the per-pixel float sums (the batch sums in 64-bit fixed point). */
typedef struct swr_batch swr_batch;
typedef struct swr_batch_job {
  swr_scene* scene;       /* built scene (jobs may share one) */
  swr_camera cam;
  swr_render_opts opts;   /* width, height, spp, max_depth, seed, mode, rr_*; tuning fields ignored */
  float* rgb_out;         /* [height*width*3] device */
} swr_batch_job;
typedef struct swr_batch_opts {
  uint32_t wave_size;     /* paths in flight, 0 = 2^23 */
  uint32_t refill;        /* as in swr_render_opts, 0 = 8 */
  uint32_t flags;         /* SWR_BATCH_* */
  uint32_t shade_batch;   /* batched adjoint: as swr_render_opts.shade_batch */
} swr_batch_opts;
#define SWR_BATCH_NO_GRAPH 1u /* launch the shade/trace rounds directly instead of from a CUDA graph */

/* A batch context owns the shared wavefront buffers and the captured CUDA graph; reuse it across
 * calls. One host thread at a time. */
int swr_batch_create(swr_batch** out);
void swr_batch_destroy(swr_batch* batch);
int swr_render_batch(swr_batch* batch, const swr_batch_job* jobs, uint32_t num_jobs,
                     const swr_batch_opts* opts, void* stream);

/* Physical-mode parameters of a built scene (no rebuild): diffuse albedo per triangle
 * ([num_triangles*3], by global triangle id) and emitted radiance L_e per object ([num_objects*3];
 * only objects marked light_source emit). Device or host memory. No counterpart in the reference,
 * whose materials are per object and fixed at load time. */
int swr_scene_set_albedo(swr_scene* scene, const float* albedo, void* stream);
int swr_scene_set_emission(swr_scene* scene, const float* emission, void* stream);

/* Gradient of sum_p dl_dimage[p] . image[p] for the SWR_MODE_PHYSICAL image that swr_render
 * produces with the same scene, camera and opts (same seed = the same sampled paths), with respect
 * to the per-triangle albedo ([num_triangles*3] by triangle id) and the per-object emission
 * ([num_objects*3]). Each camera path is re-traced from its random-number counters (path replay)
 * instead of being stored by the primal render. Outputs are overwritten. Device buffers;
 * max_depth <= 16. No counterpart in the reference (it has no differentiable renderer). */
int swr_render_adjoint(swr_scene* scene, const swr_camera* cam, const swr_render_opts* opts,
                       const float* dl_dimage, float* dl_dalbedo, float* dl_demission, void* stream);
/* As swr_render_adjoint, also returning its device time in milliseconds (CUDA events). */
int swr_render_adjoint_timed(swr_scene* scene, const swr_camera* cam, const swr_render_opts* opts,
                             const float* dl_dimage, float* dl_dalbedo, float* dl_demission,
                             void* stream, double* device_ms);

/* Batched adjoint: swr_render_adjoint for many jobs in one persistent launch (after one camera
 * launch over all jobs' pixels). Each job's gradients equal swr_render_adjoint's for that job up
 * to the order of the float atomic sums. Every distinct gradient buffer is zeroed once; jobs that
 * name the same buffers (the same scene rendered from several cameras) add into them. Only
 * opts.refill of the batch options is used. No counterpart in the reference. */
typedef struct swr_adjoint_job {
  swr_scene* scene;
  swr_camera cam;
  swr_render_opts opts;       /* SWR_MODE_PHYSICAL, max_depth <= 16; tuning fields ignored */
  const float* dl_dimage;     /* [height*width*3] device */
  float* dl_dalbedo;          /* [num_triangles*3] device */
  float* dl_demission;        /* [num_objects*3] device */
} swr_adjoint_job;
int swr_render_adjoint_batch(swr_batch* batch, const swr_adjoint_job* jobs, uint32_t num_jobs,
                             const swr_batch_opts* opts, void* stream);

/* Allocation-free variant of swr_render. It has no counterpart in the reference (whose renderer
 * is a host-thread loop): it exists for callers that must not have a library allocate device
 * memory during the call, such as applications that give all device memory to their own pool
 * up front, or frame loops that cannot afford the device-wide synchronisation a cudaMalloc or
 * cudaFree can cause. It calls no allocator; its scratch is one 64 MiB file-scope device array
 * that every device holds from the moment it loads the library until the process exits.
 * Limits: rgb_out (and samples_out when SWR_RENDER_SAMPLES_OUT is set) must be device memory;
 * spp <= 2^21; wave_size <= 65536 (0 = 65536); block_size 0 or 256; trace_blocks 0; no flag other
 * than SWR_RENDER_SAMPLES_OUT; larger requests are rejected with SWR_ERR_UNSUPPORTED. Every call
 * looks up the array's device address (cudaGetSymbolAddress) with the scene's device current, so
 * a cudaDeviceReset by the application between calls leaves no stale address; the first call on a
 * device may load the module, so make it before capturing any stream on the device. All calls share the
 * one array, so calls that overlap on the GPU (other streams or host threads) race on it and must
 * be serialised by the caller. Results equal swr_render's for the same arguments. */
int swr_render_noalloc(swr_scene* scene, const swr_camera* cam, const swr_render_opts* opts,
                       float* rgb_out, float* samples_out, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Moving objects: the object transform of GraphicsObject::init (graphics_object.cpp:12-27,54-62)
 * and the BVH refit of BVH::rebuild (bounding_volume_hierachy.cpp:77-79,130-139) on the GPU. */

/* An object's placement: position, scale and the rotation quaternion (s, x, y, z) that a scene
 * file's rotation(axis_x, axis_y, axis_z, angle) gives (swr_rotation_from_axis_angle). */
typedef struct swr_object_transform {
  float position[3];
  float scale[3];
  float rotation[4];
} swr_object_transform;
/* InputEntry::getRotation (input_parser.cpp:20-26): s = cos(angle/2), (x,y,z) = sin(angle/2) *
 * axis/|axis|, each in double and rounded to float. */
int swr_rotation_from_axis_angle(const float axis[3], float angle, float out[4]);
/* The placements of a loaded host scene's objects, in object order ([num_objects]). */
int swr_host_scene_transforms(const swr_host_scene* hs, swr_object_transform* out);
/* A scene built from a loaded host scene (as swr_scene_create on its descriptor) that also keeps
 * the object-space meshes on the device, so that swr_scene_set_transforms can move its objects. */
int swr_scene_create_from_host(const swr_host_scene* hs, const swr_build_opts* opts, swr_scene** out);
/* New placements for every object of a scene made by swr_scene_create_from_host: each object's
 * world vertices and normals are recomputed on the GPU from its object-space mesh (M = S*R*T,
 * row vectors, the reference's float order of operations), then the triangle records, the
 * reference's triangle and object boxes, the light tables and the tie ranks (the scene-level
 * order of the moved objects' boxes) are rederived and the BVH is refit in place (topology kept,
 * boxes recomputed bottom-up and requantised). Hits and renders afterwards equal those of a scene
 * loaded from a file with the same placements. The host computes the objects' order while the GPU
 * rederives and refits; the call returns once its work on stream has finished. xf: [num_objects],
 * host memory. Placements whose products overflow to a non-finite world coordinate or normal (in
 * any vertex, not only where the reference's boxes would show it) fail with SWR_ERR_INVALID and
 * leave the scene unusable until a call with valid placements succeeds. */
int swr_scene_set_transforms(swr_scene* scene, const swr_object_transform* xf, uint32_t num_objects,
                             void* stream);

/* ---------------------------------------------------------------------------------------------
 * The Vulkan application's PathTracer and denoisers (the RayTrace program: src/main.cpp:58-76,
 * src/graphic/renderer/path_tracer.cpp, src/graphic/denoiser/gauss_denoiser.cpp and
 * median_denoiser.cpp, and their shaders
 * res/shader/path_tracer_vision_raygen.rgen, path_tracer.glsl, v1.glsl, helper.glsl,
 * v1_closesthit.rchit, v1_miss.rmiss, denoise_gauss_comp.comp, denoise_median_comp.comp),
 * restated as CUDA kernels over a built scene. No graphics API is involved. Where GLSL leaves
 * precision to the implementation (division, sqrt, sin, cos, acos, normalize, multiply-add
 * fusion) one IEEE choice is fixed; the same choice is made by the CPU restatement the tests use.
 */

/* traceRay's closest hit (v1.glsl:148-161; the pipeline's opaque triangle query): the smallest
 * ray parameter t in [0.001, 10000], ties to the lower triangle id, with this library's
 * Moller-Trumbore arithmetic. Rays and hits as in swr_trace_closest; dist2 is not computed
 * (+inf). */
int swr_rt_trace_closest(swr_scene* scene, const float* ray_o, const float* ray_d, uint64_t n,
                         swr_hit* out, void* stream);

typedef struct swr_rt_opts {
  uint32_t width, height;  /* launch size = image size */
  uint32_t vision_jumps;   /* visionJumpCount (path_tracer.cpp:30-33), <= 65536 */
  uint32_t spp;            /* visionRayPerPixelCount, 1..2^24 */
  uint32_t refill;         /* idle lanes of a warp that take new pixels (1..32), 0 = 4 */
  uint32_t shade_batch;    /* lanes of a warp with a finished ray that shade together (1..32; fewer
                              when no ray of the warp is in flight), 0 = 12 */
  uint32_t blocks_per_sm;  /* resident blocks per SM targeted by the register budget: 0 (compiler's
                              choice), 5 or 6 */
  uint32_t reserved;
} swr_rt_opts;

/* One PathTracer frame (path_tracer_vision_raygen.rgen:8-60): per pixel the LCG random numbers
 * of helper.glsl seeded by the launch id, the camera ray of getVisionRay, traceRay with up to four
 * back-face retries, and visionRayPerPixelCount paths of up to visionJumpCount-1 jumps that count
 * when they reach a light from its front; lights seen directly give color * lightStrength.
 * rgb_out [height*width*3] receives finalColor (optional), rgba8_out [height*width*4] the rgba8
 * texel the shader stores (optional; clamp, *255, round to nearest even; alpha 0). Device or host
 * memory. The camera is a swr_camera (the RayTrace camera file has the same keys). */
int swr_rt_render(swr_scene* scene, const swr_camera* cam, const swr_rt_opts* opts, float* rgb_out,
                  uint8_t* rgba8_out, void* stream);

/* GaussDenoiser weights (gauss_denoiser.cpp:31-46): w[i] = exp(-(i - (k-1))^2 / (2 sigma^2)),
 * normalised by their sum; exp is the double exp rounded to float. kernel_size odd, 1..19 (the
 * shader reads w[0..kernel_size-1] only for odd sizes; the weight array holds 20 floats);
 * sigma > 0. out[kernel_size], host memory. */
int swr_rt_gauss_weights(uint32_t kernel_size, float sigma, float* out);
/* denoise_gauss_comp.comp: out = sum over in-image offsets (x outer, y inner, -k/2..k/2) of
 * texel * w[x + k/2] * w[y + k/2], stored as rgba8. in and out are separate rgba8 images
 * [height*width*4], device or host memory. */
int swr_rt_denoise_gauss(const uint8_t* rgba8_in, uint8_t* rgba8_out, uint32_t width, uint32_t height,
                         uint32_t kernel_size, float sigma, void* stream);
/* denoise_median_comp.comp: per-channel median of the 3x3 neighbourhood. The shader leaves
 * texels outside the image undefined; here they count as 0. */
int swr_rt_denoise_median(const uint8_t* rgba8_in, uint8_t* rgba8_out, uint32_t width,
                          uint32_t height, void* stream);

/* Renderer file of the RayTrace program (src/main.cpp:153-168): the first entry names the
 * renderer (PathTracer: visionJumpCount, visionRayPerPixelCount), every further entry a denoiser
 * applied in file order (GaussDenoiser: kernelSize, sigma; MedianDenoiser). The program's other
 * renderers are reported as SWR_ERR_UNSUPPORTED, unknown names as in getRenderer/getDenoiser. */
enum { SWR_DENOISER_GAUSS = 1, SWR_DENOISER_MEDIAN = 2 };
#define SWR_RT_MAX_DENOISERS 8
typedef struct swr_rt_denoiser {
  uint32_t kind;         /* SWR_DENOISER_* */
  uint32_t kernel_size;  /* Gauss: kernelSize */
  float sigma;           /* Gauss: sigma */
  uint32_t reserved;
} swr_rt_denoiser;
typedef struct swr_rt_renderer_params {
  uint32_t vision_jumps;
  uint32_t spp;
  uint32_t num_denoisers;
  uint32_t reserved;
  swr_rt_denoiser denoisers[SWR_RT_MAX_DENOISERS];
} swr_rt_renderer_params;
int swr_rt_renderer_load(const char* renderer_path, swr_rt_renderer_params* out);

/* One frame of GraphicsEngine::render (src/graphic/graphics_engine.cpp:30-70): the PathTracer
 * image, then each denoiser reading the previous image; rgba8_out receives the last image.
 * The denoisers' intermediate images and the device copy of a host rgba8_out live in a buffer the
 * scene keeps (grown by the first call that needs more), so frame loops allocate nothing per
 * frame; as the render workspace, it is the scene's, so one scene renders on one stream at a time
 * (swr_rt_render's host outputs use it too). */
int swr_rt_render_frame(swr_scene* scene, const swr_camera* cam, const swr_rt_opts* opts,
                        const swr_rt_denoiser* denoisers, uint32_t num_denoisers,
                        uint8_t* rgba8_out, void* stream);

/* Reference-style 8-bit quantisation (graphics_engine.cpp:90-95: clamp to [0,1], *255, truncate)
 * and P6 PPM writer (graphics_engine.cpp:32-40). Host memory. */
int swr_quantize_rgb8(const float* rgb, uint32_t width, uint32_t height, uint8_t* out);
int swr_write_ppm(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height);
/* The same 8-bit RGB image as PNG (8-bit RGB, uncompressed deflate blocks); the thesis tooling
 * converts the reference's PPM outputs to PNG for its comparisons. Host memory. */
int swr_write_png(const char* path, const uint8_t* rgb8, uint32_t width, uint32_t height);

#ifdef __cplusplus
}
#endif

#endif /* SWR_H */
