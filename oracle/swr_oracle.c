/* TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's SoftwareRenderer path tracer,
 * used as the checker of the parity tests (and nowhere else).
 *
 * Compiled with -ffp-contract=off so every float operation rounds once, as in the reference's
 * x86-64 build. Sources restated:
 *   closest hit      software_renderer/graphic/scene.cpp:22-56, graphic/graphics_object.cpp:64-87,
 *                    graphic/triangle.cpp:21-55, math/aabb.cpp:39-53, math/ray.cpp:4-5
 *   bounce loop      software_renderer/graphic/path_tracer.cpp:18-97
 *   sampling         software_renderer/math/random.cpp:16-35 (draws from Philox, see philox.h)
 *   reflect/refract  software_renderer/math/vector.h:319-345
 * The closest hit is found by brute force: every triangle, in the reference's visit order, that
 * passes the reference's slab test on its object box and on its own box is intersected, and the
 * first strictly smaller squared distance wins - which is what the reference's BVH walk computes,
 * since a BVH node's box contains its children's boxes and its slab test is monotone in the box.
 */
#include "swr_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "philox.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846 /* the same double as glibc's M_PI */
#endif

/* exported for known-answer tests of the generator */
void swo_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  swo_philox4x32_10(ctr, key, out);
}

typedef struct {
  float x, y, z;
} v3f;

static v3f mk(float x, float y, float z) {
  v3f r = {x, y, z};
  return r;
}
static v3f add(v3f a, v3f b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3f sub(v3f a, v3f b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static v3f scl(float s, v3f a) { return mk(s * a.x, s * a.y, s * a.z); }
static float dot(v3f a, v3f b) {
  float s = 0.0f;
  s += a.x * b.x;
  s += a.y * b.y;
  s += a.z * b.z;
  return s;
}
static v3f cross(v3f a, v3f b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static v3f normalize(v3f a) {
  double m = sqrt((double)dot(a, a));
  if (m != 0) {
    double f = 1.0 / m;
    a.x = (float)((double)a.x * f);
    a.y = (float)((double)a.y * f);
    a.z = (float)((double)a.z * f);
  }
  return a;
}
static v3f ld3(const float* p) { return mk(p[0], p[1], p[2]); }

/* aabb.cpp:39-53 with std::min(a,b) = b<a?b:a and std::max(a,b) = a<b?b:a */
static int ref_slab(const float* box, const float o[3], const float inv[3]) {
  float tmin = 0.0f, tmax = INFINITY;
  int i;
  for (i = 0; i < 3; ++i) {
    float t1 = (box[i] - o[i]) * inv[i];
    float t2 = (box[3 + i] - o[i]) * inv[i];
    float mn = (t2 < t1) ? t2 : t1;
    float mx = (t1 < t2) ? t2 : t1;
    tmin = (tmin < mn) ? mn : tmin;
    tmax = (mx < tmax) ? mx : tmax;
  }
  return tmin < tmax;
}

/* triangle.cpp:21-45 and the distance key of graphics_object.cpp:77 */
static int ref_intersect(v3f o, v3f d, v3f v0, v3f e0, v3f e1, float* t_out, float* d2_out) {
  const float EPS = 0.0000001f;
  v3f h = cross(d, e1);
  float a = dot(e0, h);
  float f, u, v, t;
  v3f s, q, p, w;
  if (a > -EPS && a < EPS) return 0;
  f = 1.0f / a;
  s = sub(o, v0);
  u = f * dot(s, h);
  if (u < 0.0f || u > 1.0f) return 0;
  q = cross(s, e0);
  v = f * dot(d, q);
  if (v < 0.0f || u + v > 1.0f) return 0;
  t = f * dot(e1, q);
  if (!(t > EPS)) return 0;
  p = add(o, scl(t, d));
  w = sub(o, p);
  *t_out = t;
  *d2_out = dot(w, w);
  return 1;
}

static uint32_t closest(const swo_scene* s, v3f o, v3f d, float* t_out, float* d2_out) {
  const float ov[3] = {o.x, o.y, o.z};
  const float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  float best = INFINITY, bt = INFINITY;
  uint32_t bi = 0xFFFFFFFFu;
  uint32_t k = 0;
  while (k < s->ntri) {
    const uint32_t obj = s->tri_obj[s->visit[k]];
    const uint32_t n = s->obj_first[obj + 1] - s->obj_first[obj];
    if (!ref_slab(s->obj_box + 6 * (size_t)obj, ov, inv)) {
      k += n;
      continue;
    }
    const uint32_t end = k + n;
    for (; k < end; ++k) {
      const uint32_t t = s->visit[k];
      float tt, d2;
      if (!ref_slab(s->tri_box + 6 * (size_t)t, ov, inv)) continue;
      if (!ref_intersect(o, d, ld3(s->v0 + 3 * (size_t)t), ld3(s->e0 + 3 * (size_t)t),
                         ld3(s->e1 + 3 * (size_t)t), &tt, &d2))
        continue;
      if (d2 < best) {
        best = d2;
        bt = tt;
        bi = t;
      }
    }
  }
  *t_out = bt;
  *d2_out = best;
  return bi;
}

/* scene.cpp:43-53: barycentric interpolation of the corner normals, then the double normalize */
static v3f shading_normal(const swo_scene* s, uint32_t t, v3f p) {
  const float* den = s->den + 4 * (size_t)t;
  v3f v0 = ld3(s->v0 + 3 * (size_t)t), e0 = ld3(s->e0 + 3 * (size_t)t), e1 = ld3(s->e1 + 3 * (size_t)t);
  v3f e2 = sub(p, v0);
  float d20 = dot(e2, e0), d21 = dot(e2, e1);
  float v = (den[2] * d20 - den[1] * d21) / den[3];
  float w = (den[0] * d21 - den[1] * d20) / den[3];
  float u = 1.0f - v - w;
  const float* nn = s->nrm + 9 * (size_t)t;
  v3f n = mk(0.0f, 0.0f, 0.0f);
  n = add(n, scl(u, ld3(nn)));
  n = add(n, scl(v, ld3(nn + 3)));
  n = add(n, scl(w, ld3(nn + 6)));
  return normalize(n);
}

static v3f hemisphere(v3f n, float u1, float u2) {
  float theta = (float)(2.0 * M_PI * (double)u1);
  float u = 2.0f * u2 - 1.0f;
  float suu = sqrtf(1.0f - u * u);
  float st = (float)sin((double)theta), ct = (float)cos((double)theta);
  v3f r = mk(suu * ct, suu * st, u);
  if (dot(r, n) < 0.0f) r = mk(-r.x, -r.y, -r.z);
  return r;
}

static v3f reflect_f(v3f I, v3f N) {
  double s = 2.0 * (double)dot(N, I);
  return mk(I.x - (float)(s * (double)N.x), I.y - (float)(s * (double)N.y),
            I.z - (float)(s * (double)N.z));
}

static v3f refract_f(v3f I, v3f N, float eta) {
  float ndi = dot(N, I);
  float k = (float)(1.0 - (double)(eta * eta) * (1.0 - (double)(ndi * ndi)));
  double sc;
  if (k < 0.0) return mk(0.0f, 0.0f, 0.0f);
  sc = (double)(eta * ndi) + sqrt((double)k);
  return mk(eta * I.x - (float)(sc * (double)N.x), eta * I.y - (float)(sc * (double)N.y),
            eta * I.z - (float)(sc * (double)N.z));
}

static v3f custom_refract_f(v3f I, v3f N, float eta) {
  float angle;
  if ((double)dot(N, I) > 0.0) N = mk(-N.x, -N.y, -N.z);
  else eta = (float)(1.0 / (double)eta);
  angle = (float)(sin(acos((double)dot(N, I))) * (double)eta);
  if (-1.0 < angle && angle < 1.0) return refract_f(I, N, eta);
  return reflect_f(I, N);
}

/* path_tracer.cpp:19-23 */
static v3f primary_dir(const swo_camera* c, uint32_t px, uint32_t py, uint32_t W, uint32_t H) {
  float cx = (float)px + 0.5f, cy = (float)py + 0.5f;
  float ux = cx / (float)W, uy = cy / (float)H;
  float in4[4] = {2.0f * ux - 1.0f, 2.0f * uy - 1.0f, 1.0f, 1.0f};
  float r[4] = {0, 0, 0, 0}, q[4] = {0, 0, 0, 0};
  int i, j;
  v3f t;
  float w4[4];
  for (i = 0; i < 4; ++i)
    for (j = 0; j < 4; ++j) r[j] += c->pi[i * 4 + j] * in4[i];
  t = normalize(mk(r[0], r[1], r[2]));
  w4[0] = t.x;
  w4[1] = t.y;
  w4[2] = t.z;
  w4[3] = 0.0f;
  for (i = 0; i < 4; ++i)
    for (j = 0; j < 4; ++j) q[j] += c->vi[i * 4 + j] * w4[i];
  return normalize(mk(q[0], q[1], q[2]));
}

/* one sample of PathTracer::traceSinglePath; returns 1 when the path ended on a light */
static int trace_single_path(const swo_scene* s, v3f o, v3f d, uint32_t depth, uint64_t seed,
                             uint32_t pixel, uint32_t sample, v3f* color) {
  v3f c = mk(1.0f, 1.0f, 1.0f);
  int backface = 1;
  uint32_t vtx = 0, i;
  for (i = 0; i < depth; ++i) {
    float t, d2, u[4], r;
    uint32_t tri = closest(s, o, d, &t, &d2), obj;
    v3f p, n, nd, prev;
    const float* m;
    if (tri == 0xFFFFFFFFu) break;
    p = add(o, scl(t, d));
    n = shading_normal(s, tri, p);
    if (backface && dot(n, d) > 0.0f) {
      o = add(p, scl(0.01f, d));
      continue;
    }
    backface = 0;
    swo_vertex_uniforms(seed, pixel, sample, vtx++, 0, u);
    r = u[0];
    obj = s->tri_obj[tri];
    m = s->mats + 9 * (size_t)obj;
    prev = d;
    nd = d;
    if (r <= m[3]) nd = hemisphere(n, u[1], u[2]);
    else if (r <= m[4]) nd = reflect_f(d, n);
    else if (r <= m[5]) nd = custom_refract_f(d, n, m[6]);
    o = add(p, scl(0.01f, nd));
    d = nd;
    if (r <= m[3]) {
      float cs = dot(n, d);
      c = mk(c.x * (m[0] * cs), c.y * (m[1] * cs), c.z * (m[2] * cs));
    }
    if (m[7] != 0.0f && dot(n, prev) <= 0.0f) {
      *color = c;
      return 1;
    }
  }
  *color = c;
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * threading */
typedef struct {
  void (*fn)(void* ctx, uint64_t begin, uint64_t end);
  void* ctx;
  uint64_t n, chunk;
  uint64_t next;
  pthread_mutex_t mu;
} pool_t;

static void* pool_worker(void* arg) {
  pool_t* p = (pool_t*)arg;
  for (;;) {
    uint64_t b;
    pthread_mutex_lock(&p->mu);
    b = p->next;
    p->next += p->chunk;
    pthread_mutex_unlock(&p->mu);
    if (b >= p->n) break;
    p->fn(p->ctx, b, b + p->chunk < p->n ? b + p->chunk : p->n);
  }
  return NULL;
}

static void parallel_for(uint64_t n, uint64_t chunk, int threads,
                         void (*fn)(void*, uint64_t, uint64_t), void* ctx) {
  pool_t p;
  pthread_t th[256];
  int i;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  p.fn = fn;
  p.ctx = ctx;
  p.n = n;
  p.chunk = chunk ? chunk : 1;
  p.next = 0;
  pthread_mutex_init(&p.mu, NULL);
  for (i = 0; i < threads; ++i) pthread_create(&th[i], NULL, pool_worker, &p);
  for (i = 0; i < threads; ++i) pthread_join(th[i], NULL);
  pthread_mutex_destroy(&p.mu);
}

/* ---------------------------------------------------------------------------------------------
 * closest hit */
typedef struct {
  const swo_scene* s;
  const float *ro, *rd;
  uint32_t* tri;
  float *d2, *t;
} trace_ctx;

static void trace_range(void* c_, uint64_t b, uint64_t e) {
  trace_ctx* c = (trace_ctx*)c_;
  uint64_t i;
  for (i = b; i < e; ++i) {
    float t, d2;
    c->tri[i] = closest(c->s, ld3(c->ro + 4 * i), ld3(c->rd + 4 * i), &t, &d2);
    if (c->d2) c->d2[i] = d2;
    if (c->t) c->t[i] = t;
  }
}

void swo_trace(const swo_scene* s, const float* ro, const float* rd, uint64_t n, uint32_t* hit_tri,
               float* hit_d2, float* hit_t, int threads) {
  trace_ctx c = {s, ro, rd, hit_tri, hit_d2, hit_t};
  parallel_for(n, 256, threads, trace_range, &c);
}

/* ---------------------------------------------------------------------------------------------
 * reference-mode render */
typedef struct {
  const swo_scene* s;
  const swo_camera* cam;
  uint32_t W, H, spp, depth, p0;
  uint64_t seed;
  float *per_sample, *per_pixel;
  uint32_t s0, spp_total; /* samples [s0, s0 + spp) of an image with spp_total samples per pixel */
} render_ctx;

static void render_range(void* c_, uint64_t b, uint64_t e) {
  render_ctx* c = (render_ctx*)c_;
  uint64_t k;
  for (k = b; k < e; ++k) {
    uint32_t pix = c->p0 + (uint32_t)k, smp;
    v3f d = primary_dir(c->cam, pix % c->W, pix / c->W, c->W, c->H);
    v3f o = ld3(c->cam->org);
    float fr = 0.0f, fg = 0.0f, fb = 0.0f;
    double sc;
    for (smp = 0; smp < c->spp; ++smp) {
      v3f col;
      int lit = trace_single_path(c->s, o, d, c->depth, c->seed, pix, c->s0 + smp, &col);
      float* ps = c->per_sample ? c->per_sample + (k * c->spp + smp) * 4 : NULL;
      if (lit) {
        fr += col.x;
        fg += col.y;
        fb += col.z;
      }
      if (ps) {
        ps[0] = lit ? col.x : 0.0f;
        ps[1] = lit ? col.y : 0.0f;
        ps[2] = lit ? col.z : 0.0f;
        ps[3] = lit ? 1.0f : 0.0f;
      }
    }
    sc = 2.0 * M_PI * (double)(1.0f / (float)c->spp_total);
    c->per_pixel[3 * k + 0] = (float)((double)fr * sc);
    c->per_pixel[3 * k + 1] = (float)((double)fg * sc);
    c->per_pixel[3 * k + 2] = (float)((double)fb * sc);
  }
}

void swo_render_reference(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                          uint32_t spp, uint32_t depth, uint64_t seed, uint32_t p0, uint32_t p1,
                          float* per_sample, float* per_pixel, int threads) {
  swo_render_reference_part(s, cam, W, H, spp, 0, spp, depth, seed, p0, p1, per_sample, per_pixel, threads);
}

void swo_render_reference_part(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                               uint32_t spp_total, uint32_t s0, uint32_t s1, uint32_t depth, uint64_t seed,
                               uint32_t p0, uint32_t p1, float* per_sample, float* per_pixel, int threads) {
  render_ctx c = {s, cam, W, H, s1 - s0, depth, p0, seed, per_sample, per_pixel, s0, spp_total};
  parallel_for(p1 - p0, 4, threads, render_range, &c);
}

/* ---------------------------------------------------------------------------------------------
 * bidirectional path tracer (bidirectional_path_tracer.cpp:20-168, scene.cpp:58-83) */

/* Scene::isOccluded: a candidate hit (the closest-hit rules) no farther than the end point */
static int occluded(const swo_scene* s, v3f a, v3f b) {
  v3f d = sub(b, a);
  float dist2 = dot(d, d), t, d2;
  uint32_t tri;
  d = normalize(d);
  tri = closest(s, a, d, &t, &d2);
  return tri != 0xFFFFFFFFu && d2 <= dist2;
}

typedef struct {
  v3f pos, nrm, col;
  int light_hit;
} hitpoint_t;

/* BidirectionalPathTracer::traceSinglePath for slots [start, end); returns the path depth */
static uint32_t bdpt_trace(const swo_scene* s, hitpoint_t* path, v3f o, v3f d, uint32_t start, uint32_t end,
                           int light_ray, uint64_t seed, uint32_t pixel, uint32_t sample, uint32_t* draws) {
  v3f c = mk(1.0f, 1.0f, 1.0f);
  uint32_t depth = 0, i;
  int backface = !light_ray;
  for (i = start; i < end; ++i) {
    float t, d2, u[4], r;
    uint32_t tri = closest(s, o, d, &t, &d2), obj;
    v3f p, n, nd, prev;
    const float* m;
    if (tri == 0xFFFFFFFFu) break;
    p = add(o, scl(t, d));
    n = shading_normal(s, tri, p);
    if (backface && dot(n, d) > 0.0f) {
      o = add(p, scl(0.01f, d));
      continue;
    }
    backface = 0;
    depth = i + 1;
    swo_vertex_uniforms(seed, pixel, sample, (*draws)++, 0, u);
    r = u[0];
    obj = s->tri_obj[tri];
    m = s->mats + 9 * (size_t)obj;
    prev = d;
    nd = d;
    if (r <= m[3]) nd = hemisphere(n, u[1], u[2]);
    else if (r <= m[4]) nd = reflect_f(d, n);
    else if (r <= m[5]) nd = custom_refract_f(d, n, m[6]);
    o = add(p, scl(0.01f, nd));
    d = nd;
    if (r <= m[3]) {
      float cs = dot(n, light_ray ? prev : d);
      c = mk(c.x * (m[0] * cs), c.y * (m[1] * cs), c.z * (m[2] * cs));
    }
    path[i].pos = p;
    path[i].nrm = n;
    path[i].col = c;
    path[i].light_hit = 0;
    if (m[7] != 0.0f && dot(n, prev) <= 0.0f) {
      path[i].light_hit = 1;
      break;
    }
  }
  return depth;
}

/* one sample of BidirectionalPathTracer::renderPixel before the 2 pi / spp scale; returns 1 when
 * the sample added anything (a light hit or a connection pass) */
static v3f bdpt_sample(const swo_scene* s, v3f org, v3f dir, uint32_t vj, uint32_t lj, uint32_t md,
                       const uint32_t* lights, uint32_t nlights, uint64_t seed, uint32_t pixel,
                       uint32_t sample) {
  hitpoint_t V[32], L[32];
  uint32_t draws = 0, dv, dl, vi, li, light, ti, nt;
  float u[4], sr1, r2, b0, b1, b2;
  v3f color = mk(0.0f, 0.0f, 0.0f), lp, ln, ld;
  const float *vt, *nn;
  memset(V, 0, sizeof(V));  /* the reference's value-initialised hit points */
  memset(L, 0, sizeof(L));
  dv = bdpt_trace(s, V, org, dir, 0, vj, 0, seed, pixel, sample, &draws);
  if (dv == 0) return color;
  if (V[dv - 1].light_hit) return V[dv - 1].col;
  /* getRandomLightSourcePoint (bidirectional_path_tracer.cpp:140-168) */
  swo_vertex_uniforms(seed, pixel, sample, draws++, 0, u);
  light = (uint32_t)(u[0] * (float)nlights);
  if (light >= nlights) light = nlights - 1;
  swo_vertex_uniforms(seed, pixel, sample, draws++, 0, u);
  sr1 = sqrtf(u[0]);
  swo_vertex_uniforms(seed, pixel, sample, draws++, 0, u);
  r2 = u[0];
  swo_vertex_uniforms(seed, pixel, sample, draws++, 0, u);
  nt = s->obj_first[lights[light] + 1] - s->obj_first[lights[light]];
  ti = (uint32_t)(u[0] * (float)nt);
  if (ti >= nt) ti = nt - 1;
  ti += s->obj_first[lights[light]];
  b0 = 1.0f - sr1;
  b1 = sr1 * (1.0f - r2);
  b2 = sr1 * r2;
  vt = s->vtx + 9 * (size_t)ti;
  nn = s->nrm + 9 * (size_t)ti;
  lp = add(add(scl(b0, ld3(vt)), scl(b1, ld3(vt + 3))), scl(b2, ld3(vt + 6)));
  ln = mk(0.0f, 0.0f, 0.0f);
  ln = add(ln, scl(b0, ld3(nn)));
  ln = add(ln, scl(b1, ld3(nn + 3)));
  ln = add(ln, scl(b2, ld3(nn + 6)));
  ln = normalize(ln);
  ld = hemisphere(ln, u[1], u[2]);
  L[0].pos = lp;
  L[0].nrm = ln;
  L[0].col = ld3(s->mats + 9 * (size_t)lights[light]);
  dl = bdpt_trace(s, L, lp, ld, 1, lj, 1, seed, pixel, sample, &draws);
  for (vi = 0; vi < dv; ++vi)
    for (li = 0; li < dl; ++li) {
      v3f a, b, d;
      float cs;
      if (vi + li > md) continue;
      a = add(V[vi].pos, scl(0.01f, V[vi].nrm));
      b = add(L[li].pos, scl(0.01f, L[li].nrm));
      if (occluded(s, a, b)) continue;
      d = normalize(sub(b, a));
      cs = dot(d, V[vi].nrm);
      color = add(color, mk(V[vi].col.x * L[li].col.x * cs, V[vi].col.y * L[li].col.y * cs,
                            V[vi].col.z * L[li].col.z * cs));
    }
  return scl(1.0f / (float)md, color);
}

typedef struct {
  const swo_scene* s;
  const swo_camera* cam;
  uint32_t W, H, spp, vj, lj, md, p0;
  uint64_t seed;
  const uint32_t* lights;
  uint32_t nlights;
  float *per_sample, *per_pixel;
} bdpt_ctx;

static void bdpt_range(void* c_, uint64_t b, uint64_t e) {
  bdpt_ctx* c = (bdpt_ctx*)c_;
  uint64_t k;
  for (k = b; k < e; ++k) {
    uint32_t pix = c->p0 + (uint32_t)k, smp;
    v3f d = primary_dir(c->cam, pix % c->W, pix / c->W, c->W, c->H);
    v3f o = ld3(c->cam->org);
    v3f f = mk(0.0f, 0.0f, 0.0f);
    double sc;
    for (smp = 0; smp < c->spp; ++smp) {
      v3f col = bdpt_sample(c->s, o, d, c->vj, c->lj, c->md, c->lights, c->nlights, c->seed, pix, smp);
      float* ps = c->per_sample ? c->per_sample + (k * c->spp + smp) * 4 : NULL;
      f = add(f, col);
      if (ps) {
        ps[0] = col.x;
        ps[1] = col.y;
        ps[2] = col.z;
        ps[3] = 1.0f;
      }
    }
    sc = 2.0 * M_PI * (double)(1.0f / (float)c->spp);
    c->per_pixel[3 * k + 0] = (float)((double)f.x * sc);
    c->per_pixel[3 * k + 1] = (float)((double)f.y * sc);
    c->per_pixel[3 * k + 2] = (float)((double)f.z * sc);
  }
}

int swo_render_bdpt(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H, uint32_t spp,
                    uint32_t vision_jumps, uint32_t light_jumps, uint32_t max_depth, uint64_t seed,
                    uint32_t p0, uint32_t p1, float* per_sample, float* per_pixel, int threads) {
  bdpt_ctx c;
  uint32_t* lights;
  uint32_t o, n = 0;
  if (!s->vtx || vision_jumps > 32 || light_jumps > 32 || max_depth == 0) return -1;
  lights = (uint32_t*)malloc(sizeof(uint32_t) * (s->nobj ? s->nobj : 1));
  for (o = 0; o < s->nobj; ++o)
    if (s->mats[9 * (size_t)o + 7] != 0.0f) lights[n++] = o;
  if (n == 0) {
    free(lights);
    return -2;
  }
  c.s = s;
  c.cam = cam;
  c.W = W;
  c.H = H;
  c.spp = spp;
  c.vj = vision_jumps;
  c.lj = light_jumps;
  c.md = max_depth;
  c.p0 = p0;
  c.seed = seed;
  c.lights = lights;
  c.nlights = n;
  c.per_sample = per_sample;
  c.per_pixel = per_pixel;
  parallel_for(p1 - p0, 4, threads, bdpt_range, &c);
  free(lights);
  return 0;
}

/* ---------------------------------------------------------------------------------------------
 * physical mode in double. Hits are chosen with the reference's float rules (the same triangle
 * the renderer finds); positions, normals, directions, throughput and sums are carried in double. */
typedef struct {
  double x, y, z;
} v3d;
static v3d dk(double x, double y, double z) {
  v3d r = {x, y, z};
  return r;
}
static double ddot(v3d a, v3d b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static v3d dadd(v3d a, v3d b) { return dk(a.x + b.x, a.y + b.y, a.z + b.z); }
static v3d dscl(double s, v3d a) { return dk(s * a.x, s * a.y, s * a.z); }
static v3d dnorm(v3d a) {
  double m = sqrt(ddot(a, a));
  return m > 0 ? dscl(1.0 / m, a) : a;
}
static v3d tod(v3f a) { return dk(a.x, a.y, a.z); }
static v3f tof(v3d a) { return mk((float)a.x, (float)a.y, (float)a.z); }

static v3d normal64(const swo_scene* s, uint32_t t, v3d p) {
  const float* den = s->den + 4 * (size_t)t;
  v3d v0 = tod(ld3(s->v0 + 3 * (size_t)t)), e0 = tod(ld3(s->e0 + 3 * (size_t)t)),
      e1 = tod(ld3(s->e1 + 3 * (size_t)t));
  v3d e2 = dk(p.x - v0.x, p.y - v0.y, p.z - v0.z);
  double d00 = ddot(e0, e0), d01 = ddot(e0, e1), d11 = ddot(e1, e1);
  double dn = d00 * d11 - d01 * d01;
  double d20 = ddot(e2, e0), d21 = ddot(e2, e1);
  double v = (d11 * d20 - d01 * d21) / dn, w = (d00 * d21 - d01 * d20) / dn, u = 1.0 - v - w;
  const float* nn = s->nrm + 9 * (size_t)t;
  (void)den;
  return dnorm(dadd(dadd(dscl(u, tod(ld3(nn))), dscl(v, tod(ld3(nn + 3)))), dscl(w, tod(ld3(nn + 6)))));
}

static v3d reflect64(v3d I, v3d N) { return dadd(I, dscl(-2.0 * ddot(N, I), N)); }

static v3d custom_refract64(v3d I, v3d N, double eta) {
  double ndi, k, ang;
  if (ddot(N, I) > 0.0) N = dscl(-1.0, N);
  else eta = 1.0 / eta;
  ang = sin(acos(fmax(-1.0, fmin(1.0, ddot(N, I))))) * eta;
  if (!(-1.0 < ang && ang < 1.0)) return reflect64(I, N);
  ndi = ddot(N, I);
  k = 1.0 - eta * eta * (1.0 - ndi * ndi);
  if (k < 0.0) return dk(0, 0, 0);
  return dadd(dscl(eta, I), dscl(-(eta * ndi + sqrt(k)), N));
}

/* One physical-mode path. Records per scattering vertex the triangle, the throughput before the
 * vertex, the multiplier factor g (albedo excluded) and whether it was diffuse, so the adjoint can
 * sweep backwards. Returns the radiance. */
#define SWO_MAXV 32
typedef struct {
  uint32_t tri[SWO_MAXV];
  v3d c[SWO_MAXV];
  double g[SWO_MAXV];
  int diffuse[SWO_MAXV];
  double q[SWO_MAXV];
  int nv;
  int emit;         /* 1 when the path ended on an emitter hit from the front */
  uint32_t emit_obj;
  v3d c_emit;       /* throughput at the emitter */
} path64;

static v3d albedo_of(const swo_scene* s, uint32_t tri) {
  if (s->albedo) return tod(ld3(s->albedo + 3 * (size_t)tri));
  return tod(ld3(s->mats + 9 * (size_t)s->tri_obj[tri]));
}
static v3d emission_of(const swo_scene* s, uint32_t obj) {
  const float* m = s->mats + 9 * (size_t)obj;
  if (s->emission) return tod(ld3(s->emission + 3 * (size_t)obj));
  return dk((double)m[0] * m[8], (double)m[1] * m[8], (double)m[2] * m[8]);
}

static v3d path_physical64(const swo_scene* s, v3f of, v3f df, uint32_t depth, uint64_t seed,
                           uint32_t pixel, uint32_t sample, uint32_t rr_depth, double rr_q,
                           path64* rec) {
  v3d c = dk(1, 1, 1), L = dk(0, 0, 0);
  v3d o = tod(of), d = tod(df);
  int backface = 1;
  uint32_t vtx = 0, i;
  if (rec) {
    rec->nv = 0;
    rec->emit = 0;
  }
  for (i = 0; i < depth; ++i) {
    float t, d2, u[4];
    uint32_t tri = closest(s, tof(o), tof(d), &t, &d2), obj;
    v3d p, n, nd, prev;
    const float* m;
    int front;
    double r, g = 1.0, q = 1.0;
    int diff = 0;
    if (tri == 0xFFFFFFFFu) break;
    {
      /* hit position from the float intersection of the float ray, carried in double */
      v3f pf = add(tof(o), scl(t, tof(d)));
      p = tod(pf);
    }
    n = normal64(s, tri, p);
    if (backface && ddot(n, d) > 0.0) {
      o = dadd(p, dscl(0.01, d));
      continue;
    }
    backface = 0;
    obj = s->tri_obj[tri];
    m = s->mats + 9 * (size_t)obj;
    front = ddot(n, d) <= 0.0;
    prev = d;
    (void)prev;
    if (m[7] != 0.0f) {
      if (front) {
        v3d le = emission_of(s, obj);
        L = dadd(L, dk(c.x * le.x, c.y * le.y, c.z * le.z));
        if (rec) {
          rec->emit = 1;
          rec->emit_obj = obj;
          rec->c_emit = c;
        }
      }
      break;
    }
    swo_vertex_uniforms(seed, pixel, sample, vtx, 0, u);
    r = u[0];
    nd = d;
    if (r <= m[3]) {
      v3d ns = front ? n : dscl(-1.0, n);
      double th = 2.0 * M_PI * (double)u[1];
      double z = 2.0 * (double)u[2] - 1.0;
      double sq = sqrt(fmax(0.0, 1.0 - z * z));
      nd = dk(sq * cos(th), sq * sin(th), z);
      if (ddot(nd, ns) < 0.0) nd = dscl(-1.0, nd);
      g = 2.0 * ddot(ns, nd);
      diff = 1;
    } else if (r <= m[4]) {
      nd = reflect64(d, n);
    } else if (r <= m[5]) {
      nd = custom_refract64(d, n, (double)m[6]);
    }
    vtx += 1;
    if (rr_depth != 0 && vtx >= rr_depth) {
      if ((double)u[3] >= rr_q) {
        if (rec && rec->nv < SWO_MAXV) {
          /* the vertex scattered but the path was terminated: it carries no gradient */
        }
        break;
      }
      q = rr_q;
    }
    if (rec && rec->nv < SWO_MAXV) {
      rec->tri[rec->nv] = tri;
      rec->c[rec->nv] = c;
      rec->g[rec->nv] = g;
      rec->diffuse[rec->nv] = diff;
      rec->q[rec->nv] = q;
      rec->nv++;
    }
    if (diff) {
      v3d a = albedo_of(s, tri);
      c = dk(c.x * a.x * g / q, c.y * a.y * g / q, c.z * a.z * g / q);
    } else {
      c = dscl(1.0 / q, c);
    }
    o = dadd(p, dscl(0.01, nd));
    d = nd;
  }
  return L;
}

typedef struct {
  const swo_scene* s;
  const swo_camera* cam;
  uint32_t W, H, spp, depth, p0, rr_depth;
  double rr_q;
  uint64_t seed;
  double *pp, *var;
  uint32_t s0, spp_total; /* samples [s0, s0 + spp) of an image with spp_total samples per pixel */
} phys_ctx;

static void phys_range(void* c_, uint64_t b, uint64_t e) {
  phys_ctx* c = (phys_ctx*)c_;
  uint64_t k;
  for (k = b; k < e; ++k) {
    uint32_t pix = c->p0 + (uint32_t)k, smp;
    v3f d = primary_dir(c->cam, pix % c->W, pix / c->W, c->W, c->H);
    v3f o = ld3(c->cam->org);
    v3d sum = dk(0, 0, 0), sq = dk(0, 0, 0);
    for (smp = 0; smp < c->spp; ++smp) {
      v3d L = path_physical64(c->s, o, d, c->depth, c->seed, pix, c->s0 + smp, c->rr_depth, c->rr_q, NULL);
      sum = dadd(sum, L);
      sq = dadd(sq, dk(L.x * L.x, L.y * L.y, L.z * L.z));
    }
    {
      double n = (double)c->spp;
      v3d mean = dscl(1.0 / n, sum);
      v3d part = dscl(1.0 / (double)c->spp_total, sum);
      c->pp[3 * k + 0] = part.x;
      c->pp[3 * k + 1] = part.y;
      c->pp[3 * k + 2] = part.z;
      if (c->var) {
        double dn = n > 1 ? n * (n - 1.0) : 1.0;
        c->var[3 * k + 0] = fmax(0.0, sq.x - n * mean.x * mean.x) / dn;
        c->var[3 * k + 1] = fmax(0.0, sq.y - n * mean.y * mean.y) / dn;
        c->var[3 * k + 2] = fmax(0.0, sq.z - n * mean.z * mean.z) / dn;
      }
    }
  }
}

void swo_render_physical64(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                           uint32_t spp, uint32_t depth, uint64_t seed, uint32_t rr_depth,
                           double rr_q, uint32_t p0, uint32_t p1, double* per_pixel,
                           double* per_pixel_var, int threads) {
  swo_render_physical64_part(s, cam, W, H, spp, 0, spp, depth, seed, rr_depth, rr_q, p0, p1, per_pixel,
                             per_pixel_var, threads);
}

void swo_render_physical64_part(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                                uint32_t spp_total, uint32_t s0, uint32_t s1, uint32_t depth, uint64_t seed,
                                uint32_t rr_depth, double rr_q, uint32_t p0, uint32_t p1, double* per_pixel,
                                double* per_pixel_var, int threads) {
  phys_ctx c = {s, cam, W, H, s1 - s0, depth, p0, rr_depth, rr_q, seed, per_pixel, per_pixel_var, s0, spp_total};
  parallel_for(p1 - p0, 4, threads, phys_range, &c);
}

/* ---------------------------------------------------------------------------------------------
 * adjoint: for every path, sweep its vertices backwards. With S the radiance leaving vertex j+1
 * per unit throughput (S = L_e at the emitter, S_j = f_j * S_{j+1} with f_j = albedo*g/q for a
 * diffuse vertex and 1/q otherwise), dL/dalbedo(tri_j) = c_j * (g_j/q_j) * S_{j+1} and
 * dL/demission(obj) = c at the emitter. Per-thread accumulators are summed at the end. */
typedef struct {
  const swo_scene* s;
  const swo_camera* cam;
  uint32_t W, H, spp, depth, rr_depth;
  double rr_q;
  uint64_t seed;
  const float* dl;
  double *ga, *ge;
  pthread_mutex_t* mu;
  uint32_t s0, spp_total; /* samples [s0, s0 + spp) of an image with spp_total samples per pixel */
} adj_ctx;

static void adj_range(void* c_, uint64_t b, uint64_t e) {
  adj_ctx* c = (adj_ctx*)c_;
  const swo_scene* s = c->s;
  double* ga = (double*)calloc((size_t)s->ntri * 3, sizeof(double));
  double* ge = (double*)calloc((size_t)s->nobj * 3, sizeof(double));
  uint64_t k;
  path64 rec;
  for (k = b; k < e; ++k) {
    uint32_t pix = (uint32_t)k, smp;
    v3f d = primary_dir(c->cam, pix % c->W, pix / c->W, c->W, c->H);
    v3f o = ld3(c->cam->org);
    const double w = 1.0 / (double)c->spp_total;
    v3d dl = dk(c->dl[3 * k] * w, c->dl[3 * k + 1] * w, c->dl[3 * k + 2] * w);
    for (smp = 0; smp < c->spp; ++smp) {
      v3d S;
      int j;
      path_physical64(s, o, d, c->depth, c->seed, pix, c->s0 + smp, c->rr_depth, c->rr_q, &rec);
      if (!rec.emit) continue;
      {
        uint32_t ob = rec.emit_obj;
        ge[3 * ob + 0] += dl.x * rec.c_emit.x;
        ge[3 * ob + 1] += dl.y * rec.c_emit.y;
        ge[3 * ob + 2] += dl.z * rec.c_emit.z;
        S = emission_of(s, ob);
      }
      for (j = rec.nv - 1; j >= 0; --j) {
        uint32_t t = rec.tri[j];
        if (rec.diffuse[j]) {
          v3d a = albedo_of(s, t);
          double gq = rec.g[j] / rec.q[j];
          ga[3 * t + 0] += dl.x * rec.c[j].x * gq * S.x;
          ga[3 * t + 1] += dl.y * rec.c[j].y * gq * S.y;
          ga[3 * t + 2] += dl.z * rec.c[j].z * gq * S.z;
          S = dk(S.x * a.x * gq, S.y * a.y * gq, S.z * a.z * gq);
        } else {
          S = dscl(1.0 / rec.q[j], S);
        }
      }
    }
  }
  pthread_mutex_lock(c->mu);
  for (k = 0; k < (uint64_t)s->ntri * 3; ++k) c->ga[k] += ga[k];
  for (k = 0; k < (uint64_t)s->nobj * 3; ++k) c->ge[k] += ge[k];
  pthread_mutex_unlock(c->mu);
  free(ga);
  free(ge);
}

void swo_adjoint_physical64(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                            uint32_t spp, uint32_t depth, uint64_t seed, uint32_t rr_depth,
                            double rr_q, const float* dl_dimg, double* g_albedo, double* g_emission,
                            int threads) {
  swo_adjoint_physical64_part(s, cam, W, H, spp, 0, spp, depth, seed, rr_depth, rr_q, dl_dimg, g_albedo,
                              g_emission, threads);
}

void swo_adjoint_physical64_part(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                                 uint32_t spp_total, uint32_t s0, uint32_t s1, uint32_t depth, uint64_t seed,
                                 uint32_t rr_depth, double rr_q, const float* dl_dimg, double* g_albedo,
                                 double* g_emission, int threads) {
  pthread_mutex_t mu;
  adj_ctx c;
  pthread_mutex_init(&mu, NULL);
  memset(g_albedo, 0, sizeof(double) * 3 * (size_t)s->ntri);
  memset(g_emission, 0, sizeof(double) * 3 * (size_t)s->nobj);
  c.s = s;
  c.cam = cam;
  c.W = W;
  c.H = H;
  c.spp = s1 - s0;
  c.s0 = s0;
  c.spp_total = spp_total;
  c.depth = depth;
  c.rr_depth = rr_depth;
  c.rr_q = rr_q;
  c.seed = seed;
  c.dl = dl_dimg;
  c.ga = g_albedo;
  c.ge = g_emission;
  c.mu = &mu;
  {
    uint64_t npx = (uint64_t)W * H, per = npx / ((uint64_t)(threads > 0 ? threads : 1) * 4);
    parallel_for(npx, per > 64 ? per : 64, threads, adj_range, &c);
  }
  pthread_mutex_destroy(&mu);
}

/* =============================================================================================
 * The Vulkan application's PathTracer and denoisers (RayTrace program), restated on the CPU as
 * the checker of the library's CUDA restatement. Sources restated:
 *   random numbers   res/shader/helper.glsl:11-41 (LCG a=6237 c=10697 m=21023, randomNormal)
 *   customRefract    res/shader/helper.glsl:43-57, GLSL reflect/refract
 *   camera ray       res/shader/v1.glsl:130-142 (getVisionRay)
 *   traceRay         res/shader/v1.glsl:148-161 (tmin 0.001, tmax 10000, back-face retries)
 *   handleHit        res/shader/v1.glsl:163-188
 *   hit payload      res/shader/v1_closesthit.rchit:9-41, v1_miss.rmiss
 *   raygen           res/shader/path_tracer_vision_raygen.rgen:8-60
 *   denoisers        res/shader/denoise_gauss_comp.comp, denoise_median_comp.comp,
 *                    src/graphic/denoiser/gauss_denoiser.cpp:31-46 (weights)
 * GLSL leaves the precision of division, sqrt, sin/cos/acos and normalize to the implementation;
 * the choice fixed here (and by the library) is: IEEE float division and sqrt, the double
 * sin/cos/acos of the widened argument rounded to float, normalize(v) = v / sqrt(dot(v, v)),
 * no fused multiply-adds. The closest hit uses the Moller-Trumbore arithmetic above with t in
 * [0.001, 10000] and ties to the lower triangle id, found by testing every triangle of every
 * object whose widened box the ray meets. Parity with
 * the shaders on a GPU ray tracing pipeline cannot be checked here (no graphics stack), so this
 * restatement is pinned only by its own known-answer tests. */

static const float RT_PI = 3.1415926538f;

/* Culling only: does the ray (t >= 0) pass through the object box widened by a margin far above
 * any float rounding of the intersection test? Evaluated in double; a miss here means no
 * triangle of the object can be accepted. */
static int rt_box_maybe(const float* box, v3f o, v3f d) {
  const double ov[3] = {o.x, o.y, o.z}, dv[3] = {d.x, d.y, d.z};
  double tmin = 0.0, tmax = INFINITY, m = 1.0;
  int i;
  for (i = 0; i < 6; ++i) m = fmax(m, fabs((double)box[i]));
  m *= 1e-3;
  for (i = 0; i < 3; ++i) {
    const double lo = (double)box[i] - m, hi = (double)box[3 + i] + m;
    if (dv[i] == 0.0) {
      if (ov[i] < lo || ov[i] > hi) return 0;
    } else {
      double t1 = (lo - ov[i]) / dv[i], t2 = (hi - ov[i]) / dv[i];
      if (t1 > t2) {
        const double x = t1;
        t1 = t2;
        t2 = x;
      }
      tmin = fmax(tmin, t1);
      tmax = fmin(tmax, t2);
    }
  }
  return tmin <= tmax;
}

static uint32_t rt_closest(const swo_scene* s, v3f o, v3f d, float* t_out) {
  float bt = INFINITY;
  uint32_t bi = 0xFFFFFFFFu, k, obj;
  for (obj = 0; obj < s->nobj; ++obj) {
    if (!rt_box_maybe(s->obj_box + 6 * (size_t)obj, o, d)) continue;
    /* objects in order and triangles in id order: a tie keeps the lower id */
    for (k = s->obj_first[obj]; k < s->obj_first[obj + 1]; ++k) {
      float t, d2;
      if (!ref_intersect(o, d, ld3(s->v0 + 3 * (size_t)k), ld3(s->e0 + 3 * (size_t)k),
                         ld3(s->e1 + 3 * (size_t)k), &t, &d2))
        continue;
      if (!(t >= 0.001f && t <= 10000.0f)) continue;
      if (t < bt) {
        bt = t;
        bi = k;
      }
    }
  }
  *t_out = bt;
  return bi;
}

static uint32_t rt_lcg_init(uint32_t x, uint32_t y) { return (625u + x * 7444u + y * 1045u) % 21023u; }
static float rt_rand(uint32_t* st) {
  *st = (6237u * *st + 10697u) % 21023u;
  return (float)*st / 21023.0f;
}
static v3f rt_normalize(v3f v) {
  float l = sqrtf(dot(v, v));
  return mk(v.x / l, v.y / l, v.z / l);
}
static v3f rt_reflect(v3f I, v3f N) {
  float s = 2.0f * dot(N, I);
  return mk(I.x - s * N.x, I.y - s * N.y, I.z - s * N.z);
}
static v3f rt_refract(v3f I, v3f N, float eta) {
  float ndi = dot(N, I);
  float k = 1.0f - eta * eta * (1.0f - ndi * ndi);
  float s;
  if (k < 0.0f) return mk(0.0f, 0.0f, 0.0f);
  s = eta * ndi + sqrtf(k);
  return mk(eta * I.x - s * N.x, eta * I.y - s * N.y, eta * I.z - s * N.z);
}
static v3f rt_custom_refract(v3f d, v3f n, float eta) {
  float ndotd = dot(n, d), angle;
  if (ndotd > 0.0f) {
    n = mk(-n.x, -n.y, -n.z);
    ndotd = dot(n, d);
  } else {
    eta = 1.0f / eta;
  }
  angle = (float)sin((double)(float)acos((double)ndotd)) * eta;
  if (-1.0f < angle && angle < 1.0f) return rt_refract(d, n, eta);
  return rt_reflect(d, n);
}
static v3f rt_random_normal_dir(uint32_t* rng, v3f n) {
  float theta = 2.0f * RT_PI * rt_rand(rng);
  float u = 2.0f * rt_rand(rng) - 1.0f;
  float suu = sqrtf(1.0f - u * u);
  v3f v = mk(suu * (float)cos((double)theta), suu * (float)sin((double)theta), u);
  if (dot(v, n) < 0.0f) v = mk(-v.x, -v.y, -v.z);
  return v;
}

typedef struct {
  v3f pos, n, color;
  float dT, rT, tT, eta;
  int light;
} rt_payload;

/* barycentric (u, v) of the Moller-Trumbore test, the same operations as ref_intersect */
static rt_payload rt_hit(const swo_scene* s, uint32_t k, v3f o, v3f d) {
  rt_payload P;
  v3f v0 = ld3(s->v0 + 3 * (size_t)k), e0 = ld3(s->e0 + 3 * (size_t)k), e1 = ld3(s->e1 + 3 * (size_t)k);
  v3f h = cross(d, e1), sv = sub(o, v0), q;
  float f = 1.0f / dot(e0, h), u, v, b0;
  const float* nr = s->nrm + 9 * (size_t)k;
  const float* m = s->mats + 9 * (size_t)s->tri_obj[k];
  u = f * dot(sv, h);
  q = cross(sv, e0);
  v = f * dot(d, q);
  b0 = 1.0f - u - v;
  P.pos = mk(v0.x + e0.x * u + e1.x * v, v0.y + e0.y * u + e1.y * v, v0.z + e0.z * u + e1.z * v);
  P.n = rt_normalize(mk(nr[0] * b0 + nr[3] * u + nr[6] * v, nr[1] * b0 + nr[4] * u + nr[7] * v,
                        nr[2] * b0 + nr[5] * u + nr[8] * v));
  P.light = m[7] != 0.0f;
  P.color = mk(m[0], m[1], m[2]);
  if (P.light) P.color = mk(m[0] * m[8], m[1] * m[8], m[2] * m[8]);
  P.dT = m[3];
  P.rT = m[4];
  P.tT = m[5];
  P.eta = m[6];
  return P;
}

/* handleHit: returns 1 for DIFFUSE_VALUE (also the value when no branch is taken) */
static int rt_handle_hit(const rt_payload* P, uint32_t* rng, v3f* o, v3f* d) {
  float r = rt_rand(rng);
  int diffuse = 1;
  if (r <= P->dT) {
    *d = rt_random_normal_dir(rng, P->n);
  } else if (r <= P->rT) {
    *d = rt_reflect(*d, P->n);
    diffuse = 0;
  } else if (r <= P->tT) {
    *d = rt_custom_refract(*d, P->n, P->eta);
    diffuse = 0;
  }
  *o = mk(P->pos.x + d->x * 0.001f, P->pos.y + d->y * 0.001f, P->pos.z + d->z * 0.001f);
  return diffuse;
}

static uint8_t rt_unorm8(float x) {
  float c = x > 0.0f ? x : 0.0f; /* NaN -> 0 */
  if (c > 1.0f) c = 1.0f;
  return (uint8_t)nearbyintf(c * 255.0f);
}

static v3f rt_pixel(const swo_scene* s, const swo_camera* cam, uint32_t x, uint32_t y, uint32_t W, uint32_t H,
                    uint32_t vj, uint32_t spp) {
  const float* vi = cam->vi;
  const float* pi = cam->pi;
  uint32_t rng = rt_lcg_init(x, y), smp, i, c;
  float ux = ((float)x + 0.5f) / (float)W, uy = ((float)y + 0.5f) / (float)H;
  float dx = ux * 2.0f - 1.0f, dy = uy * 2.0f - 1.0f, t;
  v3f o = mk(vi[12], vi[13], vi[14]), tg, w, d, sdir, fin = mk(0.0f, 0.0f, 0.0f);
  rt_payload def;
  uint32_t k;
  tg = mk(pi[0] * dx + pi[4] * dy + pi[8] * 1.0f + pi[12] * 1.0f, pi[1] * dx + pi[5] * dy + pi[9] * 1.0f + pi[13] * 1.0f,
          pi[2] * dx + pi[6] * dy + pi[10] * 1.0f + pi[14] * 1.0f);
  tg = rt_normalize(tg);
  w = mk(vi[0] * tg.x + vi[4] * tg.y + vi[8] * tg.z + vi[12] * 0.0f,
         vi[1] * tg.x + vi[5] * tg.y + vi[9] * tg.z + vi[13] * 0.0f,
         vi[2] * tg.x + vi[6] * tg.y + vi[10] * tg.z + vi[14] * 0.0f);
  sdir = rt_normalize(w);
  /* traceRay with back-face culling: up to four traces */
  for (c = 0;; ++c) {
    k = rt_closest(s, o, sdir, &t);
    if (k == 0xFFFFFFFFu) return mk(0.0f, 0.0f, 0.0f);
    def = rt_hit(s, k, o, sdir);
    if (!(dot(def.n, sdir) > 0.0f) || c == 3) break;
    o = def.pos;
  }
  if (def.light) return def.color;
  for (smp = 0; smp < spp; ++smp) {
    rt_payload cur = def;
    v3f col = mk(1.0f, 1.0f, 1.0f);
    int light_hit = 0;
    d = sdir;
    for (i = 1; i < vj; ++i) {
      if (rt_handle_hit(&cur, &rng, &o, &d)) {
        float cs = dot(d, cur.n);
        col = mk(col.x * (cur.color.x * cs), col.y * (cur.color.y * cs), col.z * (cur.color.z * cs));
      }
      k = rt_closest(s, o, d, &t);
      if (k == 0xFFFFFFFFu) break; /* color = 0 */
      cur = rt_hit(s, k, o, d);
      if (cur.light && dot(d, cur.n) <= 0.0f) {
        col = mk(col.x * cur.color.x, col.y * cur.color.y, col.z * cur.color.z);
        light_hit = 1;
        break;
      }
    }
    if (light_hit) fin = add(fin, col);
  }
  {
    float sc = (2.0f * RT_PI) / (float)spp;
    return mk(fin.x * sc, fin.y * sc, fin.z * sc);
  }
}

typedef struct {
  const swo_scene* s;
  const swo_camera* cam;
  uint32_t W, H, vj, spp, p0;
  float* rgb;
  uint8_t* rgba;
} rt_ctx;

static void rt_range(void* c_, uint64_t b, uint64_t e) {
  rt_ctx* c = (rt_ctx*)c_;
  uint64_t k;
  for (k = b; k < e; ++k) {
    uint32_t p = c->p0 + (uint32_t)k;
    v3f v = rt_pixel(c->s, c->cam, p % c->W, p / c->W, c->W, c->H, c->vj, c->spp);
    if (c->rgb) {
      c->rgb[3 * k + 0] = v.x;
      c->rgb[3 * k + 1] = v.y;
      c->rgb[3 * k + 2] = v.z;
    }
    if (c->rgba) {
      c->rgba[4 * k + 0] = rt_unorm8(v.x);
      c->rgba[4 * k + 1] = rt_unorm8(v.y);
      c->rgba[4 * k + 2] = rt_unorm8(v.z);
      c->rgba[4 * k + 3] = 0;
    }
  }
}

void swo_rt_render(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H, uint32_t vj, uint32_t spp,
                   uint32_t p0, uint32_t p1, float* rgb, uint8_t* rgba, int threads) {
  rt_ctx c = {s, cam, W, H, vj, spp, p0, rgb, rgba};
  parallel_for(p1 - p0, 4, threads, rt_range, &c);
}

typedef struct {
  const swo_scene* s;
  const float *ro, *rd;
  uint32_t* tri;
  float* t;
} rt_trace_ctx;

static void rt_trace_range(void* c_, uint64_t b, uint64_t e) {
  rt_trace_ctx* c = (rt_trace_ctx*)c_;
  uint64_t i;
  for (i = b; i < e; ++i) c->tri[i] = rt_closest(c->s, ld3(c->ro + 4 * i), ld3(c->rd + 4 * i), &c->t[i]);
}

void swo_rt_trace(const swo_scene* s, const float* ro, const float* rd, uint64_t n, uint32_t* hit_tri,
                  float* hit_t, int threads) {
  rt_trace_ctx c = {s, ro, rd, hit_tri, hit_t};
  parallel_for(n, 64, threads, rt_trace_range, &c);
}

int swo_rt_gauss_weights(uint32_t k, float sigma, float* out) {
  float sum = 0.0f;
  uint32_t i;
  if (k == 0 || k > 19 || (k & 1u) == 0) return -1;
  for (i = 0; i < k; ++i) {
    float a = (float)i - ((float)k - 1.0f), b, r;
    a = a * a;
    b = 2.0f * sigma * sigma;
    r = (float)exp((double)(-a / b));
    out[i] = r;
    sum += r;
  }
  sum = 1.0f / sum;
  for (i = 0; i < k; ++i) out[i] *= sum;
  return 0;
}

void swo_rt_denoise_gauss(const uint8_t* in, uint8_t* out, uint32_t W, uint32_t H, uint32_t k,
                          const float* g) {
  int off = (int)(k / 2), x, y, dx, dy, ch;
  for (y = 0; y < (int)H; ++y)
    for (x = 0; x < (int)W; ++x) {
      float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      for (dx = -off; dx <= off; ++dx)
        for (dy = -off; dy <= off; ++dy) {
          int px = x + dx, py = y + dy;
          if (0 <= px && px < (int)W && 0 <= py && py < (int)H)
            for (ch = 0; ch < 4; ++ch)
              c[ch] += (float)in[4 * ((size_t)py * W + px) + ch] / 255.0f * g[dx + off] * g[dy + off];
        }
      for (ch = 0; ch < 4; ++ch) out[4 * ((size_t)y * W + x) + ch] = rt_unorm8(c[ch]);
    }
}

static int cmp_float(const void* a, const void* b) {
  float x = *(const float*)a, y = *(const float*)b;
  return (x > y) - (x < y);
}

void swo_rt_denoise_median(const uint8_t* in, uint8_t* out, uint32_t W, uint32_t H) {
  int x, y, dx, dy, ch;
  for (y = 0; y < (int)H; ++y)
    for (x = 0; x < (int)W; ++x)
      for (ch = 0; ch < 4; ++ch) {
        float v[9];
        int n = 0;
        for (dx = -1; dx <= 1; ++dx)
          for (dy = -1; dy <= 1; ++dy) {
            int px = x + dx, py = y + dy;
            /* texels outside the image: undefined in the shader, 0 here */
            v[n++] = (0 <= px && px < (int)W && 0 <= py && py < (int)H)
                         ? (float)in[4 * ((size_t)py * W + px) + ch] / 255.0f
                         : 0.0f;
          }
        qsort(v, 9, sizeof(float), cmp_float);
        out[4 * ((size_t)y * W + x) + ch] = rt_unorm8(v[4]);
      }
}
