/* TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's path tracer, the checker of the
 * parity tests. Never linked into, loaded by or called from the product library. */
#ifndef SWR_ORACLE_H
#define SWR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct swo_scene {
  uint32_t ntri, nobj;
  const float* v0;        /* [ntri*3] */
  const float* e0;        /* [ntri*3] v1 - v0 */
  const float* e1;        /* [ntri*3] v2 - v0 */
  const float* den;       /* [ntri*4] d00 d01 d11 denom */
  const float* tri_box;   /* [ntri*6] lo.xyz hi.xyz (reference triangle boxes) */
  const float* obj_box;   /* [nobj*6] reference object boxes */
  const uint32_t* tri_obj;     /* [ntri] */
  const uint32_t* obj_first;   /* [nobj+1] triangle range of each object */
  const uint32_t* visit;       /* [ntri] triangle ids in the reference's visit order */
  const float* nrm;       /* [ntri*9] vertex normals of the three corners */
  const float* mats;      /* [nobj*9] color.rgb dT rT tT eta light strength */
  const float* albedo;    /* [ntri*3] physical-mode albedo (NULL: object color) */
  const float* emission;  /* [nobj*3] physical-mode emission (NULL: color * strength) */
  const float* vtx;       /* [ntri*9] corner positions v0 v1 v2 (light-point sampling) */
} swo_scene;

typedef struct swo_camera {
  float vi[16], pi[16], org[3];
} swo_camera;

/* closest hit with the reference's rules; rays as [n*4] floats (xyz used) */
void swo_trace(const swo_scene* s, const float* ro, const float* rd, uint64_t n, uint32_t* hit_tri,
               float* hit_d2, float* hit_t, int threads);

/* reference-mode radiance for pixels [p0, p1): per sample (r g b flag) and per pixel */
void swo_render_reference(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                          uint32_t spp, uint32_t depth, uint64_t seed, uint32_t p0, uint32_t p1,
                          float* per_sample, float* per_pixel, int threads);

/* physical-mode estimator evaluated in double for pixels [p0, p1) (mean over spp per pixel,
 * plus the per-pixel sample variance of the mean for statistical checks) */
void swo_render_physical64(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                           uint32_t spp, uint32_t depth, uint64_t seed, uint32_t rr_depth,
                           double rr_q, uint32_t p0, uint32_t p1, double* per_pixel,
                           double* per_pixel_var, int threads);

/* gradient of sum_p dl_dimg[p] . image[p] of the physical-mode estimator with respect to the
 * per-triangle albedo [ntri*3] and per-object emission [nobj*3], evaluated in double on the same
 * paths (same random numbers) as the renderer */
void swo_adjoint_physical64(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                            uint32_t spp, uint32_t depth, uint64_t seed, uint32_t rr_depth,
                            double rr_q, const float* dl_dimg, double* g_albedo, double* g_emission,
                            int threads);

/* The three functions above for part of each pixel's samples: samples [s0, s1) of an image with
 * spp_total samples per pixel, with the random numbers of those samples and the whole image's
 * 1/spp_total weight (times 2 pi in reference mode). per_sample holds (s1 - s0) samples per pixel;
 * per_pixel_var is only meaningful for the whole range. Parts over a partition of [0, spp_total)
 * sum to the whole image and to its gradient. */
void swo_render_reference_part(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                               uint32_t spp_total, uint32_t s0, uint32_t s1, uint32_t depth, uint64_t seed,
                               uint32_t p0, uint32_t p1, float* per_sample, float* per_pixel, int threads);
void swo_render_physical64_part(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                                uint32_t spp_total, uint32_t s0, uint32_t s1, uint32_t depth, uint64_t seed,
                                uint32_t rr_depth, double rr_q, uint32_t p0, uint32_t p1, double* per_pixel,
                                double* per_pixel_var, int threads);
void swo_adjoint_physical64_part(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H,
                                 uint32_t spp_total, uint32_t s0, uint32_t s1, uint32_t depth, uint64_t seed,
                                 uint32_t rr_depth, double rr_q, const float* dl_dimg, double* g_albedo,
                                 double* g_emission, int threads);

/* BidirectionalPathTracer radiance for pixels [p0, p1): per sample (the contribution before the
 * 2 pi / spp scale; r g b 1) and per pixel. Returns -2 for a scene without light sources. */
int swo_render_bdpt(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H, uint32_t spp,
                    uint32_t vision_jumps, uint32_t light_jumps, uint32_t max_depth, uint64_t seed,
                    uint32_t p0, uint32_t p1, float* per_sample, float* per_pixel, int threads);

/* The Vulkan application's PathTracer (RayTrace program) for pixels [p0, p1): finalColor [n*3]
 * and the stored rgba8 texel [n*4] (either may be NULL). */
void swo_rt_render(const swo_scene* s, const swo_camera* cam, uint32_t W, uint32_t H, uint32_t vision_jumps,
                   uint32_t spp, uint32_t p0, uint32_t p1, float* rgb, uint8_t* rgba, int threads);
/* traceRay's closest hit: triangle id (0xFFFFFFFF on a miss) and t */
void swo_rt_trace(const swo_scene* s, const float* ro, const float* rd, uint64_t n, uint32_t* hit_tri,
                  float* hit_t, int threads);
/* GaussDenoiser weights; -1 for a kernel size that is not odd in 1..19 */
int swo_rt_gauss_weights(uint32_t kernel_size, float sigma, float* out);
void swo_rt_denoise_gauss(const uint8_t* in, uint8_t* out, uint32_t W, uint32_t H, uint32_t kernel_size,
                          const float* weights);
void swo_rt_denoise_median(const uint8_t* in, uint8_t* out, uint32_t W, uint32_t H);

#ifdef __cplusplus
}
#endif

#endif
