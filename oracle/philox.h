/* Philox-4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
 * as easy as 1, 2, 3", SC'11), restated for the oracle. TEST INFRASTRUCTURE ONLY.
 *
 * The path tracer draws its random numbers from this generator keyed by (seed) and a counter of
 * (pixel, sample, vertex, stream): one call yields the four uniforms of one path vertex. The
 * oracle, the Philox shim linked into the reference, and the CUDA kernels all use this keying, so
 * the same path sees the same numbers everywhere. */
#ifndef SWR_ORACLE_PHILOX_H
#define SWR_ORACLE_PHILOX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

static inline void swo_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2],
                                     uint32_t out[4]) {
  uint32_t x0 = ctr_in[0], x1 = ctr_in[1], x2 = ctr_in[2], x3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  int r;
  for (r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * x0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t y0 = hi1 ^ x1 ^ k0;
    uint32_t y2 = hi0 ^ x3 ^ k1;
    x0 = y0;
    x1 = lo1;
    x2 = y2;
    x3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = x0;
  out[1] = x1;
  out[2] = x2;
  out[3] = x3;
}

/* top 24 bits scaled by 2^-24: exact in float, in [0, 1) */
static inline float swo_u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

/* the four uniforms of one path vertex */
static inline void swo_vertex_uniforms(uint64_t seed, uint32_t pixel, uint32_t sample,
                                       uint32_t vertex, uint32_t stream, float u[4]) {
  uint32_t ctr[4] = {pixel, sample, vertex, stream};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  int i;
  swo_philox4x32_10(ctr, key, o);
  for (i = 0; i < 4; ++i) u[i] = swo_u01(o[i]);
}

#ifdef __cplusplus
}
#endif

#endif
