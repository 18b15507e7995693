// TEST INFRASTRUCTURE ONLY. Replacement definitions for the reference's RandomGenerator
// (software_renderer/math/random.h:9-22), linked into the reference build in place of
// math/random.cpp. The reference seeds a mutex-guarded mt19937 from std::random_device, so its
// images are not reproducible; this shim draws from Philox-4x32-10 keyed by a thread-local cursor
// (seed, pixel, sample, vertex) that the harness sets before each sample, so that the reference
// and the CUDA path tracer consume identical random numbers.
//
// Draw layout per path vertex (one Philox call): u[0] chooses the scatter event (rand() in
// path_tracer.cpp:62), u[1] and u[2] are the two uniforms of the hemisphere sample (the two
// rand() calls of random.cpp:17-18). The direction math restates random.cpp:16-35: theta is
// 2*pi*u taken in double and stored to float, u' = 2u-1, sqrtf(1-u'^2), double sin/cos.
#include "../oracle/philox.h"

#include <cmath>

#include "math/random.h"

struct SwrCursor {
  uint64_t seed = 0;
  uint32_t pixel = 0;
  uint32_t sample = 0;
  uint32_t vertex = 0;
  float u[4] = {0, 0, 0, 0};
};
static thread_local SwrCursor g_cursor;

extern "C" void swr_shim_set_cursor(uint64_t seed, uint32_t pixel, uint32_t sample) {
  g_cursor.seed = seed;
  g_cursor.pixel = pixel;
  g_cursor.sample = sample;
  g_cursor.vertex = 0;
}

extern "C" uint32_t swr_shim_vertices_drawn() { return g_cursor.vertex; }

RandomGenerator::RandomGenerator() : rng(), distribution(0.0f, 1.0f) {}

RandomGenerator::~RandomGenerator() {}

float RandomGenerator::rand() {
  swo_vertex_uniforms(g_cursor.seed, g_cursor.pixel, g_cursor.sample, g_cursor.vertex, 0,
                      g_cursor.u);
  g_cursor.vertex++;
  return g_cursor.u[0];
}

Vector3f RandomGenerator::randomNormal() {
  float theta = 2.0f * M_PI * g_cursor.u[1];
  float u = 2.0f * g_cursor.u[2] - 1.0f;
  float suu = sqrtf(1.0f - u * u);
  float sinTheta = (float)std::sin((double)theta);
  float cosTheta = (float)std::cos((double)theta);
  return Vector3f({suu * cosTheta, suu * sinTheta, u});
}

Vector3f RandomGenerator::randomNormalDirection(const Vector3f& normal) {
  Vector3f v = randomNormal();
  if (v.dot(normal) < 0.0f) v *= -1.0f;
  return v;
}
