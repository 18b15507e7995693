// Host-side float math with the operation order of the reference's math templates.
//
// Every routine here reproduces, operation for operation, the rounding sequence of
// software_renderer/math/{vector.h,matrix.h,matrix.cpp,rotation.cpp,aabb.cpp}. That is what
// makes the world-space vertices, triangle edges, boxes and camera matrices produced by this
// library bit-identical to the reference's. This file must be compiled without FP contraction
// (-ffp-contract=off) on an SSE2 target, which is how the reference's own x86-64 build behaves.
//
// Conventions carried over from the reference:
//  * Matrix * vector is the row-vector form ret[j] = sum_i m[i][j] * v[i]   (matrix.h:245-253)
//  * sums start from +0.0f and accumulate left to right                       (vector.h:203-241)
//  * normalize() takes a double magnitude and multiplies by a double factor   (vector.h:210-225)
//  * sin/cos/tan/acos are the double-precision libm functions (the reference binds the double
//    overloads: its objects import sincos, tan and acos, not the float variants).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace swr {

struct V2 {
  float v[2];
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
};

struct V3 {
  float v[3];
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
};

struct V4 {
  float v[4];
  float& operator[](int i) { return v[i]; }
  float operator[](int i) const { return v[i]; }
};

inline V3 v3(float x, float y, float z) { return V3{{x, y, z}}; }
inline V4 v4(float x, float y, float z, float w) { return V4{{x, y, z, w}}; }

inline V3 add(const V3& a, const V3& b) { return v3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline V3 sub(const V3& a, const V3& b) { return v3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline V3 mulv(const V3& a, const V3& b) { return v3(a[0] * b[0], a[1] * b[1], a[2] * b[2]); }
// float scalar * vector (vector.h:269-276 with S = float)
inline V3 scale(float s, const V3& a) { return v3(s * a[0], s * a[1], s * a[2]); }
// double scalar * float vector: each product is taken in double, then stored to float
inline V3 scaled(double s, const V3& a) {
  return v3((float)(s * (double)a[0]), (float)(s * (double)a[1]), (float)(s * (double)a[2]));
}
inline V3 addsc(const V3& a, float s) { return v3(a[0] + s, a[1] + s, a[2] + s); }
inline V3 subsc(const V3& a, float s) { return v3(a[0] - s, a[1] - s, a[2] - s); }

// dot: sum = 0; sum += a[i]*b[i]  (vector.h:235-241)
inline float dot(const V3& a, const V3& b) {
  float s = 0.0f;
  s += a[0] * b[0];
  s += a[1] * b[1];
  s += a[2] * b[2];
  return s;
}
inline float mag2(const V3& a) { return dot(a, a); }
inline float dist2(const V3& a, const V3& b) { return mag2(sub(a, b)); }

// cross (vector.h:288-297)
inline V3 cross(const V3& a, const V3& b) {
  return v3(a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]);
}

// normalize: double magnitude of the float squared magnitude, double factor (vector.h:210-225)
inline V3 normalized(V3 a) {
  double m = std::sqrt((double)mag2(a));
  if (m != 0) {
    double f = 1.0 / m;
    for (int i = 0; i < 3; ++i) a[i] = (float)((double)a[i] * f);
  }
  return a;
}
inline double magnitude(const V3& a) { return std::sqrt((double)mag2(a)); }

// 4x4 float matrix, m[row][col], identity by default (matrix.h:39-43)
struct M4 {
  float m[4][4];
  static M4 identity() {
    M4 r;
    std::memset(r.m, 0, sizeof(r.m));
    for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
    return r;
  }
};

// Matrix product, each entry accumulated from +0.0f over n = 0..3 (matrix.h:216-241)
inline M4 matmul(const M4& a, const M4& b) {
  M4 r;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      float s = 0.0f;
      for (int n = 0; n < 4; ++n) s += a.m[i][n] * b.m[n][j];
      r.m[i][j] = s;
    }
  return r;
}

// Row-vector transform ret[j] = sum_i m[i][j]*v[i] (matrix.h:245-253)
inline V4 xform(const M4& m, const V4& v) {
  V4 r = v4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r[j] += m.m[i][j] * v[i];
  return r;
}

// Determinants by first-row cofactor expansion, with the reference's minor layout
// (matrix.h:124-140 subMatrix, :189-210 det).
inline float det2(const float a[2][2]) { return a[0][0] * a[1][1] - a[0][1] * a[1][0]; }

inline void minor3(const float a[3][3], int ri, int rj, float out[2][2]) {
  int oi = 0;
  for (int i = 0; i < 3; ++i) {
    if (i == ri) continue;
    int oj = 0;
    for (int j = 0; j < 3; ++j) {
      if (j == rj) continue;
      out[oi][oj++] = a[i][j];
    }
    ++oi;
  }
}

inline float det3(const float a[3][3]) {
  float d = 0.0f;
  for (int i = 0; i < 3; ++i) {
    float sub[2][2];
    minor3(a, 0, i, sub);
    if (i % 2 == 0) d += a[0][i] * det2(sub);
    else d -= a[0][i] * det2(sub);
  }
  return d;
}

inline void minor4(const M4& a, int ri, int rj, float out[3][3]) {
  int oi = 0;
  for (int i = 0; i < 4; ++i) {
    if (i == ri) continue;
    int oj = 0;
    for (int j = 0; j < 4; ++j) {
      if (j == rj) continue;
      out[oi][oj++] = a.m[i][j];
    }
    ++oi;
  }
}

inline float det4(const M4& a) {
  float d = 0.0f;
  for (int i = 0; i < 4; ++i) {
    float sub[3][3];
    minor4(a, 0, i, sub);
    if (i % 2 == 0) d += a.m[0][i] * det3(sub);
    else d -= a.m[0][i] * det3(sub);
  }
  return d;
}

// Inverse = (1/det) * adjugate; cof[i][j] = det(minor(j, i)), negated for odd i+j
// (matrix.h:175-187, :212-214, :261-269).
inline M4 inverse(const M4& a) {
  M4 cof;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      float sub[3][3];
      minor4(a, j, i, sub);
      float c = det3(sub);
      if ((i + j) % 2 == 1) c *= -1;
      cof.m[i][j] = c;
    }
  float s = 1.0f / det4(a);
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) cof.m[i][j] *= s;
  return cof;
}

inline M4 scale_matrix(const V3& s) {
  M4 r = M4::identity();
  r.m[0][0] = s[0];
  r.m[1][1] = s[1];
  r.m[2][2] = s[2];
  return r;
}

inline M4 translation_matrix(const V3& p) {
  M4 r = M4::identity();
  r.m[3][0] = p[0];
  r.m[3][1] = p[1];
  r.m[3][2] = p[2];
  return r;
}

// Look-at view matrix (matrix.cpp:23-44)
inline M4 look_at(const V3& pos, const V3& at, const V3& up) {
  M4 r = M4::identity();
  const V3 f = normalized(sub(at, pos));
  const V3 s = normalized(cross(f, up));
  const V3 u = cross(s, f);
  r.m[0][0] = s[0];
  r.m[1][0] = s[1];
  r.m[2][0] = s[2];
  r.m[0][1] = u[0];
  r.m[1][1] = u[1];
  r.m[2][1] = u[2];
  r.m[0][2] = -f[0];
  r.m[1][2] = -f[1];
  r.m[2][2] = -f[2];
  r.m[3][0] = -dot(s, pos);
  r.m[3][1] = -dot(u, pos);
  r.m[3][2] = dot(f, pos);
  return r;
}

// Perspective projection (matrix.cpp:46-61); tan is the double libm function
inline M4 perspective(float aspect, float fov, float nearZ, float farZ, bool invertY) {
  M4 r = M4::identity();
  const float s = (float)std::tan((double)(fov / 2.0f));
  r.m[0][0] = 1.0f / (aspect * s);
  r.m[1][1] = 1.0f / s;
  r.m[2][2] = -(farZ + nearZ) / (farZ - nearZ);
  r.m[2][3] = -1.0f;
  r.m[3][2] = -(2.0f * farZ * nearZ) / (farZ - nearZ);
  r.m[3][3] = 0.0f;
  if (invertY) r.m[1][1] *= -1;
  return r;
}

// Quaternion rotation (rotation.cpp:7-8, :33-56)
struct Rot {
  float s = 1.0f;
  V3 v = v3(0.0f, 0.0f, 0.0f);

  static Rot from_axis_angle(V3 axis, float angle) {
    Rot r;
    const float half = angle / 2.0f;
    r.s = (float)std::cos((double)half);
    r.v = scaled(std::sin((double)half), normalized(axis));
    return r;
  }

  M4 matrix() const {
    M4 r = M4::identity();
    if (magnitude(v) > 0) {
      float a2 = s * s;
      float x2 = v[0] * v[0];
      float y2 = v[1] * v[1];
      float z2 = v[2] * v[2];
      r.m[0][0] = a2 + x2 - y2 - z2;
      r.m[1][1] = a2 - x2 + y2 - z2;
      r.m[2][2] = a2 - x2 - y2 + z2;
      r.m[3][3] = a2 + x2 + y2 + z2;
      r.m[0][1] = 2.0f * (v[0] * v[1] + s * v[2]);
      r.m[0][2] = 2.0f * (v[0] * v[2] - s * v[1]);
      r.m[1][0] = 2.0f * (v[0] * v[1] - s * v[2]);
      r.m[1][2] = 2.0f * (v[1] * v[2] + s * v[0]);
      r.m[2][0] = 2.0f * (v[0] * v[2] + s * v[1]);
      r.m[2][1] = 2.0f * (v[1] * v[2] - s * v[0]);
    }
    return r;
  }
};

// Axis-aligned box with the reference's first-point padding of +-1e-4 (aabb.cpp:26-37).
struct Box {
  bool empty = true;
  V3 lo = v3(0.0f, 0.0f, 0.0f);
  V3 hi = v3(0.0f, 0.0f, 0.0f);

  void add(const V3& p) {
    if (empty) {
      lo = subsc(p, 0.0001f);
      hi = addsc(p, 0.0001f);
      empty = false;
    } else {
      for (int i = 0; i < 3; ++i) {
        // std::min(a,b) = (b < a) ? b : a ; std::max(a,b) = (a < b) ? b : a
        lo[i] = (p[i] < lo[i]) ? p[i] : lo[i];
        hi[i] = (hi[i] < p[i]) ? p[i] : hi[i];
      }
    }
  }

  // union of two boxes (aabb.cpp:16-22)
  static Box merge(const Box& a, const Box& b) {
    Box r;
    r.empty = false;
    for (int i = 0; i < 3; ++i) {
      r.lo[i] = (b.lo[i] < a.lo[i]) ? b.lo[i] : a.lo[i];
      r.hi[i] = (a.hi[i] < b.hi[i]) ? b.hi[i] : a.hi[i];
    }
    return r;
  }

  // 0.5f * (min + max)  (aabb.cpp:55-57)
  V3 center() const { return scale(0.5f, swr::add(lo, hi)); }
};

}  // namespace swr
