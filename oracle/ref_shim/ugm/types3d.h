// Clean-room stand-in for the reference's graphics-math submodule (cpp-graphics-module,
// "ugm"), whose sources are not in the reference tree.  TEST INFRASTRUCTURE ONLY: it
// exists so that the reference's own hot-path sources (src/raygen/bvh.cpp,
// raycommon.cpp, medium.cpp, bsdf.cpp) compile unchanged into oracle/_ref, where
// their outputs pin the oracle.  Written from the call sites in those files: only
// the members and operators they use, with plain IEEE float arithmetic (no fused
// multiply-add: the recipe builds with -ffp-contract=off).  The types are
// aggregates (no constructors), because the reference nests them in anonymous
// unions; `vec3(x, y, z)` is C++20 parenthesised aggregate initialisation.
#pragma once

#include <cmath>
#include <cstdint>

namespace ugm {

struct vec2 {
  float x, y;
  vec2 operator+(const vec2& o) const { return vec2(x + o.x, y + o.y); }
  vec2 operator-(const vec2& o) const { return vec2(x - o.x, y - o.y); }
  vec2 operator*(float s) const { return vec2(x * s, y * s); }
  vec2 operator*(const vec2& o) const { return vec2(x * o.x, y * o.y); }
  vec2 operator/(float s) const { return vec2(x / s, y / s); }
  vec2 operator/(double s) const { return vec2((float)(x / s), (float)(y / s)); }
  bool operator==(const vec2& o) const { return x == o.x && y == o.y; }
  static const vec2 zero, one;
};
inline constexpr vec2 vec2::zero{0.0f, 0.0f};
inline constexpr vec2 vec2::one{1.0f, 1.0f};

struct vec3 {
  float x, y, z;
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  vec3 operator+(const vec3& o) const { return vec3(x + o.x, y + o.y, z + o.z); }
  vec3 operator-(const vec3& o) const { return vec3(x - o.x, y - o.y, z - o.z); }
  vec3 operator-() const { return vec3(-x, -y, -z); }
  vec3 operator*(float s) const { return vec3(x * s, y * s, z * s); }
  vec3 operator*(const vec3& o) const { return vec3(x * o.x, y * o.y, z * o.z); }
  vec3 operator/(float s) const { return vec3(x / s, y / s, z / s); }
  vec3& operator+=(const vec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
  vec3& operator-=(const vec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
  vec3& operator*=(float s) { x *= s; y *= s; z *= s; return *this; }
  vec3& operator/=(float s) { x /= s; y /= s; z /= s; return *this; }
  bool operator==(const vec3& o) const { return x == o.x && y == o.y && z == o.z; }
  bool operator!=(const vec3& o) const { return !(*this == o); }
  float length() const { return sqrtf(x * x + y * y + z * z); }
  // returns the unit vector (the receiver is left unchanged)
  vec3 normalize() const {
    const float l = length();
    return l > 0.0f ? vec3(x / l, y / l, z / l) : *this;
  }
  static const vec3 zero, one;
};
inline constexpr vec3 vec3::zero{0.0f, 0.0f, 0.0f};
inline constexpr vec3 vec3::one{1.0f, 1.0f, 1.0f};

inline vec3 operator*(float s, const vec3& v) { return v * s; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline vec3 cross(const vec3& a, const vec3& b) {
  return vec3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline vec3 normalize(const vec3& v) { return v.normalize(); }

struct vec4 {
  float x, y, z, w;
  vec4 operator*(float s) const { return vec4(x * s, y * s, z * s, w * s); }
  vec4 operator+(const vec4& o) const { return vec4(x + o.x, y + o.y, z + o.z, w + o.w); }
  vec4 operator-() const { return vec4(-x, -y, -z, -w); }
};
inline float dot(const vec4& a, const vec4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// A ray does not normalise its direction (shadow rays carry p - hit with
// maxt 0.99999).
struct Ray {
  vec3 origin, dir;
};

struct BoundingBox {
  vec3 min, max;
  static BoundingBox fromTriangle(const vec3& a, const vec3& b, const vec3& c) {
    BoundingBox bb;
    bb.min = vec3(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)), fminf(a.z, fminf(b.z, c.z)));
    bb.max = vec3(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)), fmaxf(a.z, fmaxf(b.z, c.z)));
    return bb;
  }
};

struct Triangle {
  vec3 v1, v2, v3;
};
struct TriangleNUV {
  vec3 v1, v2, v3;
  vec3 n1, n2, n3;
  vec2 uv1, uv2, uv3;
};
struct TriangleNUV2TBC {
  vec3 v1, v2, v3;
  vec3 n1, n2, n3;
  vec2 uv1, uv2, uv3, uv4, uv5, uv6;
};

}  // namespace ugm

using namespace ugm;
