// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// the free functions the reference's hot-path sources call.  TEST
// INFRASTRUCTURE ONLY.  randomValue() and randomRayInHemisphere() are
// defined by the harness (oracle/ref_harness.cpp), which feeds them from a
// caller-supplied stream of uniforms.
#pragma once

#include <cmath>

#include "color.h"
#include "types2d.h"
#include "types3d.h"

namespace ugm {

float randomValue();
vec3 randomRayInHemisphere(const vec3& normal);

template <class T>
inline T clamp(T v, T lo, T hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}
inline float lerp(float a, float b, float t) { return a + (b - a) * t; }
inline bool extremelyClose(const vec2& a, const vec2& b) { return fabsf(a.x - b.x) < 1e-6f && fabsf(a.y - b.y) < 1e-6f; }
inline bool extremelyClose(const vec3& a, const vec3& b) {
  return fabsf(a.x - b.x) < 1e-6f && fabsf(a.y - b.y) < 1e-6f && fabsf(a.z - b.z) < 1e-6f;
}

}  // namespace ugm

using namespace ugm;
