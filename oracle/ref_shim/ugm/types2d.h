// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// 2D types named by the reference's headers.  TEST INFRASTRUCTURE ONLY.
#pragma once

#include <cmath>

#include "types3d.h"

namespace ugm {

struct BBox2D {
  vec2 min, max;
  static BBox2D fromTriangle(const vec2& a, const vec2& b, const vec2& c) {
    BBox2D bb;
    bb.min = vec2(fminf(a.x, fminf(b.x, c.x)), fminf(a.y, fminf(b.y, c.y)));
    bb.max = vec2(fmaxf(a.x, fmaxf(b.x, c.x)), fmaxf(a.y, fmaxf(b.y, c.y)));
    return bb;
  }
};

template <class T>
struct size2 {
  T width, height;
  size2(T w, T h) : width(w), height(h) {}
};
typedef size2<float> sizef;
typedef size2<int> sizei;

}  // namespace ugm

using namespace ugm;
