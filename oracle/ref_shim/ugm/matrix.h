// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// a 4x4 matrix in the row-vector convention p' = [p 1] * M.  TEST
// INFRASTRUCTURE ONLY (the pinned functions never transform).
#pragma once

#include "types3d.h"

namespace ugm {

struct Matrix4 {
  float m[16];
  Matrix4() {
    for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.0f : 0.0f;
  }
  Matrix4 operator*(const Matrix4& o) const {
    Matrix4 r;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) {
        float s = 0.0f;
        for (int k = 0; k < 4; ++k) s += m[i * 4 + k] * o.m[k * 4 + j];
        r.m[i * 4 + j] = s;
      }
    return r;
  }
};

inline vec4 operator*(const vec4& v, const Matrix4& M) {
  const float* m = M.m;
  return vec4(v.x * m[0] + v.y * m[4] + v.z * m[8] + v.w * m[12], v.x * m[1] + v.y * m[5] + v.z * m[9] + v.w * m[13],
              v.x * m[2] + v.y * m[6] + v.z * m[10] + v.w * m[14], v.x * m[3] + v.y * m[7] + v.z * m[11] + v.w * m[15]);
}

}  // namespace ugm

using namespace ugm;
