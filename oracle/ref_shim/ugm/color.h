// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// float RGB / RGBA colours with the operators the reference's hot-path sources
// use.  TEST INFRASTRUCTURE ONLY.
#pragma once

namespace ugm {

struct color3 {
  float r, g, b;
  float& operator[](int i) { return i == 0 ? r : (i == 1 ? g : b); }
  float operator[](int i) const { return i == 0 ? r : (i == 1 ? g : b); }
  color3 operator+(const color3& o) const { return color3(r + o.r, g + o.g, b + o.b); }
  color3 operator-(const color3& o) const { return color3(r - o.r, g - o.g, b - o.b); }
  color3 operator*(const color3& o) const { return color3(r * o.r, g * o.g, b * o.b); }
  color3 operator*(float s) const { return color3(r * s, g * s, b * s); }
  color3 operator/(float s) const { return color3(r / s, g / s, b / s); }
  color3& operator+=(const color3& o) { r += o.r; g += o.g; b += o.b; return *this; }
  color3& operator*=(const color3& o) { r *= o.r; g *= o.g; b *= o.b; return *this; }
  color3& operator*=(float s) { r *= s; g *= s; b *= s; return *this; }
  color3& operator/=(float s) { r /= s; g /= s; b /= s; return *this; }
  bool operator==(const color3& o) const { return r == o.r && g == o.g && b == o.b; }
  bool operator!=(const color3& o) const { return !(*this == o); }
  static const color3 zero, one;
};
inline constexpr color3 color3::zero{0.0f, 0.0f, 0.0f};
inline constexpr color3 color3::one{1.0f, 1.0f, 1.0f};
inline color3 operator*(float s, const color3& c) { return c * s; }
typedef color3 color3f;

struct color4 {
  union {
    struct {
      float r, g, b, a;
    };
    struct {
      color3 rgb;
      float alpha_;
    };
  };
  color4() = default;
  constexpr color4(float r_, float g_, float b_, float a_) : r(r_), g(g_), b(b_), a(a_) {}
  color4 operator*(float s) const { return color4(r * s, g * s, b * s, a * s); }
  color4 operator+(const color4& o) const { return color4(r + o.r, g + o.g, b + o.b, a + o.a); }
};
typedef color4 color4f;

}  // namespace ugm

using namespace ugm;
