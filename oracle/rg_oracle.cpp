// rg_oracle.cpp - TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of RayGen's shader-5 (BSDF) render path, used as the
// correctness oracle for the B200 tracer and as the timed CPU baseline.
// It is never linked into, loaded by, or called from the product path; only
// tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm
// load it.  Every function names the reference file:line it follows (paths
// relative to the RayGen project).
//
// Parity status: pinned to the reference's own code.  The reference's
// hot-path sources (bvh.cpp, raycommon.cpp, medium.cpp, bsdf.cpp) compile
// unchanged against a clean-room stand-in for its missing math submodule
// (oracle/ref_shim, oracle/ref_harness.cpp, `make ref`), and
// tests/golden/make_ref_golden.py records their outputs: BVH closest / any
// hits on three scenes up to the 4M-triangle benchmark scene, the Halton
// sampler, the GGX / dielectric helpers and the homogeneous / procedural
// medium.  tests/test_golden_ref.py checks this file against them (ids,
// Halton values and GGX helpers bit for bit).  The full renderer
// (rayrenderer.cpp) needs more of the missing submodules (image filters and
// codecs, matrix rotations) and is not compiled; the estimator above the
// pinned functions is checked by the analytic known-answer tests in
// tests/test_oracle_kat.py.
//
// Deliberate, documented deviations from the reference:
//  * RNG: the global rand()/randomValue() calls become a counter-based hash
//    keyed by (pixel, sample, vertex, slot, seed); the Halton LDS with
//    Cranley-Patterson rotation (raycommon.cpp:35-92) is kept, salted with
//    seed-1 (seed 1 == the reference's unsalted scramble).
//  * Mix shader: "tree" mode sums all lobes exactly as bsdf.cpp:579-610;
//    "select" mode picks one lobe with probability w_i/sum(w) and weights by
//    sum(w) (same mean), which is what the GPU runs.
//  * Accumulation is FP64 (sum, sum of squares).
//  * Denoise guide buffers are taken from the pixel-centre primary ray and
//    the depth guide uses |hit| in view space (the reference reuses the
//    previous pixel's ray, rayrenderer.cpp:819-844, and mixes view and world
//    space for the distance).

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <random>
#include <thread>
#include <vector>

#include "../include/raygen_b200.h"

namespace orc {

// ---------------------------------------------------------------- math ----
// ugm-style vector math written out in the reference's evaluation order.
struct V3 {
  float x, y, z;
  V3() : x(0), y(0), z(0) {}
  V3(float a, float b, float c) : x(a), y(b), z(c) {}
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
static inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
static inline V3 operator*(V3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline V3 operator*(V3 a, V3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
static inline V3& operator*=(V3& a, V3 b) { a = a * b; return a; }
static inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline V3 cross(V3 a, V3 b) {
  return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float length(V3 a) { return sqrtf(dot(a, a)); }
static inline V3 normalize(V3 a) {
  const float l = length(a);
  return l > 0.0f ? V3(a.x / l, a.y / l, a.z / l) : a;
}
static inline V3 reflect(V3 d, V3 n) { return d - n * (dot(d, n) * 2.0f); }  // raycommon.h:39-41
static inline float maxc(V3 c) { return fmaxf(c.x, fmaxf(c.y, c.z)); }
static inline bool isZero(V3 c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
typedef V3 C3;

static const float kPi = 3.14159265358979323846f;
static const float SURFACE_THICKNESS = 0.0001f;  // raycommon.h:21
static const float MAX_RAY_DISTANCE = 1.0e6f;    // raycommon.h:34
static const float RAY_MAX_DISTANCE = 100.0f;    // rayrenderer.h:48
static const float RR_MIN_PROB = 0.05f, RR_MAX_PROB = 0.95f;  // rayrenderer.cpp:44-45

struct Ray {
  V3 o, d;
};

// raycommon.h:76-78
static inline Ray ThicknessRay(V3 o, V3 d) { return Ray{o + normalize(d) * SURFACE_THICKNESS, d}; }
// raycommon.h:82-85
static inline Ray SurfaceRay(V3 hit, V3 dir, V3 n) {
  const float side = (dot(dir, n) >= 0.0f) ? 1.0f : -1.0f;
  return Ray{hit + n * (side * SURFACE_THICKNESS), dir};
}

// ----------------------------------------------------------------- RNG ----
// hashPixel: raycommon.cpp:35-41
static inline uint32_t hashPixel(uint32_t x, uint32_t y, uint32_t salt) {
  uint32_t v = x * 73856093u ^ y * 19349663u ^ salt * 83492791u;
  v ^= v >> 16; v *= 0x7feb352du;
  v ^= v >> 15; v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}
// radicalInverse: raycommon.cpp:48-61
static inline float radicalInverse(uint32_t i, int base) {
  const float invBase = 1.0f / (float)base;
  float invBaseN = 1.0f;
  uint64_t rev = 0;
  while (i > 0) {
    uint64_t next = i / base;
    uint64_t digit = i - next * base;
    rev = rev * base + digit;
    invBaseN *= invBase;
    i = (uint32_t)next;
  }
  float v = (float)rev * invBaseN;
  return v < 1.0f ? v : 0.9999999f;
}
static const int LDS_PRIMES[16] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41, 43, 47, 53};

// pcg4d (Jarzynski & Olano, "Hash Functions for GPU Rendering", JCGT 2020).
static inline uint32_t pcg4d_x(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  uint32_t v0 = a * 1664525u + 1013904223u, v1 = b * 1664525u + 1013904223u;
  uint32_t v2 = c * 1664525u + 1013904223u, v3 = d * 1664525u + 1013904223u;
  v0 += v1 * v3; v1 += v2 * v0; v2 += v0 * v1; v3 += v1 * v2;
  v0 ^= v0 >> 16; v1 ^= v1 >> 16; v2 ^= v2 >> 16; v3 ^= v3 >> 16;
  v0 += v1 * v3; v1 += v2 * v0; v2 += v0 * v1; v3 += v1 * v2;
  return v0;
}

enum Slot {
  S_LOBE = 0, S_LIGHT = 1, S_MESH = 2, S_TRI = 3, S_VNDF0 = 4, S_VNDF1 = 5, S_RR = 6,
  S_FRESNEL = 7, S_CHROMA = 8, S_HEMI0 = 9, S_HEMI1 = 10, S_POINT = 11, S_ENV0 = 12,
  S_ENV1 = 13, S_FLIGHT = 14, S_PHASE0 = 15, S_PHASE1 = 16, S_MEDRR = 17, S_EYETR = 18,
  S_DTSTEP = 19, S_DTACC = 20, S_EMIS = 21, S_VOLPICK = 22, S_VOLU = 23,
  S_LDS = 63
};

struct Ctx {
  uint32_t px, py, pixel, sample, seed, scramble;
  int dimBase;
  int vertex;  // next vertex index (surface hit or scatter event)
  void begin(uint32_t x, uint32_t y, uint32_t w, uint32_t s, uint32_t sd) {
    px = x; py = y; pixel = y * w + x; sample = s; seed = sd;
    scramble = hashPixel(x, y, sd - 1u);  // ldsBeginPixelSample, raycommon.cpp:65-69
    dimBase = 2; vertex = 0;
  }
  float prng(int v, int slot) const {
    const uint32_t h = pcg4d_x(pixel, sample, ((uint32_t)v << 6) | (uint32_t)slot, seed);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
  }
  // k-th draw of a repeated use at vertex v (delta-tracking steps, emission strata)
  float prngk(int v, int slot, int k) const {
    const uint32_t h = pcg4d_x(pixel, sample, ((uint32_t)k << 16) | ((uint32_t)v << 6) | (uint32_t)slot, seed);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
  }
  // ldsNext1D: raycommon.cpp:71-87 (dimension passed explicitly)
  float lds(int dim) const {
    if (dim >= 16) return prng(dim, S_LDS);
    const float v = radicalInverse(sample + 1u, LDS_PRIMES[dim]);
    const uint32_t hash = hashPixel((uint32_t)dim, 0u, scramble);
    const float offset = (float)(hash >> 8) * (1.0f / (float)(1u << 24));
    float w = v + offset;
    if (w >= 1.0f) w -= 1.0f;
    return w;
  }
  int ldsDirDim(int v) const { return dimBase + 4 * v; }
  int ldsNeeDim(int v) const { return dimBase + 4 * v + 2; }
};

static inline int pickIndex(float u, int n) {
  int i = (int)(u * (float)n);
  return i < n - 1 ? i : n - 1;
}

// cosineWeightedDirection: raycommon.cpp:94-115
static V3 cosineWeightedDirection(V3 normal, float r1, float r2) {
  float theta = acosf(sqrtf(1.0f - r1));
  float phi = 2.0f * kPi * r2;
  float x = sinf(theta) * cosf(phi);
  float y = sinf(theta) * sinf(phi);
  float z = cosf(theta);
  V3 tangent;
  if (fabsf(normal.x) > fabsf(normal.y)) tangent = normalize(cross(V3(0.0f, 1.0f, 0.0f), normal));
  else tangent = normalize(cross(V3(1.0f, 0.0f, 0.0f), normal));
  V3 bitangent = cross(normal, tangent);
  return normalize(tangent * x + bitangent * y + normal * z);
}

// ugm randomRayInHemisphere (not vendored): uniform direction on the sphere,
// flipped into the normal's hemisphere.
static V3 randomRayInHemisphere(V3 n, float u1, float u2) {
  const float z = 1.0f - 2.0f * u1;
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  const float phi = 2.0f * kPi * u2;
  V3 d(r * cosf(phi), r * sinf(phi), z);
  if (dot(d, n) < 0.0f) d = -d;
  return d;
}

// ldsPointInTriangle: raycommon.cpp:117-122 (u, v: two LDS draws)
static inline V3 ldsPointInTriangle(V3 v1, V3 v2, V3 v3, float u, float v) {
  if (u + v > 1.0f) { u = 1.0f - u; v = 1.0f - v; }
  return v1 + (v2 - v1) * u + (v3 - v1) * v;
}
// buildTangentFrame: bsdf.cpp:129-135
static inline void buildTangentFrame(V3 n, V3& t, V3& b) {
  const V3 up = fabsf(n.y) > 0.99f ? V3(1, 0, 0) : V3(0, 1, 0);
  t = normalize(cross(up, n));
  b = cross(n, t);
}
// sampleGGXVNDF: bsdf.cpp:139-161 (Heitz 2018), view direction in the local frame
static inline V3 sampleGGXVNDF(V3 Ve, float ax, float ay, float u1, float u2) {
  const V3 Vh = normalize(V3(ax * Ve.x, ay * Ve.y, Ve.z));
  const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
  const V3 T1 = lensq > 0.0f ? V3(-Vh.y, Vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : V3(1, 0, 0);
  const V3 T2 = cross(Vh, T1);
  const float rr = sqrtf(u1);
  const float phi = 2.0f * kPi * u2;
  const float t1 = rr * cosf(phi);
  float t2 = rr * sinf(phi);
  const float sw = 0.5f * (1.0f + Vh.z);
  t2 = (1.0f - sw) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + sw * t2;
  const V3 Nh = T1 * t1 + T2 * t2 + Vh * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2));
  return normalize(V3(ax * Nh.x, ay * Nh.y, fmaxf(0.0f, Nh.z)));
}
// smithG1: bsdf.cpp:164-170
static inline float smithG1Aniso(V3 w, float ax, float ay) {
  if (w.z <= 0.0f) return 0.0f;
  const float ax2 = (ax * w.x) * (ax * w.x), ay2 = (ay * w.y) * (ay * w.y);
  const float lambda = 0.5f * (sqrtf(1.0f + (ax2 + ay2) / (w.z * w.z)) - 1.0f);
  return 1.0f / (1.0f + lambda);
}

// ---------------------------------------------------------------- scene ----
struct Tri {
  V3 v1, v2, v3, n1, n2, n3;
  float uv[6];
  V3 npd;      // ti.normalizedpd
  float tia;   // ti.a
  float area;
  V3 bmin, bmax;
  int mesh, obj;
};

struct Material {
  C3 color;
  float glossy, roughness, transparency, refraction, ior, chroma, metallic, aniso, anisoRot,
      emission, spotRange;
  int texture;
  float tiling[2];
};

// ---- participating media (medium.h / medium.cpp) -------------------------
// The procedural fields are written in the reference's evaluation order; the
// device kernels evaluate the same expressions with explicit round-to-nearest
// operations, so with this file built without contraction the noise,
// density, emission and bending values agree bit for bit.

// Integer lattice hash -> [0, 1): medium.cpp:127-136
static inline float hash3(int x, int y, int z) {
  uint32_t h = (uint32_t)x * 374761393u + (uint32_t)y * 668265263u + (uint32_t)z * 2147483647u;
  h = (h ^ (h >> 13)) * 1274126177u;
  h ^= h >> 16;
  return (float)(h & 0x00FFFFFFu) / (float)0x01000000u;
}
static inline float smoothstep01(float x) { return x * x * (3.0f - 2.0f * x); }
// valueNoise3D: medium.cpp:142-163
static float valueNoise3D(float x, float y, float z) {
  const int xi = (int)floorf(x), yi = (int)floorf(y), zi = (int)floorf(z);
  const float xf = smoothstep01(x - (float)xi), yf = smoothstep01(y - (float)yi), zf = smoothstep01(z - (float)zi);
  const float c000 = hash3(xi, yi, zi), c100 = hash3(xi + 1, yi, zi);
  const float c010 = hash3(xi, yi + 1, zi), c110 = hash3(xi + 1, yi + 1, zi);
  const float c001 = hash3(xi, yi, zi + 1), c101 = hash3(xi + 1, yi, zi + 1);
  const float c011 = hash3(xi, yi + 1, zi + 1), c111 = hash3(xi + 1, yi + 1, zi + 1);
  const float x00 = c000 * (1.0f - xf) + c100 * xf;
  const float x10 = c010 * (1.0f - xf) + c110 * xf;
  const float x01 = c001 * (1.0f - xf) + c101 * xf;
  const float x11 = c011 * (1.0f - xf) + c111 * xf;
  const float y0 = x00 * (1.0f - yf) + x10 * yf;
  const float y1 = x01 * (1.0f - yf) + x11 * yf;
  return y0 * (1.0f - zf) + y1 * zf;
}
// fbmNormalised: medium.cpp:171-185 (densityAt's loop, :276-301, is the same)
static float fbmNormalised(float x, float y, float z, float freq, int octaves, float gain, float lac) {
  float fx = x * freq, fy = y * freq, fz = z * freq;
  float amp = 1.0f, total = 0.0f, ampSum = 0.0f;
  const int oct = octaves > 0 ? octaves : 1;
  for (int i = 0; i < oct; i++) {
    total += amp * valueNoise3D(fx, fy, fz);
    ampSum += amp;
    amp *= gain;
    fx *= lac; fy *= lac; fz *= lac;
  }
  return ampSum > 0.0f ? total / ampSum : 0.0f;
}

struct PathPt { V3 p; float radius, t; };

// HomogeneousMedium after prepare() and bake() (medium.cpp:18-101), camera space.
struct Medium {
  C3 sigma_s_eff, sigma_e_eff, sigma_t;
  float hero = 0.0f, g = 0.0f, density = 1.0f;
  int mode = 0, field = 0;  // emission mode (0 constant 1 cone 2 path), density field (0 none 1 fBm)
  bool hazeOn = false;      // heatHaze
  float tMaxHero = 0.0f;    // sigma_t_max_hero
  V3 coneOriginR, coneAxisR;
  float coneLength = 1, coneRadius = 0.3f, coneIntensity = 50, conePeakAxial = 0.15f, conePeakSharpness = 5;
  C3 coneInner, coneOuter;
  int coneSamples = 4;
  std::vector<PathPt> pathPointsR;
  int pathCount = 0;
  C3 pathInner, pathOuter;
  float pathIntensity = 1, pathFalloffPower = 2;
  int pathSamples = 6;
  float noiseFrequency = 1, noiseGain = 0.5f, noiseLacunarity = 2, noiseAmplitude = 1, noiseBias = 0;
  int noiseOctaves = 4;
  V3 noiseOffset;
  float iorAmplitude = 0.005f, iorFrequency = 4, iorGain = 0.5f, iorLacunarity = 2, iorFalloff = 0;
  int iorOctaves = 3, iorMarchSteps = 16;
  V3 iorOffset;

  static bool isZero3(const C3& c) { return c.x == 0.0f && c.y == 0.0f && c.z == 0.0f; }
  // medium.h:226-234
  bool active() const {
    if (hero > 0.0f) return true;
    if (mode == 1 && coneIntensity > 0.0f) return true;
    if (mode == 2 && pathIntensity > 0.0f && pathCount >= 2) return true;
    if (hazeOn && iorAmplitude > 0.0f) return true;
    return !isZero3(sigma_e_eff);
  }
  bool heatHaze() const { return hazeOn && iorAmplitude > 0.0f && iorMarchSteps > 0; }  // medium.h:240-242
  bool heterogeneous() const { return field != 0; }
  C3 transmittance(float d) const {            // medium.cpp:103-108
    if (d <= 0.0f) return C3(1, 1, 1);
    return C3(expf(-sigma_t.x * d), expf(-sigma_t.y * d), expf(-sigma_t.z * d));
  }
  static float ew(float st, float d) { return st < 1e-6f ? d : (1.0f - expf(-st * d)) / st; }
  C3 emissionAlongRay(float d) const {          // medium.cpp:118-123
    if (d <= 0.0f) return C3();
    return C3(sigma_e_eff.x * ew(sigma_t.x, d), sigma_e_eff.y * ew(sigma_t.y, d),
              sigma_e_eff.z * ew(sigma_t.z, d));
  }
  // densityAt: medium.cpp:276-301
  float densityAt(V3 p) const {
    if (field == 0) return 1.0f;
    const float n = fbmNormalised(p.x - noiseOffset.x, p.y - noiseOffset.y, p.z - noiseOffset.z, noiseFrequency,
                                  noiseOctaves, noiseGain, noiseLacunarity);
    return fmaxf(0.0f, noiseAmplitude * n + noiseBias);
  }
  // emissionAt: medium.cpp:303-404
  C3 emissionAt(V3 p) const {
    if (mode == 0) {
      if (field == 0) return sigma_e_eff;
      const float dn = densityAt(p);
      return C3(sigma_e_eff.x * dn, sigma_e_eff.y * dn, sigma_e_eff.z * dn);
    }
    if (mode == 2) {
      const size_t n = pathPointsR.size();
      if (n < 2) return C3();
      float bestD2 = std::numeric_limits<float>::infinity(), bestT = 0.0f, bestRadius = 0.0f;
      for (size_t i = 0; i + 1 < n; i++) {
        const PathPt& a = pathPointsR[i];
        const PathPt& b = pathPointsR[i + 1];
        const float abx = b.p.x - a.p.x, aby = b.p.y - a.p.y, abz = b.p.z - a.p.z;
        const float ab2 = abx * abx + aby * aby + abz * abz;
        if (ab2 < 1e-12f) continue;
        const float apx = p.x - a.p.x, apy = p.y - a.p.y, apz = p.z - a.p.z;
        float u = (apx * abx + apy * aby + apz * abz) / ab2;
        if (u < 0.0f) u = 0.0f;
        else if (u > 1.0f) u = 1.0f;
        const float qx = a.p.x + abx * u, qy = a.p.y + aby * u, qz = a.p.z + abz * u;
        const float dx = p.x - qx, dy = p.y - qy, dz = p.z - qz;
        const float d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < bestD2) {
          bestD2 = d2;
          bestT = a.t + (b.t - a.t) * u;
          bestRadius = a.radius + (b.radius - a.radius) * u;
        }
      }
      if (bestRadius <= 0.0f) return C3();
      if (bestD2 >= bestRadius * bestRadius) return C3();
      const float r = sqrtf(bestD2) / bestRadius;
      const float radial = powf(fmaxf(0.0f, 1.0f - r), pathFalloffPower);
      if (radial <= 0.0f) return C3();
      const float tb = bestT < 0.0f ? 0.0f : (bestT > 1.0f ? 1.0f : bestT);
      const C3 col(pathInner.x * (1.0f - tb) + pathOuter.x * tb, pathInner.y * (1.0f - tb) + pathOuter.y * tb,
                   pathInner.z * (1.0f - tb) + pathOuter.z * tb);
      float scale = radial * pathIntensity * fmaxf(0.0f, density);
      if (field != 0) scale *= densityAt(p);
      return C3(col.x * scale, col.y * scale, col.z * scale);
    }
    const float rx = p.x - coneOriginR.x, ry = p.y - coneOriginR.y, rz = p.z - coneOriginR.z;
    const float axialT = rx * coneAxisR.x + ry * coneAxisR.y + rz * coneAxisR.z;
    if (coneLength <= 0.0f) return C3();
    const float u = axialT / coneLength;
    if (u < 0.0f || u > 1.0f) return C3();
    const float px = rx - coneAxisR.x * axialT, py = ry - coneAxisR.y * axialT, pz = rz - coneAxisR.z * axialT;
    const float radial2 = px * px + py * py + pz * pz;
    if (coneRadius <= 0.0f) return C3();
    const float v2 = radial2 / (coneRadius * coneRadius);
    if (v2 > 1.0f) return C3();
    const float dx = (u - conePeakAxial) * conePeakSharpness;
    const float axialFalloff = expf(-(dx * dx));
    const float radialFalloff = (1.0f - v2) * (1.0f - v2);
    const float t = axialFalloff * radialFalloff;
    if (t <= 0.0f) return C3();
    const C3 col(coneInner.x * t + coneOuter.x * (1.0f - t), coneInner.y * t + coneOuter.y * (1.0f - t),
                 coneInner.z * t + coneOuter.z * (1.0f - t));
    float scale = t * coneIntensity * fmaxf(0.0f, density);
    if (field != 0) scale *= densityAt(p);
    return C3(col.x * scale, col.y * scale, col.z * scale);
  }
  // emissionIntegralAlongRay: medium.cpp:443-473 (jitter per stratum from the k-th draw)
  C3 emissionIntegral(const Ray& ray, float maxT, const Ctx& c, int v) const {
    if (mode == 0) return emissionAlongRay(maxT);
    if (maxT <= 0.0f) return C3();
    const int count = mode == 2 ? pathSamples : coneSamples;
    const int N = count > 0 ? count : 1;
    const float dt = maxT / (float)N;
    C3 acc;
    for (int i = 0; i < N; i++) {
      const float t = ((float)i + c.prngk(v, S_EMIS, i)) * dt;
      const V3 p(ray.o.x + ray.d.x * t, ray.o.y + ray.d.y * t, ray.o.z + ray.d.z * t);
      const C3 se = emissionAt(p);
      if (isZero3(se)) continue;
      const C3 tr = transmittance(t);
      acc.x += se.x * tr.x * dt;
      acc.y += se.y * tr.y * dt;
      acc.z += se.z * tr.z * dt;
    }
    return acc;
  }
  // sampleDeltaTracking: medium.cpp:406-441
  bool sampleDeltaTracking(const Ray& ray, float maxT, const Ctx& c, int v, float& outT, float& outDensity) const {
    if (tMaxHero <= 0.0f || maxT <= 0.0f) return false;
    const float peak = hero > 0.0f ? tMaxHero / hero : 1.0f;
    if (peak <= 0.0f) return false;
    float t = 0.0f;
    for (int i = 0; i < 64; i++) {
      const float xi = fminf(0.9999999f, fmaxf(0.0f, c.prngk(v, S_DTSTEP, i)));
      t += -logf(1.0f - xi) / tMaxHero;
      if (t >= maxT) return false;
      const V3 p(ray.o.x + ray.d.x * t, ray.o.y + ray.d.y * t, ray.o.z + ray.d.z * t);
      const float d = densityAt(p);
      const float pAccept = peak > 0.0f ? d / peak : 1.0f;
      if (c.prngk(v, S_DTACC, i) < pAccept) {
        outT = t;
        outDensity = d;
        return true;
      }
    }
    return false;
  }
  // iorAt: medium.cpp:186-215
  float iorAt(V3 p) const {
    if (!hazeOn) return 1.0f;
    const float n = fbmNormalised(p.x - iorOffset.x, p.y - iorOffset.y, p.z - iorOffset.z, iorFrequency, iorOctaves,
                                  iorGain, iorLacunarity);
    float ampMul = 1.0f;
    if (iorFalloff != 0.0f && coneLength > 0.0f) {
      const float axialT = (p.x - coneOriginR.x) * coneAxisR.x + (p.y - coneOriginR.y) * coneAxisR.y +
                           (p.z - coneOriginR.z) * coneAxisR.z;
      float u = axialT / coneLength;
      if (u < 0.0f) u = 0.0f;
      else if (u > 1.0f) u = 1.0f;
      const float mag = iorFalloff < 0.0f ? -iorFalloff : iorFalloff;
      const float t = iorFalloff >= 0.0f ? u : (1.0f - u);
      ampMul = 1.0f - mag * t;
      if (ampMul < 0.0f) ampMul = 0.0f;
    }
    return 1.0f + iorAmplitude * ampMul * (n - 0.5f) * 2.0f;
  }
  // bendRay with iorGradientAt: medium.cpp:217-274
  Ray bendRay(const Ray& ray, float length) const {
    if (length <= 0.0f || !heatHaze())
      return Ray{V3(ray.o.x + ray.d.x * length, ray.o.y + ray.d.y * length, ray.o.z + ray.d.z * length), ray.d};
    const int N = iorMarchSteps;
    const float ds = length / (float)N;
    const float h = iorFrequency > 0.0f ? (0.5f / iorFrequency) : 0.05f;
    const float inv2h = 0.5f / h;
    V3 pos = ray.o, dir = ray.d;
    for (int i = 0; i < N; i++) {
      const V3 mid(pos.x + dir.x * (ds * 0.5f), pos.y + dir.y * (ds * 0.5f), pos.z + dir.z * (ds * 0.5f));
      const float n = iorAt(mid);
      const float gx = (iorAt(V3(mid.x + h, mid.y, mid.z)) - iorAt(V3(mid.x - h, mid.y, mid.z))) * inv2h;
      const float gy = (iorAt(V3(mid.x, mid.y + h, mid.z)) - iorAt(V3(mid.x, mid.y - h, mid.z))) * inv2h;
      const float gz = (iorAt(V3(mid.x, mid.y, mid.z + h)) - iorAt(V3(mid.x, mid.y, mid.z - h))) * inv2h;
      const float gd = gx * dir.x + gy * dir.y + gz * dir.z;
      const float px = gx - dir.x * gd, py = gy - dir.y * gd, pz = gz - dir.z * gd;
      const float invN = n > 1e-6f ? (1.0f / n) : 1.0f;
      const V3 nd(dir.x + px * (ds * invN), dir.y + py * (ds * invN), dir.z + pz * (ds * invN));
      const float l2 = nd.x * nd.x + nd.y * nd.y + nd.z * nd.z;
      if (l2 > 1e-12f) {
        const float invL = 1.0f / sqrtf(l2);
        dir = V3(nd.x * invL, nd.y * invL, nd.z * invL);
      }
      pos = V3(pos.x + dir.x * ds, pos.y + dir.y * ds, pos.z + dir.z * ds);
    }
    return Ray{pos, dir};
  }
  float sampleFreeFlight(float u) const {       // medium.cpp:475-480
    if (hero <= 0.0f) return 1e30f;
    const float xi = fminf(0.9999999f, fmaxf(0.0f, u));
    return -logf(1.0f - xi) / hero;
  }
  float freeFlightPdf(float t) const { return hero * expf(-hero * t); }       // medium.h:299-301
  float survival(float d) const { return expf(-hero * d); }                    // medium.h:306-308
  V3 samplePhase(V3 wo, float u1, float u2) const {                          // medium.cpp:496-517
    float cosTheta;
    if (fabsf(g) < 1e-3f) cosTheta = 1.0f - 2.0f * u1;
    else {
      const float sqr = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
      cosTheta = (1.0f + g * g - sqr * sqr) / (2.0f * g);
    }
    const float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
    const float phi = 2.0f * kPi * u2;
    V3 t1, t2;
    if (fabsf(wo.x) > fabsf(wo.y)) {
      const float inv = 1.0f / sqrtf(wo.x * wo.x + wo.z * wo.z);
      t1 = V3(-wo.z * inv, 0.0f, wo.x * inv);
    } else {
      const float inv = 1.0f / sqrtf(wo.y * wo.y + wo.z * wo.z);
      t1 = V3(0.0f, wo.z * inv, -wo.y * inv);
    }
    t2 = cross(wo, t1);
    return normalize(t1 * (sinTheta * cosf(phi)) + t2 * (sinTheta * sinf(phi)) + wo * cosTheta);
  }
  float phasePdf(V3 wo, V3 wi) const {                                         // medium.cpp:519-525
    const float c = dot(wo, wi);
    const float denom = 1.0f + g * g - 2.0f * g * c;
    return (1.0f - g * g) * (float)(1.0 / (4.0 * M_PI)) / (denom * sqrtf(fmaxf(1e-8f, denom)));
  }
};

// EmissiveVolumeSource (rayrenderer.h:71-75): the medium and, for constant
// emission, the owning object's location in camera space.
struct VolLight { int medium; V3 anchor; };

struct BVHNode {  // bvh.h:22-30
  V3 bmin; uint32_t firstOrLeft;
  V3 bmax; uint16_t count, axis;
};

struct PointLight { V3 pos, normal; int mat; };

struct Texture { int w, h, hdr; std::vector<float> rgba; };

struct Settings {
  int W, H, spp, shader, aa, colorSampling, denoise, levels;
  float sigC, sigN, sigD, intensity, clampMax;
  int adaptive, adaptiveBase, adaptiveMode;
  float adaptiveThreshold;
  C3 worldColor; float backColor[4];
  uint32_t seed; int maxDepth, rrDepth, lightFix, threads, mixTree;
};

struct Scene {
  std::vector<Tri> tris;
  std::vector<uint32_t> prims;
  std::vector<BVHNode> nodes;
  std::vector<std::vector<int>> meshTris;
  std::vector<int> meshObj;
  std::vector<std::vector<int>> objMeshes;
  std::vector<int> objMat, objMedium;
  std::vector<Material> mats;
  std::vector<Medium> media;
  int globalMedium = -1;
  std::vector<VolLight> vols;    // emissive volumes, object order
  std::vector<int> areaLights;   // object ids
  std::vector<PointLight> points;
  std::vector<Texture> textures;
  // equirectangular environment (Scene::envmap*, scene.h:187-190)
  int envTex = -1;
  int envW = 0, envH = 0;
  float envIntensity = 1.0f, envCosY = 1.0f, envSinY = 0.0f, envTotal = 0.0f;
  std::vector<float> envMarg, envCond;  // H+1 ; H x (W+1)
  // cubemap environment (Scene::envCubemapFaces, scene.h:198-222): faces px nx py ny pz nz
  bool envCube = false;
  int envFace[6] = {-1, -1, -1, -1, -1, -1};
  int envCubeW = 0;                     // face size of the sampling CDF (0: none)
  float envCubeTotal = 0.0f;
  std::vector<float> cubeMargFace, cubeMargY, cubeCond;  // 7 ; 6 x (W+1) ; 6 x W x (W+1)
  // camera (RenderThreadContext, rayrenderer.cpp:97-132)
  V3 camLoc;
  float fov, viewNear, viewFar, dof, aperture, apertureRot, exposure;
  int blades;
  Settings st;
};

// ------------------------------------------------------------------ BVH ----
// TriangleBVH::build / buildRecursive: bvh.cpp:76-231
struct Bin { V3 bmin, bmax; int count; };
static inline void growBox(V3& mn, V3& mx, V3 bmn, V3 bmx) {
  mn = V3(fminf(mn.x, bmn.x), fminf(mn.y, bmn.y), fminf(mn.z, bmn.z));
  mx = V3(fmaxf(mx.x, bmx.x), fmaxf(mx.y, bmx.y), fmaxf(mx.z, bmx.z));
}
static inline float surfaceArea(V3 mn, V3 mx) {
  const float dx = mx.x - mn.x, dy = mx.y - mn.y, dz = mx.z - mn.z;
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct Builder {
  Scene& s;
  std::vector<V3> cent;
  int bins;
  void recurse(uint32_t nodeIdx, uint32_t first, uint32_t count) {
    V3 pmn(FLT_MAX, FLT_MAX, FLT_MAX), pmx(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    V3 cmn = pmn, cmx = pmx;
    for (uint32_t i = first; i < first + count; i++) {
      const Tri& t = s.tris[s.prims[i]];
      growBox(pmn, pmx, t.bmin, t.bmax);
      growBox(cmn, cmx, cent[i], cent[i]);
    }
    s.nodes[nodeIdx].bmin = pmn;
    s.nodes[nodeIdx].bmax = pmx;
    auto makeLeaf = [&]() {
      s.nodes[nodeIdx].firstOrLeft = first;
      s.nodes[nodeIdx].count = (uint16_t)std::min<uint32_t>(count, 0xFFFFu);
      s.nodes[nodeIdx].axis = 0;
    };
    if (count <= 4) { makeLeaf(); return; }
    const V3 cext = cmx - cmn;
    int axis = 0;
    if (cext.y > cext.x) axis = 1;
    if (cext.z > ((axis == 0) ? cext.x : cext.y)) axis = 2;
    const float cmin = cmn[axis];
    const float cextAxis = cext[axis];
    if (cextAxis < 1e-12f) { makeLeaf(); return; }
    const float scale = (float)bins / cextAxis;
    std::vector<Bin> bb(bins, Bin{V3(FLT_MAX, FLT_MAX, FLT_MAX), V3(-FLT_MAX, -FLT_MAX, -FLT_MAX), 0});
    auto binOf = [&](uint32_t i) {
      int b = (int)((cent[i][axis] - cmin) * scale);
      if (b < 0) b = 0;
      if (b >= bins) b = bins - 1;
      return b;
    };
    for (uint32_t i = first; i < first + count; i++) {
      const int b = binOf(i);
      const Tri& t = s.tris[s.prims[i]];
      growBox(bb[b].bmin, bb[b].bmax, t.bmin, t.bmax);
      bb[b].count++;
    }
    std::vector<float> la(bins - 1), ra(bins - 1);
    std::vector<int> lc(bins - 1), rc(bins - 1);
    {
      V3 mn(FLT_MAX, FLT_MAX, FLT_MAX), mx(-FLT_MAX, -FLT_MAX, -FLT_MAX);
      int c = 0;
      for (int i = 0; i < bins - 1; i++) {
        if (bb[i].count > 0) growBox(mn, mx, bb[i].bmin, bb[i].bmax);
        c += bb[i].count;
        la[i] = c > 0 ? surfaceArea(mn, mx) : 0.0f;
        lc[i] = c;
      }
      mn = V3(FLT_MAX, FLT_MAX, FLT_MAX); mx = V3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
      c = 0;
      for (int i = bins - 1; i > 0; i--) {
        if (bb[i].count > 0) growBox(mn, mx, bb[i].bmin, bb[i].bmax);
        c += bb[i].count;
        ra[i - 1] = c > 0 ? surfaceArea(mn, mx) : 0.0f;
        rc[i - 1] = c;
      }
    }
    const float parentArea = surfaceArea(pmn, pmx);
    const float invParent = parentArea > 0.0f ? 1.0f / parentArea : 0.0f;
    float bestCost = (float)count * 1.5f;
    int bestBin = -1;
    for (int i = 0; i < bins - 1; i++) {
      if (lc[i] == 0 || rc[i] == 0) continue;
      const float cost = 1.0f + 1.5f * invParent * (la[i] * lc[i] + ra[i] * rc[i]);
      if (cost < bestCost) { bestCost = cost; bestBin = i; }
    }
    if (bestBin < 0) { makeLeaf(); return; }
    uint32_t mid = first;
    for (uint32_t i = first; i < first + count; i++) {
      if (binOf(i) <= bestBin) {
        std::swap(s.prims[i], s.prims[mid]);
        std::swap(cent[i], cent[mid]);
        mid++;
      }
    }
    const uint32_t leftCount = mid - first, rightCount = count - leftCount;
    if (leftCount == 0 || rightCount == 0) { makeLeaf(); return; }
    const uint32_t leftIdx = (uint32_t)s.nodes.size();
    s.nodes.emplace_back();
    s.nodes.emplace_back();
    s.nodes[nodeIdx].firstOrLeft = leftIdx;
    s.nodes[nodeIdx].count = 0;
    s.nodes[nodeIdx].axis = (uint16_t)axis;
    recurse(leftIdx, first, leftCount);
    recurse(leftIdx + 1, mid, rightCount);
  }
};

static void buildBVH(Scene& s, int bins) {
  s.nodes.clear();
  s.prims.resize(s.tris.size());
  for (size_t i = 0; i < s.tris.size(); i++) s.prims[i] = (uint32_t)i;
  if (s.tris.empty()) return;
  Builder b{s, {}, bins};
  b.cent.resize(s.tris.size());
  for (size_t i = 0; i < s.tris.size(); i++)
    b.cent[i] = (s.tris[i].bmin + s.tris[i].bmax) * 0.5f;
  s.nodes.reserve(s.tris.size() * 2);
  s.nodes.emplace_back();
  b.recurse(0, 0, (uint32_t)s.tris.size());
}

struct HitInfo {  // RayTriangleIntersectionInfo, raycommon.h:168-180
  int tri = -1;
  float t = MAX_RAY_DISTANCE;
  V3 hit;
  float u = 0, v = 0, w = 0;
};

// Triangle-test products in a fixed FMA form (the device evaluates the same
// operations in the same order, so hits agree bit for bit):
//   dotF(a, b) = fma(a.z, b.z, fma(a.y, b.y, a.x * b.x)); crossF likewise per component.
static inline float dotF(V3 a, V3 b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
static inline V3 crossF(V3 a, V3 b) {
  return V3(fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x)));
}

// RenderMeshTriangle::intersectsRay(closest): raycommon.cpp:200-235
static inline bool intersectClosestTri(const Tri& tr, int id, const Ray& ray, HitInfo& info) {
  const V3 edge1 = tr.v2 - tr.v1;
  const V3 edge2 = tr.v3 - tr.v1;
  const V3 pvec = crossF(ray.d, edge2);
  const float det = dotF(edge1, pvec);
  if (fabsf(det) < 1e-8f) return false;
  const float invDet = 1.0f / det;
  const V3 tvec = ray.o - tr.v1;
  const float u = dotF(tvec, pvec) * invDet;
  if (u < 0.0f || u > 1.0f) return false;
  const V3 qvec = crossF(tvec, edge1);
  const float v = dotF(ray.d, qvec) * invDet;
  if (v < 0.0f || u + v > 1.0f) return false;
  const float t = dotF(edge2, qvec) * invDet;
  if (t < 0.0f) return false;
  if (t >= info.t) return false;
  info.t = t;
  info.hit = ray.o + ray.d * t;
  info.u = u; info.v = v; info.w = 1.0f - u - v;
  info.tri = id;
  return true;
}

// RenderMeshTriangle::intersectsRay(any): raycommon.cpp:151-198
static inline bool intersectAnyTri(const Tri& tr, const Ray& ray, float maxt) {
  const float EPS = 1e-6f;
  const V3 edge1 = tr.v2 - tr.v1;
  const V3 edge2 = tr.v3 - tr.v1;
  const V3 h = crossF(ray.d, edge2);
  const float a = dotF(edge1, h);
  if (fabsf(a) < EPS) return false;
  const float f = 1.0f / a;
  const V3 s = ray.o - tr.v1;
  const float u = f * dotF(s, h);
  if (u < 0.0f || u > 1.0f) return false;
  const V3 q = crossF(s, edge1);
  const float v = f * dotF(ray.d, q);
  if (v < 0.0f || u + v > 1.0f) return false;
  const float t = f * dotF(edge2, q);
  return t > EPS && t < maxt;
}

static inline bool slab(const BVHNode& n, const Ray& r, V3 inv, float tcap) {
  const float t1x = (n.bmin.x - r.o.x) * inv.x, t2x = (n.bmax.x - r.o.x) * inv.x;
  const float t1y = (n.bmin.y - r.o.y) * inv.y, t2y = (n.bmax.y - r.o.y) * inv.y;
  const float t1z = (n.bmin.z - r.o.z) * inv.z, t2z = (n.bmax.z - r.o.z) * inv.z;
  const float tmin = fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fminf(t1z, t2z));
  const float tmax = fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fmaxf(t1z, t2z));
  return !(tmax < 0.0f || tmin > tmax || tmin > tcap);
}
static inline V3 invDir(V3 d) {
  return V3(fabsf(d.x) > 1e-20f ? 1.0f / d.x : 1e30f, fabsf(d.y) > 1e-20f ? 1.0f / d.y : 1e30f,
            fabsf(d.z) > 1e-20f ? 1.0f / d.z : 1e30f);
}

// TriangleBVH::intersectClosest: bvh.cpp:233-285
static bool intersectClosest(const Scene& s, const Ray& ray, HitInfo& info) {
  if (s.nodes.empty()) return false;
  const V3 inv = invDir(ray.d);
  const int dirSign[3] = {inv.x < 0.0f, inv.y < 0.0f, inv.z < 0.0f};
  uint32_t stack[64];
  int sp = 0;
  stack[sp++] = 0;
  bool any = false;
  while (sp > 0) {
    const BVHNode& n = s.nodes[stack[--sp]];
    if (!slab(n, ray, inv, info.t)) continue;
    if (n.count > 0) {
      for (uint16_t i = 0; i < n.count; i++) {
        const uint32_t id = s.prims[n.firstOrLeft + i];
        if (intersectClosestTri(s.tris[id], (int)id, ray, info)) any = true;
      }
    } else {
      const uint32_t l = n.firstOrLeft, r = l + 1;
      if (dirSign[n.axis]) { stack[sp++] = l; stack[sp++] = r; }
      else { stack[sp++] = r; stack[sp++] = l; }
    }
  }
  return any;
}

enum Pred { P_AREA = 0, P_POINT = 1, P_AO = 2, P_ALL = 3, P_VOL = 4 };
// occluder predicates: rayrenderer.cpp:1956-1959 (area), :2211-2215 (point/env), :2388-2390 (AO)
static inline bool occluder(const Scene& s, int tri, int pred) {
  const Material& m = s.mats[s.objMat[s.tris[tri].obj]];
  switch (pred) {
    case P_AREA: return m.transparency < 0.01f && m.emission <= 0.0f;
    case P_POINT: if (m.emission > 0.0f) return false; return m.transparency < 0.01f || m.refraction > 0.1f;
    case P_AO: return m.transparency < 0.01f;
    case P_VOL: if (m.emission > 0.0f) return false; return m.transparency < 0.01f && m.refraction <= 0.1f;  // rayrenderer.cpp:2167-2171
    default: return true;
  }
}

// TriangleBVH::intersectAny: bvh.h:63-101
static bool intersectAny(const Scene& s, const Ray& ray, float maxT, int pred) {
  if (s.nodes.empty()) return false;
  const V3 inv = invDir(ray.d);
  uint32_t stack[64];
  int sp = 0;
  stack[sp++] = 0;
  while (sp > 0) {
    const BVHNode& n = s.nodes[stack[--sp]];
    if (!slab(n, ray, inv, maxT)) continue;
    if (n.count > 0) {
      for (uint16_t i = 0; i < n.count; i++) {
        const uint32_t id = s.prims[n.firstOrLeft + i];
        if (intersectAnyTri(s.tris[id], ray, maxT) && occluder(s, (int)id, pred)) return true;
      }
    } else {
      stack[sp++] = n.firstOrLeft + 1;
      stack[sp++] = n.firstOrLeft;
    }
  }
  return false;
}

// ------------------------------------------------------------- shading ----
struct Vi { V3 normal; float uvx = 0, uvy = 0; };

// calcVertexInterpolation(info): rayrenderer.cpp:2354-2362
static Vi interp(const Scene& s, const HitInfo& h) {
  const Tri& t = s.tris[h.tri];
  Vi vi;
  vi.uvx = t.uv[0] * h.w + t.uv[2] * h.u + t.uv[4] * h.v;
  vi.uvy = t.uv[1] * h.w + t.uv[3] * h.u + t.uv[5] * h.v;
  vi.normal = normalize(t.n1 * h.w + t.n2 * h.u + t.n3 * h.v);
  return vi;
}
// calcVertexInterpolation(tri, p): rayrenderer.cpp:2337-2352 (unnormalised)
static V3 interpAt(const Tri& t, V3 p) {
  const V3 f1 = t.v1 - p, f2 = t.v2 - p, f3 = t.v3 - p;
  const float a1 = length(cross(f2, f3)) * t.tia;
  const float a2 = length(cross(f3, f1)) * t.tia;
  const float a3 = length(cross(f1, f2)) * t.tia;
  return t.n1 * a1 + t.n2 * a2 + t.n3 * a3;
}
// geomNormal: bsdf.cpp:27-30
static inline V3 geomNormal(const Tri& t, V3 shadingN) {
  return dot(t.npd, shadingN) >= 0.0f ? t.npd : -t.npd;
}
// srgbToLinear / Texture::sample: texture.cpp:204-241
static inline float srgbToLinear(float c) {
  if (c <= 0.04045f) return c * (1.0f / 12.92f);
  return powf((c + 0.055f) * (1.0f / 1.055f), 2.4f);
}
static C3 texSample(const Scene& s, int tex, float u, float v) {
  const Texture& T = s.textures[tex];
  if (T.w <= 0 || T.h <= 0) return C3();
  if (!(u == u) || !(v == v)) return C3();
  float fu = u - floorf(u), fv = v - floorf(v);
  if (fu < 0.0f || fu >= 1.0f) fu = 0.0f;
  if (fv < 0.0f || fv >= 1.0f) fv = 0.0f;
  int x = std::min(std::max((int)(fu * T.w), 0), T.w - 1);
  int y = std::min(std::max((int)(fv * T.h), 0), T.h - 1);
  const float* p = &T.rgba[((size_t)y * T.w + x) * 4];
  C3 c(p[0], p[1], p[2]);
  if (!T.hdr) c = C3(srgbToLinear(c.x), srgbToLinear(c.y), srgbToLinear(c.z));
  return c;
}
static C3 albedoOf(const Scene& s, const Material& m, const Vi& vi) {
  C3 a = m.color;
  if (m.texture >= 0) a = a * texSample(s, m.texture, vi.uvx * m.tiling[0], vi.uvy * m.tiling[1]);
  return a;
}

struct Param {  // BSDFParam, bsdf.h:20-61
  const HitInfo* info;
  Ray inray;
  Vi vi;
  int passes = 0;
  C3 throughput = C3(1, 1, 1);
  float bsdfPdf = 0.0f;
  int chroma = -1;
  int medium = -1;
  int vertex = 0;
};

struct Tracer {
  const Scene& s;
  Ctx& c;
  Tracer(const Scene& sc, Ctx& cx) : s(sc), c(cx) {}

  const Material& matOfTri(int tri) const { return s.mats[s.objMat[s.tris[tri].obj]]; }

  // areaLightSampledArea: rayrenderer.cpp:1910-1914
  float sampledArea(int tri) const {
    const Tri& t = s.tris[tri];
    return (float)s.meshTris[t.mesh].size() * t.area;
  }
  float lightCountFactor() const {
    return s.st.lightFix ? (float)s.areaLights.size() : 1.0f;
  }

  // Uniform (object, mesh, triangle, point) pick shared by traceAreaLight and
  // sampleAreaLightForNEE; returns false when the object has no triangles.
  bool pickLightPoint(int lightObj, int v, int& tri, V3& p) const {
    const auto& meshes = s.objMeshes[lightObj];
    if (meshes.empty()) return false;
    const int mesh = meshes[pickIndex(c.prng(v, S_MESH), (int)meshes.size())];
    const auto& tl = s.meshTris[mesh];
    if (tl.empty()) return false;
    tri = tl[pickIndex(c.prng(v, S_TRI), (int)tl.size())];
    const Tri& t = s.tris[tri];
    p = ldsPointInTriangle(t.v1, t.v2, t.v3, c.lds(c.ldsNeeDim(v)), c.lds(c.ldsNeeDim(v) + 1));
    return true;
  }

  // traceAreaLight: rayrenderer.cpp:1916-1984
  C3 traceAreaLight(int lightObj, V3 hit, V3 n, int v) const {
    int tri; V3 p;
    if (!pickLightPoint(lightObj, v, tri, p)) return C3();
    const V3 lightRay = p - hit;
    const V3 lightDir = normalize(lightRay);
    const float dotObj = dot(lightDir, n);
    if (dotObj <= 0.0f) return C3();
    const V3 ln = interpAt(s.tris[tri], p);
    const float dotLight = dot(-lightDir, ln);
    if (dotLight <= 0.0f) return C3();
    const Ray ray = SurfaceRay(hit, lightRay, n);
    if (intersectAny(s, ray, 0.99999f, P_AREA)) return C3();
    const Material& lm = s.mats[s.objMat[lightObj]];
    const float area = sampledArea(tri);
    const float r2 = dot(lightRay, lightRay);
    const float pl = r2 / (dotLight * area) / lightCountFactor();
    const float pb = dotObj / kPi;
    const float wl = pl * pl / (pl * pl + pb * pb);
    return lm.color * lm.emission * (dotObj * dotLight * area / (kPi * r2)) * wl * lightCountFactor();
  }

  // sampleAreaLightForNEE: rayrenderer.cpp:1986-2036
  bool sampleAreaLightForNEE(V3 hit, V3 n, int v, V3& outDir, float& outPdf, C3& outLe) const {
    const int N = (int)s.areaLights.size();
    if (N <= 0) return false;
    const int lo = s.areaLights[pickIndex(c.prng(v, S_LIGHT), N)];
    int tri; V3 p;
    if (!pickLightPoint(lo, v, tri, p)) return false;
    const V3 lightRay = p - hit;
    const V3 dir = normalize(lightRay);
    const float cosObj = dot(dir, n);
    if (cosObj <= 0.0f) return false;
    const V3 ln = interpAt(s.tris[tri], p);
    const float cosLight = dot(-dir, ln);
    if (cosLight <= 0.0f) return false;
    const Ray sr = SurfaceRay(hit, lightRay, n);
    if (intersectAny(s, sr, 0.99999f, P_AREA)) return false;
    const Material& lm = s.mats[s.objMat[lo]];
    const float r2 = dot(lightRay, lightRay);
    outDir = dir;
    outPdf = r2 / (cosLight * sampledArea(tri)) / lightCountFactor();
    outLe = lm.color * lm.emission;
    return true;
  }

  // sampleVolumeLightForNEE: rayrenderer.cpp:2067-2203 (the volume pick and
  // the equiangular draw come from this vertex's own keys)
  bool sampleVolumeLightForNEE(V3 hit, V3 n, int v, V3& outDir, float& outPdf, C3& outLe) const {
    const int N = (int)s.vols.size();
    if (N <= 0) return false;
    const VolLight& ev = s.vols[pickIndex(c.prng(v, S_VOLPICK), N)];
    const Medium& m = s.media[ev.medium];
    V3 segA, segB;
    if (m.mode == 1) {
      segA = m.coneOriginR;
      segB = m.coneOriginR + m.coneAxisR * m.coneLength;
    } else {
      segA = ev.anchor;
      segB = segA;
    }
    const V3 segDir = segB - segA;
    const float segLen = length(segDir);
    const V3 axis = segLen > 1e-6f ? segDir * (1.0f / segLen) : V3(0.0f, 0.0f, -1.0f);
    const V3 toA = segA - hit;
    const float along = dot(toA, axis);
    const V3 perp = toA - axis * along;
    const float D = length(perp);
    if (!(D > 1e-5f) && segLen <= 1e-6f) return false;
    const float thA = atanf(along / fmaxf(D, 1e-5f)), thB = atanf((along + segLen) / fmaxf(D, 1e-5f));
    if (!(fabsf(thB - thA) > 1e-6f) && segLen > 1e-6f) return false;
    const float theta = thA + c.prng(v, S_VOLU) * (thB - thA);
    const float tS = D * tanf(theta);
    const V3 sp = segLen > 1e-6f ? segA + axis * (tS - along) : segA;
    const V3 toS = sp - hit;
    const float r2 = dot(toS, toS);
    const float r = sqrtf(r2);
    if (!(r > 1e-5f)) return false;
    if (intersectAny(s, SurfaceRay(hit, toS, n), 0.99999f, P_VOL)) return false;
    C3 se = m.emissionAt(sp);
    if (isZero(se)) return false;
    if (m.hero > 0.0f) se = se * m.transmittance(r);
    const float pdfT = D / (fmaxf(1e-6f, fabsf(thB - thA)) * (D * D + tS * tS));
    outDir = toS * (1.0f / r);
    outPdf = pdfT * r2 * (float)N;
    outLe = se;
    return true;
  }

  // tracePointLight: rayrenderer.cpp:2205-2269
  C3 tracePointLight(const PointLight& pl, V3 hit, V3 n) const {
    const V3 lightray = pl.pos - hit;
    const Ray ray = SurfaceRay(hit, lightray, n);
    if (intersectAny(s, ray, 0.99999f, P_POINT)) return C3();
    const V3 ldir = normalize(lightray);
    const float dotToObject = dot(ldir, n);
    float dotToLight = dot(ldir, pl.normal);
    if (!(dotToObject > 0.0f)) return C3();
    const Material& lm = s.mats[pl.mat];
    if (lm.spotRange > 0.0f) {
      const float spotDot = cosf(lm.spotRange * 0.5f * (180.0f / kPi));  // RADIAN_TO_DEGREE as written
      const float e0 = fmaxf(spotDot - 0.1f, 0.0f), e1 = fminf(spotDot + 0.1f, 1.0f);
      float x = (dotToLight - e0) / (e1 - e0);
      x = fminf(fmaxf(x, 0.0f), 1.0f);
      dotToLight = dotToLight * (x * x * (3.0f - 2.0f * x));
    } else {
      dotToLight = fabsf(dotToObject);
    }
    if (!(dotToLight > 0.0f)) return C3();
    const float da = powf(length(lightray), -2.0f);
    const float lum = lm.emission * dotToLight * da;
    C3 col = lm.color * lum;
    return C3(fminf(fmaxf(col.x, 0.0f), 1.0f), fminf(fmaxf(col.y, 0.0f), 1.0f), fminf(fmaxf(col.z, 0.0f), 1.0f));
  }

  // traceLight: rayrenderer.cpp:2271-2293
  C3 traceLight(V3 hit, V3 n, int v) const {
    C3 a, p;
    const int na = (int)s.areaLights.size(), np = (int)s.points.size();
    if (na > 0) a = traceAreaLight(s.areaLights[pickIndex(c.prng(v, S_LIGHT), na)], hit, n, v);
    if (np > 0) {
      if (np == 1) p = tracePointLight(s.points[0], hit, n);
      else p = tracePointLight(s.points[pickIndex(c.prng(v, S_POINT), np)], hit, n);
    }
    return a + p;
  }

  // ---- environment map: equirectangular or cubemap ----------------------
  bool envSampling() const { return s.envTex >= 0 && s.envW > 0 && s.envTotal > 0.0f; }
  bool cubeSampling() const { return s.envCubeW > 0 && s.envCubeTotal > 0.0f; }
  // face and face-local (s, t) of a rotated direction (OpenGL convention, rayrenderer.cpp:1311-1333)
  static int cubeFace(float rx, float ry, float rz, float& sc, float& tc, float& ma) {
    const float ax = fabsf(rx), ay = fabsf(ry), az = fabsf(rz);
    int face;
    if (ax >= ay && ax >= az) {
      ma = ax;
      if (rx > 0) { face = 0; sc = -rz; tc = ry; }
      else { face = 1; sc = rz; tc = ry; }
    } else if (ay >= ax && ay >= az) {
      ma = ay;
      if (ry > 0) { face = 2; sc = rx; tc = rz; }
      else { face = 3; sc = rx; tc = -rz; }
    } else {
      ma = az;
      if (rz > 0) { face = 4; sc = rx; tc = ry; }
      else { face = 5; sc = -rx; tc = ry; }
    }
    return face;
  }
  const float* cubeTexel(int face, int x, int y) const {
    return &s.textures[s.envFace[face]].rgba[((size_t)y * s.envCubeW + x) * 4];
  }
  const float* envTexel(int x, int y) const {
    return &s.textures[s.envTex].rgba[((size_t)y * s.envW + x) * 4];
  }
  static float texelLum(const float* c) { return fmaxf(0.0f, 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]); }

  // sampleEnvironment, equirectangular branch (rayrenderer.cpp:1299-1348):
  // view-space direction, yaw about +Y, lat-long lookup through Texture::sample.
  C3 sampleEnvironment(V3 dir) const {
    if (s.envTex < 0 && !s.envCube) return C3();
    const V3 d = normalize(dir);
    const float rx = d.x * s.envCosY - d.z * s.envSinY;
    const float rz = d.x * s.envSinY + d.z * s.envCosY;
    if (s.envCube) {  // the cubemap takes precedence (rayrenderer.cpp:1310-1340)
      float sc, tc, ma;
      const int face = cubeFace(rx, d.y, rz, sc, tc, ma);
      const float u = 0.5f * (sc / ma + 1.0f);
      const float v = 0.5f * (1.0f - tc / ma);
      return texSample(s, s.envFace[face], u, v) * s.envIntensity;
    }
    const float u = 0.5f + atan2f(rz, rx) * (float)(0.5 / M_PI);
    const float v = 0.5f - asinf(fminf(fmaxf(d.y, -1.0f), 1.0f)) * (float)(1.0 / M_PI);
    return texSample(s, s.envTex, u, v) * s.envIntensity;
  }

  // envmapDirectionPdf, equirectangular branch (rayrenderer.cpp:1521-1573)
  float envmapDirectionPdf(V3 dir) const {
    const V3 d = normalize(dir);
    const float rx = d.x * s.envCosY - d.z * s.envSinY;
    const float rz = d.x * s.envSinY + d.z * s.envCosY;
    if (cubeSampling()) {  // rayrenderer.cpp:1530-1555
      float sc, tc, ma;
      const int face = cubeFace(rx, d.y, rz, sc, tc, ma);
      if (ma <= 0.0f) return 0.0f;
      const float u = 0.5f * (sc / ma + 1.0f);
      const float v = 0.5f * (1.0f - tc / ma);
      const int W = s.envCubeW;
      int x = (int)(u * W); if (x < 0) x = 0; if (x >= W) x = W - 1;
      int y = (int)(v * W); if (y < 0) y = 0; if (y >= W) y = W - 1;
      const float lum = texelLum(cubeTexel(face, x, y));
      return lum * (float)(W * W) / (4.0f * s.envCubeTotal);
    }
    if (!envSampling()) return 0.0f;
    const int W = s.envW, H = s.envH;
    const float u = 0.5f + atan2f(rz, rx) * (float)(0.5 / M_PI);
    const float v = 0.5f - asinf(fminf(fmaxf(d.y, -1.0f), 1.0f)) * (float)(1.0 / M_PI);
    int x = (int)(u * W); if (x < 0) x = 0; if (x >= W) x = W - 1;
    int y = (int)(v * H); if (y < 0) y = 0; if (y >= H) y = H - 1;
    const float lum = texelLum(envTexel(x, y));
    const float sinTheta = sinf((float)M_PI * v);
    if (sinTheta <= 0.0f) return 0.0f;
    const float pdfUV = (lum * sinTheta) / s.envTotal;
    return pdfUV * (float)(W * H) / (2.0f * (float)(M_PI * M_PI) * sinTheta);
  }

  // searchCDF (rayrenderer.cpp:1353-1362): largest i with cdf[i] <= u in [0, n-1]
  static int searchCDF(const float* cdf, int n, float u) {
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (cdf[mid + 1] <= u) lo = mid + 1;
      else hi = mid;
    }
    return lo < n ? lo : n - 1;
  }

  // sampleEnvmapDirection, equirectangular branch (rayrenderer.cpp:1426-1482)
  void sampleEnvmapDirection(float u0, float u1, V3& outDir, float& outPdf) const {
    outDir = V3(0, 1, 0);
    outPdf = 0.0f;
    if (cubeSampling()) {  // face, row, texel from the three-level CDF (rayrenderer.cpp:1384-1433)
      const int W = s.envCubeW, H = W;
      const int face = searchCDF(s.cubeMargFace.data(), 6, u0);
      const float faceLo = s.cubeMargFace[face], faceSpan = s.cubeMargFace[face + 1] - faceLo;
      const float u0r = faceSpan > 0.0f ? (u0 - faceLo) / faceSpan : 0.5f;
      const float* marY = &s.cubeMargY[(size_t)face * (H + 1)];
      const int y = searchCDF(marY, H, u0r);
      const float yLo = marY[y], ySpan = marY[y + 1] - yLo;
      const float yFrac = ySpan > 0.0f ? (u0r - yLo) / ySpan : 0.5f;
      const float* condX = &s.cubeCond[((size_t)face * H + y) * (W + 1)];
      const int x = searchCDF(condX, W, u1);
      const float xLo = condX[x], xSpan = condX[x + 1] - xLo;
      const float xFrac = xSpan > 0.0f ? (u1 - xLo) / xSpan : 0.5f;
      const float u = (x + xFrac) / (float)W;
      const float v = (y + yFrac) / (float)H;
      const float sc = 2.0f * u - 1.0f, tc = 1.0f - 2.0f * v;
      V3 l;  // cubeFaceDir (rayrenderer.cpp:1367-1376)
      switch (face) {
        case 0: l = V3(1.0f, tc, -sc); break;
        case 1: l = V3(-1.0f, tc, sc); break;
        case 2: l = V3(sc, 1.0f, tc); break;
        case 3: l = V3(sc, -1.0f, -tc); break;
        case 4: l = V3(sc, tc, 1.0f); break;
        default: l = V3(-sc, tc, -1.0f); break;
      }
      outDir = normalize(V3(l.x * s.envCosY + l.z * s.envSinY, l.y, -l.x * s.envSinY + l.z * s.envCosY));
      const float lum = texelLum(cubeTexel(face, x, y));
      outPdf = lum * (float)(W * H) / (4.0f * s.envCubeTotal);
      return;
    }
    if (!envSampling()) return;
    const int W = s.envW, H = s.envH;
    const int y = searchCDF(s.envMarg.data(), H, u0);
    const float* row = &s.envCond[(size_t)y * (W + 1)];
    const int x = searchCDF(row, W, u1);
    const float yPrev = s.envMarg[y], ySpan = s.envMarg[y + 1] - yPrev;
    const float xPrev = row[x], xSpan = row[x + 1] - xPrev;
    const float yFrac = ySpan > 0.0f ? (u0 - yPrev) / ySpan : 0.5f;
    const float xFrac = xSpan > 0.0f ? (u1 - xPrev) / xSpan : 0.5f;
    const float u = (x + xFrac) / (float)W;
    const float v = (y + yFrac) / (float)H;
    const float phi = (u - 0.5f) * 2.0f * (float)M_PI;
    const float theta = (0.5f - v) * (float)M_PI;
    const float cosT = cosf(theta);
    const float dx = cosT * cosf(phi), dy = sinf(theta), dz = cosT * sinf(phi);
    const float wx = dx * s.envCosY + dz * s.envSinY;
    const float wz = -dx * s.envSinY + dz * s.envCosY;
    outDir = normalize(V3(wx, dy, wz));
    const float lum = texelLum(envTexel(x, y));
    const float sinTheta = sinf((float)M_PI * v);
    if (sinTheta <= 0.0f) return;
    const float pdfUV = (lum * sinTheta) / s.envTotal;
    outPdf = pdfUV * (float)(W * H) / (2.0f * (float)(M_PI * M_PI) * sinTheta);
  }

  // sampleEnvmapForNEE (rayrenderer.cpp:2038-2065): luminance-IS direction,
  // front-facing test, unbounded shadow ray with the point/env occluders.
  bool sampleEnvmapForNEE(V3 hit, V3 n, int v, V3& outDir, float& outPdf, C3& outLi) const {
    if (!envSampling() && !cubeSampling()) return false;
    V3 dir;
    float pdf = 0.0f;
    sampleEnvmapDirection(c.prng(v, S_ENV0), c.prng(v, S_ENV1), dir, pdf);
    if (pdf <= 0.0f) return false;
    if (dot(dir, n) <= 0.0f) return false;
    if (intersectAny(s, SurfaceRay(hit, dir, n), 1e30f, P_POINT)) return false;
    outDir = dir;
    outPdf = pdf;
    outLi = sampleEnvironment(dir);
    return true;
  }

  // traceEnvmapLight (rayrenderer.cpp:1484-1519): Lambertian env NEE; the MIS
  // partner is the caller's bsdfPdf argument.
  C3 traceEnvmapLight(V3 hit, V3 n, float bsdfPdf, int v) const {
    V3 dir;
    float pdf = 0.0f;
    C3 Li;
    if (!sampleEnvmapForNEE(hit, n, v, dir, pdf, Li)) return C3();
    const float cosObj = dot(dir, n);
    float w = 1.0f;
    if (bsdfPdf > 0.0f) w = (pdf * pdf) / (pdf * pdf + bsdfPdf * bsdfPdf);
    return Li * (cosObj * w / ((float)M_PI * pdf));
  }

  // Miss radiance with the BSDF-side MIS weight (rayrenderer.cpp:1619-1630).
  C3 missRadiance(const Ray& ray, const Param* sp) const {
    C3 env = sampleEnvironment(ray.d);
    if (sp && sp->bsdfPdf > 0.0f) {
      const float envPdf = envmapDirectionPdf(ray.d);
      const float b2 = sp->bsdfPdf * sp->bsdfPdf, e2 = envPdf * envPdf;
      const float w = (b2 + e2 > 0.0f) ? b2 / (b2 + e2) : 1.0f;
      env = env * w;
    }
    return env;
  }

  // lambertTraceLights: rayrenderer.cpp:2319-2335
  C3 lambertTraceLights(V3 hit, V3 n, int v) const {
    C3 a, p;
    const int na = (int)s.areaLights.size();
    if (na > 0) a = traceAreaLight(s.areaLights[pickIndex(c.prng(v, S_LIGHT), na)], hit, n, v);
    for (const auto& pl : s.points) p += tracePointLight(pl, hit, n);
    return a + p + s.st.worldColor;
  }

  // calcAO: rayrenderer.cpp:2381-2409 (cosine directions from the LDS stream)
  float calcAO(V3 hit, V3 n, float dist, int v) const {
    float sum = 0.0f;
    const int N = s.st.spp;
    for (int i = 0; i < N; i++) {
      const int d0 = c.dimBase + 4 * v + 4 + 2 * i;
      const V3 dir = cosineWeightedDirection(n, c.lds(d0), c.lds(d0 + 1));
      const Ray r = ThicknessRay(hit, dir);
      if (!intersectAny(s, r, dist, P_AO)) sum += fmaxf(dot(dir, n), 0.0f);
    }
    return sum / (float)N;
  }

  bool chooseSelect(float u, float wa, float wb) const { return u * (wa + wb) < wa; }

  // ---- lobes (bsdf.cpp) -------------------------------------------------
  // DiffuseShader::shade: bsdf.cpp:54-108
  C3 diffuse(Param& p) {
    const Tri& tr = s.tris[p.info->tri];
    const Material& m = matOfTri(p.info->tri);
    const int v = p.vertex;
    const int d0 = c.ldsDirDim(v);
    const V3 dir = cosineWeightedDirection(p.vi.normal, c.lds(d0), c.lds(d0 + 1));
    const Ray ray = SurfaceRay(p.info->hit, dir, geomNormal(tr, p.vi.normal));
    C3 albedo(1, 1, 1);
    if (s.st.colorSampling) albedo = albedoOf(s, m, p.vi);
    const C3 savedT = p.throughput;
    const float savedPdf = p.bsdfPdf;
    p.throughput *= albedo;
    const float cosS = fmaxf(0.0f, dot(dir, p.vi.normal));
    p.bsdfPdf = cosS * (float)(1.0 / M_PI);
    C3 col = traceLight(p.info->hit, p.vi.normal, v);
    col += tracePath(ray, &p);
    // the MIS partner passed is this vertex's own cosine-sampled pdf (bsdf.cpp:86-88)
    col += traceEnvmapLight(p.info->hit, p.vi.normal, p.bsdfPdf, v);
    {  // volume-light NEE, no MIS (bsdf.cpp:91-101)
      V3 vDir; float vPdf = 0.0f; C3 vLe;
      if (sampleVolumeLightForNEE(p.info->hit, p.vi.normal, v, vDir, vPdf, vLe) && vPdf > 0.0f) {
        const float cosL = fmaxf(0.0f, dot(vDir, p.vi.normal));
        col += vLe * (cosL * (float)(1.0 / M_PI) / vPdf);
      }
    }
    p.throughput = savedT;
    p.bsdfPdf = savedPdf;
    return col * albedo;
  }

  // GlossyShader::shade: bsdf.cpp:173-374
  C3 glossy(Param& p) {
    const Tri& tr = s.tris[p.info->tri];
    const Material& m = matOfTri(p.info->tri);
    const int v = p.vertex;
    const V3 normal = p.vi.normal;
    const V3 inDir = p.inray.d;
    C3 albedo = m.color;
    if (s.st.colorSampling && m.texture >= 0) albedo = albedoOf(s, m, p.vi);
    const C3 F0 = (m.metallic >= 1.0f) ? albedo
        : (albedo * m.metallic + C3(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic));
    auto schlickF = [&](float VdotH) {
      const float a1 = fmaxf(0.0f, 1.0f - VdotH);
      const float a5 = a1 * a1 * a1 * a1 * a1;
      return F0 + (C3(1, 1, 1) - F0) * a5;
    };
    if (m.roughness < 1e-3f) {
      const V3 gN = geomNormal(tr, normal);
      V3 r = reflect(inDir, normal);
      if (dot(r, gN) <= 0.0f) r = reflect(inDir, gN);
      const float cosI = fmaxf(0.0f, -dot(inDir, normal));
      const C3 F = schlickF(cosI);
      const C3 savedT = p.throughput; const float savedPdf = p.bsdfPdf;
      p.throughput *= F; p.bsdfPdf = 0.0f;
      const C3 in = tracePath(SurfaceRay(p.info->hit, r, gN), &p);
      p.throughput = savedT; p.bsdfPdf = savedPdf;
      return in * F;
    }
    V3 t, b;
    buildTangentFrame(normal, t, b);
    if (fabsf(m.anisoRot) > 0.0f) {
      const float a = m.anisoRot * (float)(M_PI / 180.0);
      const float ca = cosf(a), sa = sinf(a);
      const V3 t2 = t * ca + b * sa, b2 = b * ca - t * sa;
      t = t2; b = b2;
    }
    const float aniso = fmaxf(-0.99f, fminf(0.99f, m.aniso));
    const float r2 = m.roughness * m.roughness;
    const float ax = fmaxf(1e-3f, r2 * (1.0f - aniso));
    const float ay = fmaxf(1e-3f, r2 * (1.0f + aniso));
    const V3 V = -inDir;
    const V3 Vl(dot(V, t), dot(V, b), dot(V, normal));
    if (Vl.z <= 0.0f) return C3();
    auto smithG1 = [&](V3 w) { return smithG1Aniso(w, ax, ay); };
    const float G1v = smithG1(Vl);
    auto evalGlossy = [&](V3 dw, C3& fCos, float& pdfB) {
      const V3 Ll(dot(dw, t), dot(dw, b), dot(dw, normal));
      if (Ll.z <= 0.0f) return false;
      V3 Hl = Vl + Ll;
      const float hl2 = Hl.x * Hl.x + Hl.y * Hl.y + Hl.z * Hl.z;
      if (hl2 <= 0.0f) return false;
      Hl = Hl * (1.0f / sqrtf(hl2));
      if (Hl.z <= 0.0f) return false;
      const float VdotH = fmaxf(0.0f, dot(Vl, Hl));
      if (VdotH <= 0.0f) return false;
      const float hx = Hl.x / ax, hy = Hl.y / ay;
      const float den = hx * hx + hy * hy + Hl.z * Hl.z;
      const float D = 1.0f / (kPi * ax * ay * den * den);
      const float G1l = smithG1(Ll);
      fCos = schlickF(VdotH) * (D * G1v * G1l / (4.0f * Vl.z));
      pdfB = G1v * D / (4.0f * Vl.z);
      return true;
    };
    C3 direct;
    {
      V3 lDir; float pl = 0.0f; C3 Le;
      if (sampleAreaLightForNEE(p.info->hit, normal, v, lDir, pl, Le)) {
        C3 fCos; float pb = 0.0f;
        if (evalGlossy(lDir, fCos, pb)) {
          const float w = pl * pl / (pl * pl + pb * pb);
          direct += Le * fCos * (w / pl);
        }
      }
    }
    {  // envmap NEE with MIS (bsdf.cpp:302-314)
      V3 eDir; float pe = 0.0f; C3 Li;
      if (sampleEnvmapForNEE(p.info->hit, normal, v, eDir, pe, Li)) {
        C3 fCos; float pb = 0.0f;
        if (evalGlossy(eDir, fCos, pb)) {
          const float w = pe * pe / (pe * pe + pb * pb);
          direct += Li * fCos * (w / pe);
        }
      }
    }
    {  // volume-light NEE, no MIS (bsdf.cpp:316-328)
      V3 vDir; float vPdf = 0.0f; C3 vLe;
      if (sampleVolumeLightForNEE(p.info->hit, normal, v, vDir, vPdf, vLe) && vPdf > 0.0f) {
        C3 fCos; float pb = 0.0f;
        if (evalGlossy(vDir, fCos, pb)) direct += vLe * fCos * (1.0f / vPdf);
      }
    }
    const float u1 = c.prng(v, S_VNDF0), u2 = c.prng(v, S_VNDF1);
    const V3 H = sampleGGXVNDF(Vl, ax, ay, u1, u2);
    const V3 Ll = H * (2.0f * dot(Vl, H)) - Vl;
    if (Ll.z <= 0.0f) return direct;
    const V3 L = t * Ll.x + b * Ll.y + normal * Ll.z;
    const V3 gN = geomNormal(tr, normal);
    if (dot(L, gN) <= 0.0f) return direct;
    const float VdotH = fmaxf(0.0f, dot(Vl, H));
    const C3 F = schlickF(VdotH);
    const C3 weight = F * smithG1(Ll);
    const float hx = H.x / ax, hy = H.y / ay;
    const float den = hx * hx + hy * hy + H.z * H.z;
    const float D = 1.0f / (kPi * ax * ay * den * den);
    const float pdfS = G1v * D / (4.0f * Vl.z);
    const C3 savedT = p.throughput; const float savedPdf = p.bsdfPdf;
    p.throughput *= weight; p.bsdfPdf = pdfS;
    const C3 in = tracePath(SurfaceRay(p.info->hit, L, gN), &p);
    p.throughput = savedT; p.bsdfPdf = savedPdf;
    return direct + in * weight;
  }

  // fresnelSchlick / refract: bsdf.cpp:32-52
  static float fresnelSchlick(float cosTheta, float ior) {
    float r0 = (1.0f - ior) / (1.0f + ior);
    r0 = r0 * r0;
    const float m = 1.0f - cosTheta;
    return r0 + (1.0f - r0) * (m * m) * (m * m) * m;
  }
  static V3 refract(V3 d, V3 n, float r) {
    const V3 nl = dot(d, n) < 0 ? n : -n;
    const bool into = dot(nl, n) > 0;
    if (into) r = 1.0f / r;
    const float c = dot(d, nl);
    const float t = 1.0f - r * r * (1.0f - c * c);
    if (t < 0) return reflect(d, n);
    return normalize(d * r - n * ((into ? 1.0f : -1.0f) * (c * r + sqrtf(t))));
  }

  // RefractionShader::shade: bsdf.cpp:376-483
  C3 refraction(Param& p) {
    const Tri& tr = s.tris[p.info->tri];
    const Material& m = matOfTri(p.info->tri);
    const int v = p.vertex;
    const V3 normal = p.vi.normal, inDir = p.inray.d;
    const float cosTheta = fabsf(dot(inDir, normal));
    float ior = m.ior;
    C3 chanMask(1, 1, 1);
    if (m.chroma > 0.0f) {
      bool first = false;
      if (p.chroma < 0) { p.chroma = (int)fminf(2.0f, floorf(c.prng(v, S_CHROMA) * 3.0f)); first = true; }
      const int ch = p.chroma;
      if (ch == 0) ior = m.ior * (1.0f - m.chroma);
      else if (ch == 2) ior = m.ior * (1.0f + m.chroma);
      if (first) chanMask = ch == 0 ? C3(3, 0, 0) : (ch == 1 ? C3(0, 3, 0) : C3(0, 0, 3));
    }
    const float F = fresnelSchlick(cosTheta, ior);
    const bool pickReflect = c.prng(v, S_FRESNEL) < F;
    V3 dir = pickReflect ? reflect(inDir, normal) : refract(inDir, normal, ior);
    if (m.roughness > 0.0f)
      dir = normalize(dir + randomRayInHemisphere(normal, c.prng(v, S_HEMI0), c.prng(v, S_HEMI1)) * m.roughness);
    const V3 gN = geomNormal(tr, normal);
    if (pickReflect && dot(dir, gN) <= 0.0f) dir = reflect(inDir, gN);
    const C3 savedT = p.throughput; const float savedPdf = p.bsdfPdf; const int savedMed = p.medium;
    p.throughput *= m.color;
    p.bsdfPdf = 0.0f;
    const float dIn = dot(inDir, normal), dOut = dot(dir, normal);
    if (dIn * dOut > 0.0f) {
      if (dIn < 0.0f) { const int im = s.objMedium[tr.obj]; if (im >= 0) p.medium = im; }
      else p.medium = s.globalMedium;
    }
    const C3 col = tracePath(SurfaceRay(p.info->hit, dir, gN), &p);
    p.throughput = savedT; p.bsdfPdf = savedPdf; p.medium = savedMed;
    return col * m.color * chanMask;
  }

  // TransparencyShader::shade: bsdf.cpp:513-546
  C3 transparency(Param& p) {
    const Tri& tr = s.tris[p.info->tri];
    const Material& m = matOfTri(p.info->tri);
    const C3 savedT = p.throughput; const int savedMed = p.medium;
    p.throughput *= C3(m.transparency, m.transparency, m.transparency);
    const float dIn = dot(p.inray.d, p.vi.normal);
    if (dIn < 0.0f) { const int im = s.objMedium[tr.obj]; if (im >= 0) p.medium = im; }
    else p.medium = s.globalMedium;
    const C3 col = tracePath(SurfaceRay(p.info->hit, p.inray.d, geomNormal(tr, p.vi.normal)), &p);
    p.throughput = savedT; p.medium = savedMed;
    return col * m.transparency;
  }

  // MixShader::shade: bsdf.cpp:579-610 (tree) or one-lobe selection (select)
  C3 mix(Param& p) {
    const Material& m = matOfTri(p.info->tri);
    const float wd = 1.0f - m.glossy - m.refraction;
    const float w[3] = {wd, m.glossy, m.refraction};
    const C3 savedT = p.throughput;
    C3 col;
    if (s.st.mixTree) {
      for (int i = 0; i < 3; i++) {
        if (!(w[i] > 0.00001f)) continue;
        p.throughput = savedT * w[i];
        const C3 r = i == 0 ? diffuse(p) : (i == 1 ? glossy(p) : refraction(p));
        col += r * w[i];
      }
    } else {
      float sum = 0.0f;
      for (int i = 0; i < 3; i++) if (w[i] > 0.00001f) sum += w[i];
      if (sum > 0.0f) {
        const float u = c.prng(p.vertex, S_LOBE) * sum;
        int pick = -1;
        float acc = 0.0f;
        for (int i = 0; i < 3; i++) {
          if (!(w[i] > 0.00001f)) continue;
          pick = i;
          acc += w[i];
          if (u < acc) break;
        }
        p.throughput = savedT * w[pick];
        const C3 r = pick == 0 ? diffuse(p) : (pick == 1 ? glossy(p) : refraction(p));
        col = r * sum;
      }
    }
    p.throughput = savedT;
    return col;
  }

  // RayBSDFShaderProvider::shade: rayrenderer.cpp:2776-2896
  C3 shade5(const HitInfo& info, const Ray& inray, const Vi& vi, const Param* sp, int medOverride = -2) {
    const Material& m = matOfTri(info.tri);
    Param p;
    p.info = &info; p.inray = inray; p.vi = vi;
    p.vertex = c.vertex++;
    p.medium = medOverride >= -1 ? medOverride : (sp ? sp->medium : s.globalMedium);
    if (m.emission > 0.0f) {
      const C3 e = m.color * m.emission;
      if (sp && sp->bsdfPdf > 0.0f) {
        const float cosLight = -dot(inray.d, vi.normal);
        if (cosLight <= 0.0f) return C3();
        const V3 dv = info.hit - inray.o;
        const float r2 = dot(dv, dv);
        const float pl = r2 / (cosLight * sampledArea(info.tri)) / lightCountFactor();
        const float pb = sp->bsdfPdf;
        return e * (pb * pb / (pb * pb + pl * pl));
      }
      return e;
    }
    if (dot(inray.d, vi.normal) > 0.0f) {
      if (m.transparency > 0.001f) {
        if (sp && sp->passes + 1 <= s.st.maxDepth) {
          p.passes = sp->passes + 1;
          p.throughput = sp->throughput;
          return transparency(p);
        }
        return C3();
      } else if (m.refraction < 0.001f && m.glossy > 0.001f) {
        return C3();
      }
    }
    if (sp) {
      if (sp->passes + 1 >= s.st.maxDepth) {
        if (1.0f - m.glossy - m.refraction > 0.00001f) {
          const C3 light = traceLight(info.hit, vi.normal, p.vertex);
          C3 col;
          if (s.st.colorSampling) col = albedoOf(s, m, vi);
          return light * col;
        }
        return C3();
      }
      p.passes = sp->passes + 1;
      p.throughput = sp->throughput;
      p.chroma = sp->chroma;
      p.bsdfPdf = sp->bsdfPdf;
      float rrWeight = 1.0f;
      if (p.passes >= s.st.rrDepth) {
        float q = maxc(p.throughput);
        q = fminf(RR_MAX_PROB, fmaxf(RR_MIN_PROB, q));
        if (c.prng(p.vertex, S_RR) >= q) return C3();
        rrWeight = 1.0f / q;
      }
      if (m.transparency > 0.001f) return transparency(p) * rrWeight;
      return mix(p) * rrWeight;
    }
    if (m.transparency > 0.01f) {
      if (s.st.mixTree) {
        Param p2 = p;
        const C3 a = mix(p) * (1.0f - m.transparency);
        return a + transparency(p2);
      }
      // select: transparency branch with probability t, mix with 1 - t
      if (c.prng(p.vertex, S_EYETR) < m.transparency) return transparency(p) * (1.0f / m.transparency);
      return mix(p);
    }
    return mix(p);
  }

  // Lambert providers: lambert.cpp:14-65 ; simple: rayrenderer.h:456-459 ; AO: :472-474
  C3 shadeSimple(const HitInfo& info, const Ray& inray, const Vi& vi, const Param* sp, int depth) {
    const Material& m = matOfTri(info.tri);
    const int shader = s.st.shader;
    const int v = c.vertex++;
    if (shader == 0) {
      const V3 L = normalize(V3(1, 1, 1));
      const float n = 0.1f + fmaxf(dot(L, vi.normal), 0.0f);
      return C3(n, n, n);
    }
    if (shader == 1) {
      const float a = fminf(fmaxf(calcAO(info.hit, vi.normal, RAY_MAX_DISTANCE, v), 0.0f), 1.0f);
      return C3(a, a, a);
    }
    if (m.emission > 0.0f) return m.color * m.emission;
    const C3 light = lambertTraceLights(info.hit, vi.normal, v) * 0.3f;
    auto through = [&]() -> C3 {
      if (depth + 1 >= s.st.maxDepth) return C3();
      return tracePathSimple(ThicknessRay(info.hit, inray.d), depth + 1);
    };
    if (shader == 2) {
      C3 col = light;
      if (s.st.colorSampling) col = col * albedoOf(s, m, vi);
      if (m.transparency > 0.0f)
        col = m.color * (light + C3(0.5f, 0.5f, 0.5f)) * (1.0f - m.transparency) + through() * m.transparency;
      return col;
    }
    // shader 3
    C3 col = light * 0.2f + light * 0.8f * calcAO(info.hit, vi.normal, 2.0f, v);
    if (s.st.colorSampling) col = col * albedoOf(s, m, vi);
    if (m.transparency > 0.0f) col += through() * m.transparency;
    (void)sp;
    return col;
  }

  C3 tracePathSimple(const Ray& ray, int depth) {
    HitInfo info;
    intersectClosest(s, ray, info);
    if (info.tri >= 0) return shadeSimple(info, ray, interp(s, info), nullptr, depth);
    return sampleEnvironment(ray.d);  // tracePath miss without BSDF parameters
  }

  // tracePath: rayrenderer.cpp:1596-1864.  `medOverride` >= -1 replaces the
  // segment's medium (the eye segment after a heat-haze bend).
  C3 tracePath(const Ray& ray, const Param* sp, int medOverride = -2) {
    HitInfo info;
    intersectClosest(s, ray, info);
    const int medId = medOverride >= -1 ? medOverride : (sp ? sp->medium : s.globalMedium);
    const Medium* med = medId >= 0 ? &s.media[medId] : nullptr;
    if (!med || !med->active()) {
      if (info.tri >= 0) return shade5(info, ray, interp(s, info), sp, medOverride);
      return missRadiance(ray, sp);
    }
    if (med->heatHaze()) {
      // rayrenderer.cpp:1645-1660: march to the next surface bending the ray,
      // then go on in the outer (global) medium with the same parameters.  A
      // heat-haze global medium bends once and the path goes on without a
      // medium (the reference recurses without end there).
      const float maxTh = info.tri >= 0 ? info.t : RAY_MAX_DISTANCE;
      const Ray bent = med->bendRay(ray, fminf(maxTh, 1000.0f));
      c.vertex++;  // every segment has its own key index
      int outer = s.globalMedium;
      if (outer >= 0 && s.media[outer].heatHaze()) outer = -1;
      if (!sp) return tracePath(bent, nullptr, outer);
      Param q = *sp;
      q.medium = outer;
      return tracePath(bent, &q);
    }
    const float maxT = info.tri >= 0 ? info.t : RAY_MAX_DISTANCE;
    const int v = c.vertex;  // the event index this segment ends in
    bool scattered;
    float tFlight, densAt = 1.0f;
    if (med->heterogeneous()) {  // delta tracking (rayrenderer.cpp:1672-1680)
      scattered = med->sampleDeltaTracking(ray, maxT, c, v, tFlight, densAt);
      if (!scattered) tFlight = maxT;
    } else {
      tFlight = med->sampleFreeFlight(c.prng(v, S_FLIGHT));
      scattered = tFlight < maxT;
    }
    const C3 medEm = med->emissionIntegral(ray, scattered ? tFlight : maxT, c, v);
    if (scattered) {
      c.vertex++;
      C3 sw;
      if (med->heterogeneous()) {  // sigma_s(p) / sigma_t_max (rayrenderer.cpp:1706-1709)
        const float inv = med->tMaxHero > 0.0f ? 1.0f / med->tMaxHero : 0.0f;
        sw = C3(med->sigma_s_eff.x * densAt * inv, med->sigma_s_eff.y * densAt * inv, med->sigma_s_eff.z * densAt * inv);
      } else {
        const float pHero = med->freeFlightPdf(tFlight);
        const C3 Tr = med->transmittance(tFlight);
        if (pHero > 0.0f) sw = C3(med->sigma_s_eff.x * Tr.x / pHero, med->sigma_s_eff.y * Tr.y / pHero,
                                 med->sigma_s_eff.z * Tr.z / pHero);
      }
      if (isZero(sw)) return medEm;
      const V3 pos = ray.o + ray.d * tFlight;
      const int passes = sp ? sp->passes + 1 : 1;
      if (passes > s.st.maxDepth) return medEm;
      C3 direct;
      const V3 proxy = -ray.d;
      V3 lDir; float pl = 0.0f; C3 Le;
      if (sampleAreaLightForNEE(pos, proxy, v, lDir, pl, Le) && pl > 0.0f)
        direct += Le * med->phasePdf(-ray.d, lDir) * (1.0f / pl);
      V3 eDir; float pe = 0.0f; C3 Li;
      if (sampleEnvmapForNEE(pos, proxy, v, eDir, pe, Li) && pe > 0.0f)
        direct += Li * med->phasePdf(-ray.d, eDir) * (1.0f / pe);
      V3 vDir; float vPdf = 0.0f; C3 vLe;
      if (sampleVolumeLightForNEE(pos, proxy, v, vDir, vPdf, vLe) && vPdf > 0.0f)
        direct += vLe * med->phasePdf(-ray.d, vDir) * (1.0f / vPdf);
      const V3 nd = med->samplePhase(ray.d, c.prng(v, S_PHASE0), c.prng(v, S_PHASE1));
      Param q;
      q.info = &info; q.inray = ray; q.passes = passes; q.medium = medId;
      if (sp) { q.throughput = sp->throughput; q.chroma = sp->chroma; }
      q.bsdfPdf = 0.0f;
      q.vertex = v;
      float rrW = 1.0f;
      if (passes >= s.st.rrDepth) {
        const C3 tt = q.throughput * sw;
        float qq = maxc(tt);
        qq = fminf(RR_MAX_PROB, fmaxf(RR_MIN_PROB, qq));
        if (c.prng(v, S_MEDRR) >= qq) return medEm + sw * direct;
        rrW = 1.0f / qq;
      }
      const C3 ind = tracePath(ThicknessRay(pos, nd), &q) * rrW;
      return medEm + sw * (direct + ind);
    }
    C3 surfW(1, 1, 1);
    if (!med->heterogeneous()) {  // delta tracking passes the surface with weight 1
      const float surv = med->survival(maxT);
      if (surv > 0.0f) {
        const C3 Tr = med->transmittance(maxT);
        surfW = C3(Tr.x / surv, Tr.y / surv, Tr.z / surv);
      }
    }
    if (info.tri >= 0) {
      Vi vi = interp(s, info);
      const V3 gpd = s.tris[info.tri].npd;
      const V3 geomN = dot(gpd, ray.d) <= 0.0f ? gpd : -gpd;
      if (dot(ray.d, vi.normal) > 0.0f && dot(ray.d, geomN) < 0.0f) vi.normal = geomN;
      return medEm + surfW * shade5(info, ray, vi, sp);
    }
    return medEm + surfW * missRadiance(ray, sp);
  }

  // traceEyeRay: rayrenderer.cpp:1254-1297 ; returns rgb of the color4
  C3 traceEyeRay(const Ray& ray) {
    HitInfo info;
    intersectClosest(s, ray, info);
    const C3 back(s.st.backColor[0], s.st.backColor[1], s.st.backColor[2]);
    const C3 env = info.tri >= 0 ? C3() : sampleEnvironment(ray.d);  // rayrenderer.cpp:1292-1296
    if (s.st.shader != 5) {
      if (info.tri >= 0) {
        const C3 r = shadeSimple(info, ray, interp(s, info), nullptr, 0);
        return C3(fmaxf(r.x, 0.0f), fmaxf(r.y, 0.0f), fmaxf(r.z, 0.0f));
      }
      return isZero(env) ? back : env;
    }
    const Medium* gm = s.globalMedium >= 0 ? &s.media[s.globalMedium] : nullptr;
    if (gm && gm->active()) {
      const C3 r = tracePath(ray, nullptr);
      if (info.tri >= 0 || !isZero(r)) return C3(fmaxf(r.x, 0.0f), fmaxf(r.y, 0.0f), fmaxf(r.z, 0.0f));
      return back;
    }
    if (info.tri >= 0) {
      const C3 r = shade5(info, ray, interp(s, info), nullptr);
      return C3(fmaxf(r.x, 0.0f), fmaxf(r.y, 0.0f), fmaxf(r.z, 0.0f));
    }
    return isZero(env) ? back : env;
  }
};

// ------------------------------------------------------------- driver ----
struct Image {
  int W, H;
  std::vector<double> sum, sumSq;  // 3 per pixel
  std::vector<int> n;
  std::vector<float> normal, albedo, albedoA, depth;
};

static void primaryRay(const Scene& s, Ctx& c, int x, int y, float dx, float dy, float vs, Ray& ray) {
  // accumulatePixelSamples ray generation: rayrenderer.cpp:855-934
  const float jx = c.lds(0), jy = c.lds(1);
  const bool aa = s.st.aa != 0;
  const float jxo = aa ? (jx - 0.5f) : 0.0f, jyo = aa ? (jy - 0.5f) : 0.0f;
  const float aperture = s.aperture > 0.0f ? 1.0f / s.aperture : 0.0f;
  if (s.dof >= 0.001f && aperture > 0.0f) {
    c.dimBase = 4;
    const float pxDx = dx + jxo * vs, pxDy = dy - jyo * vs;
    const V3 fp(pxDx * s.dof, pxDy * s.dof, -s.dof);
    const float du = c.lds(2), dv = c.lds(3);
    float ox, oy;
    if (s.blades >= 3) {
      const int N = s.blades;
      const float u0 = du * (float)N;
      const int wedge = (int)fminf((float)(N - 1), floorf(u0));
      float ss = u0 - (float)wedge, tt = dv;
      if (ss + tt > 1.0f) { ss = 1.0f - ss; tt = 1.0f - tt; }
      const float step = 2.0f * kPi / (float)N;
      const float rot = s.apertureRot * (float)(M_PI / 180.0);
      const float a0 = rot + step * (float)wedge, a1 = a0 + step;
      ox = (cosf(a0) * ss + cosf(a1) * tt) * aperture;
      oy = (sinf(a0) * ss + sinf(a1) * tt) * aperture;
    } else {
      const float a = 2.0f * du - 1.0f, b = 2.0f * dv - 1.0f;
      float r, phi;
      if (a == 0.0f && b == 0.0f) { r = 0.0f; phi = 0.0f; }
      else if (a * a > b * b) { r = a; phi = (float)(M_PI / 4.0) * (b / a); }
      else { r = b; phi = (float)(M_PI / 2.0) - (float)(M_PI / 4.0) * (a / b); }
      ox = r * cosf(phi) * aperture;
      oy = r * sinf(phi) * aperture;
    }
    ray.o = V3(ox, oy, 0.0f);
    ray.d = normalize(fp - ray.o);
  } else {
    c.dimBase = 2;
    ray.o = V3();
    ray.d = normalize(V3(dx + jxo * vs, dy - jyo * vs, -1.0f));
  }
  (void)x; (void)y;
}

static void renderPixelSamples(const Scene& s, Image& img, int x, int y, int s0, int count) {
  const float W = (float)s.st.W, H = (float)s.st.H;
  const float fovDeg = fminf(fmaxf(s.fov, 1.0f), 179.0f);
  const float vs = (2.0f * tanf(fovDeg * (float)(M_PI / 180.0) * 0.5f)) / H;
  const float dx = ((float)x + 0.5f - W * 0.5f) * vs;
  const float dy = -((float)y + 0.5f - H * 0.5f) * vs;
  const size_t pi = (size_t)y * s.st.W + x;
  Ctx c;
  double sr = 0, sg = 0, sb = 0, qr = 0, qg = 0, qb = 0;
  for (int i = s0; i < s0 + count; i++) {
    c.begin((uint32_t)x, (uint32_t)y, (uint32_t)s.st.W, (uint32_t)i, s.st.seed);
    Ray ray;
    primaryRay(s, c, x, y, dx, dy, vs, ray);
    Tracer t(s, c);
    C3 r = t.traceEyeRay(ray);
    if (s.st.clampMax > 0.0f)
      r = C3(fminf(r.x, s.st.clampMax), fminf(r.y, s.st.clampMax), fminf(r.z, s.st.clampMax));
    sr += r.x; sg += r.y; sb += r.z;
    qr += (double)r.x * r.x; qg += (double)r.y * r.y; qb += (double)r.z * r.z;
  }
  img.sum[pi * 3 + 0] += sr; img.sum[pi * 3 + 1] += sg; img.sum[pi * 3 + 2] += sb;
  img.sumSq[pi * 3 + 0] += qr; img.sumSq[pi * 3 + 1] += qg; img.sumSq[pi * 3 + 2] += qb;
  img.n[pi] += count;
}

// AOV guides (rayrenderer.cpp:819-844), from the pixel-centre primary ray.
static void writeAov(const Scene& s, Image& img, int x, int y) {
  const float W = (float)s.st.W, H = (float)s.st.H;
  const float fovDeg = fminf(fmaxf(s.fov, 1.0f), 179.0f);
  const float vs = (2.0f * tanf(fovDeg * (float)(M_PI / 180.0) * 0.5f)) / H;
  const float dx = ((float)x + 0.5f - W * 0.5f) * vs;
  const float dy = -((float)y + 0.5f - H * 0.5f) * vs;
  Ray ray{V3(), normalize(V3(dx, dy, -1.0f))};
  HitInfo info;
  intersectClosest(s, ray, info);
  const size_t pi = (size_t)y * s.st.W + x;
  if (info.tri >= 0) {
    const Vi vi = interp(s, info);
    const V3 nc = vi.normal * 0.5f + V3(0.5f, 0.5f, 0.5f);
    const Material& m = s.mats[s.objMat[s.tris[info.tri].obj]];
    float d = length(info.hit) / s.viewFar;
    d = sqrtf(d);
    d = 1.0f - fminf(fmaxf(d, 0.0f), 1.0f);
    img.normal[pi * 3 + 0] = nc.x; img.normal[pi * 3 + 1] = nc.y; img.normal[pi * 3 + 2] = nc.z;
    img.albedo[pi * 3 + 0] = m.color.x; img.albedo[pi * 3 + 1] = m.color.y; img.albedo[pi * 3 + 2] = m.color.z;
    img.albedoA[pi] = 1.0f;
    img.depth[pi] = d;
  } else {
    img.normal[pi * 3 + 0] = img.normal[pi * 3 + 1] = img.normal[pi * 3 + 2] = 0.5f;
    img.albedo[pi * 3 + 0] = s.st.backColor[0]; img.albedo[pi * 3 + 1] = s.st.backColor[1];
    img.albedo[pi * 3 + 2] = s.st.backColor[2];
    img.albedoA[pi] = s.st.backColor[3];
    img.depth[pi] = 0.0f;
  }
}

struct TileT { int x, y, w, h; };
// buildTileList: rayrenderer.cpp:717-746
static std::vector<TileT> buildTiles(int W, int H) {
  std::vector<TileT> t;
  for (int y = 0; y < H; y += 32)
    for (int x = 0; x < W; x += 32) t.push_back({x, y, std::min(32, W - x), std::min(32, H - y)});
  std::mt19937 rng(0xC0FFEEu);
  std::shuffle(t.begin(), t.end(), rng);
  return t;
}

template <class F>
static void parallelTiles(int threads, size_t n, F&& fn) {
  std::atomic<size_t> next(0);
  auto worker = [&]() {
    for (;;) {
      const size_t i = next.fetch_add(1);
      if (i >= n) return;
      fn(i);
    }
  };
  if (threads <= 1) { worker(); return; }
  std::vector<std::thread> th;
  for (int i = 0; i < threads; i++) th.emplace_back(worker);
  for (auto& t : th) t.join();
}

// computeTileNoise per pixel: rayrenderer.cpp:1038-1087
static float pixelRelSem(const Image& img, size_t pi, bool& counted) {
  const int n = img.n[pi];
  counted = true;
  if (n <= 1) return 1e9f;
  counted = false;
  const double invN = 1.0 / n;
  double m[3], q[3];
  for (int k = 0; k < 3; k++) { m[k] = img.sum[pi * 3 + k] * invN; q[k] = img.sumSq[pi * 3 + k] * invN; }
  const float maxMean = (float)std::max(m[0], std::max(m[1], m[2]));
  if (maxMean < 1e-3f) return 0.0f;
  counted = true;
  float worst = 0.0f;
  for (int k = 0; k < 3; k++) {
    const float var = fmaxf(0.0f, (float)(q[k] - m[k] * m[k]));
    const float sem = sqrtf(var * (float)invN);
    worst = fmaxf(worst, sem / fmaxf((float)m[k], 1e-3f));
  }
  return worst;
}

static void render(const Scene& s, Image& img) {
  const int W = s.st.W, H = s.st.H;
  img.W = W; img.H = H;
  img.sum.assign((size_t)W * H * 3, 0.0);
  img.sumSq.assign((size_t)W * H * 3, 0.0);
  img.n.assign((size_t)W * H, 0);
  img.normal.assign((size_t)W * H * 3, 0.0f);
  img.albedo.assign((size_t)W * H * 3, 0.0f);
  img.albedoA.assign((size_t)W * H, 0.0f);
  img.depth.assign((size_t)W * H, 0.0f);
  const auto tiles = buildTiles(W, H);
  const int threads = std::max(1, s.st.threads);
  const bool aov = s.st.denoise != 0;
  auto runTiles = [&](const std::vector<size_t>& list, int s0, int cnt, bool perPixelMask,
                      const std::vector<uint8_t>* mask) {
    parallelTiles(threads, list.size(), [&](size_t i) {
      const TileT& t = tiles[list[i]];
      for (int y = t.y; y < t.y + t.h; y++)
        for (int x = t.x; x < t.x + t.w; x++) {
          if (perPixelMask && !(*mask)[(size_t)y * W + x]) continue;
          if (s0 == 0 && aov) writeAov(s, img, x, y);
          renderPixelSamples(s, img, x, y, s0, cnt);
        }
    });
  };
  std::vector<size_t> all(tiles.size());
  for (size_t i = 0; i < all.size(); i++) all[i] = i;
  if (!s.st.adaptive) {
    runTiles(all, 0, s.st.spp, false, nullptr);
    return;
  }
  // renderAdaptive: rayrenderer.cpp:1162-1252 (tile mode) ; per-pixel mode
  const int target = std::max(1, s.st.spp);
  const int base = std::max(1, s.st.adaptiveBase);
  int spent = std::min(base, target);
  runTiles(all, 0, spent, false, nullptr);
  while (spent < target) {
    const int cnt = std::min(base, target - spent);
    if (s.st.adaptiveMode == RG_ADAPTIVE_TILE) {
      std::vector<size_t> active;
      for (size_t ti = 0; ti < tiles.size(); ti++) {
        const TileT& t = tiles[ti];
        double acc = 0.0;
        int cntPix = 0;
        for (int y = t.y; y < t.y + t.h; y++)
          for (int x = t.x; x < t.x + t.w; x++) {
            bool counted;
            const float r = pixelRelSem(img, (size_t)y * W + x, counted);
            if (counted) { acc += r; cntPix++; }
          }
        const float noise = cntPix ? (float)(acc / cntPix) : 0.0f;
        if (noise > s.st.adaptiveThreshold) active.push_back(ti);
      }
      if (active.empty()) break;
      runTiles(active, spent, cnt, false, nullptr);
    } else {
      std::vector<uint8_t> mask((size_t)W * H, 0);
      size_t nact = 0;
      for (size_t pi = 0; pi < (size_t)W * H; pi++) {
        bool counted;
        const float r = pixelRelSem(img, pi, counted);
        if (counted && r > s.st.adaptiveThreshold) { mask[pi] = 1; nact++; }
      }
      if (nact == 0) break;
      runTiles(all, spent, cnt, true, &mask);
    }
    spent += cnt;
  }
}

// atrousPass: rayrenderer.cpp:2536-2608
static void atrousPass(int w, int h, const float* src, float* dst, const float* normal, const float* depth,
                       int step, float sigC, float sigN, float sigD) {
  static const float k[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
  const float invC2 = 1.0f / (2.0f * sigC * sigC + 1e-8f);
  const float dScale = 1.0f / (sigD * (float)step + 1e-8f);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t ci = (size_t)y * w + x;
      const V3 cc(src[ci * 3], src[ci * 3 + 1], src[ci * 3 + 2]);
      const V3 cn(normal[ci * 3] * 2.0f - 1.0f, normal[ci * 3 + 1] * 2.0f - 1.0f, normal[ci * 3 + 2] * 2.0f - 1.0f);
      const float cd = depth[ci];
      const float cl = 0.2126f * cc.x + 0.7152f * cc.y + 0.0722f * cc.z;
      V3 sum; float ws = 0.0f;
      for (int ky = 0; ky < 5; ++ky) {
        const int ny = y + (ky - 2) * step;
        if (ny < 0 || ny >= h) continue;
        for (int kx = 0; kx < 5; ++kx) {
          const int nx = x + (kx - 2) * step;
          if (nx < 0 || nx >= w) continue;
          const size_t si = (size_t)ny * w + nx;
          const V3 sc(src[si * 3], src[si * 3 + 1], src[si * 3 + 2]);
          const V3 sn(normal[si * 3] * 2.0f - 1.0f, normal[si * 3 + 1] * 2.0f - 1.0f, normal[si * 3 + 2] * 2.0f - 1.0f);
          const float sl = 0.2126f * sc.x + 0.7152f * sc.y + 0.0722f * sc.z;
          const float ld = sl - cl;
          const float wc = expf(-(ld * ld) * invC2);
          float nd = sn.x * cn.x + sn.y * cn.y + sn.z * cn.z;
          if (nd < 0.0f) nd = 0.0f;
          const float wn = powf(nd, sigN);
          const float wd = expf(-fabsf(depth[si] - cd) * dScale);
          const float wgt = k[kx] * k[ky] * wc * wn * wd;
          sum = sum + sc * wgt;
          ws += wgt;
        }
      }
      const V3 f = ws > 1e-8f ? V3(sum.x / ws, sum.y / ws, sum.z / ws) : cc;
      dst[ci * 3] = f.x; dst[ci * 3 + 1] = f.y; dst[ci * 3 + 2] = f.z;
    }
}

// denoiseImage: rayrenderer.cpp:2649-2772
static void denoise(int w, int h, const float* noisy, const float* normal, const float* depth,
                    const float* albedo, const float* albedoA, int levels, float sigC, float sigN,
                    float sigD, float intensity, float* out) {
  const size_t n = (size_t)w * h;
  std::vector<float> A(n * 3), B(n * 3);
  auto lum = [](const float* c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; };
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const size_t ci = (size_t)y * w + x;
      float c[3] = {noisy[ci * 3], noisy[ci * 3 + 1], noisy[ci * 3 + 2]};
      float maxN = 0.0f;
      for (int dy = -1; dy <= 1; ++dy) {
        const int ny = y + dy;
        if (ny < 0 || ny >= h) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          if (dx == 0 && dy == 0) continue;
          const int nx = x + dx;
          if (nx < 0 || nx >= w) continue;
          const float l = lum(&noisy[((size_t)ny * w + nx) * 3]);
          if (l > maxN) maxN = l;
        }
      }
      const float cl = lum(c);
      const float cap = 1.5f * maxN + 0.01f;
      if (cl > cap) { const float sc = cap / cl; c[0] *= sc; c[1] *= sc; c[2] *= sc; }
      if (albedoA[ci] > 0.5f) {
        for (int k = 0; k < 3; k++) A[ci * 3 + k] = fminf(c[k] / fmaxf(albedo[ci * 3 + k], 0.3f), 3.0f);
      } else {
        for (int k = 0; k < 3; k++) A[ci * 3 + k] = c[k];
      }
    }
  float* src = A.data();
  float* dst = B.data();
  for (int l = 0; l < std::max(1, levels); ++l) {
    atrousPass(w, h, src, dst, normal, depth, 1 << l, sigC, sigN, sigD);
    std::swap(src, dst);
  }
  const float t = fminf(fmaxf(intensity, 0.0f), 1.0f), sN = 1.0f - t;
  for (size_t ci = 0; ci < n; ci++)
    for (int k = 0; k < 3; k++) {
      const float f = src[ci * 3 + k];
      const float r = albedoA[ci] > 0.5f ? f * albedo[ci * 3 + k] : f;
      out[ci * 3 + k] = noisy[ci * 3 + k] * sN + r * t;
    }
}

// applyPostProcess (rayrenderer.cpp:598-696): energy-based HDR bloom on an
// RGBA image in place.  Extract the luminance above the threshold (with the
// knee curve), area-average it into a glow buffer of size_aspect x the image
// (downsampleArea, :386-413), blur it twice with a Gaussian of sigma / sqrt 2
// where sigma = radius x W x size_aspect (separableGaussianBlur, :423-475),
// upsample bilinearly (texel centres aligned, edges clamped: the reference's
// Image::resize lives in the graphics-module submodule, not in its tree) and
// add strength x glow.
static void bloom(int W, int H, float* hdr, float threshold, float strength, float radius, float sizeAspect,
                  float curve) {
  if (W <= 0 || H <= 0) return;
  threshold = fmaxf(threshold, 0.0f);
  curve = fmaxf(curve, 1e-3f);
  const float aspect = fmaxf(0.02f, sizeAspect);
  const int gw = std::max(1, (int)((float)W * aspect));
  const int gh = std::max(1, (int)((float)H * aspect));
  std::vector<float> glow((size_t)gw * gh * 3, 0.0f), tmp(glow.size());
  for (int y = 0; y < gh; ++y) {
    const int y0 = (int)((int64_t)y * H / gh);
    const int y1 = std::max(y0 + 1, (int)((int64_t)(y + 1) * H / gh));
    for (int x = 0; x < gw; ++x) {
      const int x0 = (int)((int64_t)x * W / gw);
      const int x1 = std::max(x0 + 1, (int)((int64_t)(x + 1) * W / gw));
      float ar = 0.0f, ag = 0.0f, ab = 0.0f;
      int count = 0;
      for (int sy = y0; sy < y1 && sy < H; ++sy)
        for (int sx = x0; sx < x1 && sx < W; ++sx) {
          const float* c = &hdr[((size_t)sy * W + sx) * 4];
          const float L = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
          float gr = 0.0f, gg = 0.0f, gb = 0.0f;
          if (L > threshold && L > 1e-6f) {
            float scale = (L - threshold) / L;
            if (curve != 1.0f) scale = powf(scale, curve);
            gr = c[0] * scale; gg = c[1] * scale; gb = c[2] * scale;
          }
          ar += gr; ag += gg; ab += gb;
          count++;
        }
      if (count > 0) {
        const float inv = 1.0f / (float)count;
        float* o = &glow[((size_t)y * gw + x) * 3];
        o[0] = ar * inv; o[1] = ag * inv; o[2] = ab * inv;
      }
    }
  }
  const float sigmaDown = fmaxf(0.0f, radius) * (float)W * aspect;
  if (sigmaDown >= 0.5f) {
    const float sigma = sigmaDown * 0.70710678f;
    if (sigma >= 0.25f) {
      const int r = std::max(1, (int)ceilf(sigma * 3.0f));
      std::vector<float> k(2 * r + 1);
      float sum = 0.0f;
      const float twoSigmaSq = 2.0f * sigma * sigma;
      for (int i = 0; i < 2 * r + 1; ++i) {
        const float x = (float)(i - r);
        k[i] = expf(-(x * x) / twoSigmaSq);
        sum += k[i];
      }
      const float invSum = 1.0f / sum;
      for (float& w : k) w *= invSum;
      auto pass = [&](const std::vector<float>& src, std::vector<float>& dst, bool vertical) {
        for (int y = 0; y < gh; ++y)
          for (int x = 0; x < gw; ++x) {
            float a[3] = {0.0f, 0.0f, 0.0f};
            for (int t = -r; t <= r; ++t) {
              int sx = x, sy = y;
              if (vertical) sy = std::min(std::max(y + t, 0), gh - 1);
              else sx = std::min(std::max(x + t, 0), gw - 1);
              const float* c = &src[((size_t)sy * gw + sx) * 3];
              for (int ch = 0; ch < 3; ch++) a[ch] += c[ch] * k[t + r];
            }
            float* o = &dst[((size_t)y * gw + x) * 3];
            o[0] = a[0]; o[1] = a[1]; o[2] = a[2];
          }
      };
      for (int twice = 0; twice < 2; ++twice) {
        pass(glow, tmp, false);
        pass(tmp, glow, true);
      }
    }
  }
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      float sx = ((float)x + 0.5f) * (float)gw / (float)W - 0.5f;
      float sy = ((float)y + 0.5f) * (float)gh / (float)H - 0.5f;
      sx = fminf(fmaxf(sx, 0.0f), (float)(gw - 1));
      sy = fminf(fmaxf(sy, 0.0f), (float)(gh - 1));
      const int x0 = (int)sx, y0 = (int)sy;
      const int x1 = std::min(x0 + 1, gw - 1), y1 = std::min(y0 + 1, gh - 1);
      const float fx = sx - (float)x0, fy = sy - (float)y0;
      float* a = &hdr[((size_t)y * W + x) * 4];
      for (int ch = 0; ch < 3; ch++) {
        auto at = [&](int xx, int yy) { return glow[((size_t)yy * gw + xx) * 3 + ch]; };
        auto lerp = [](float p, float q, float t) { return p + (q - p) * t; };
        const float g = lerp(lerp(at(x0, y0), at(x1, y0), fx), lerp(at(x0, y1), at(x1, y1), fx), fy);
        a[ch] = a[ch] + g * strength;
      }
    }
}

// applyTonemapGamma: rayrenderer.cpp:2610-2647
static void tonemap(int w, int h, const float* src, float* dst) {
  const float invGamma = 1.0f / 2.2f;
  for (size_t i = 0; i < (size_t)w * h; i++) {
    const float* c = &src[i * 4];
    const float L = 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2];
    float mr = 0, mg = 0, mb = 0;
    if (L > 1e-6f) {
      const float sc = (L / (L + 1.0f)) / L;
      mr = c[0] * sc; mg = c[1] * sc; mb = c[2] * sc;
      const float peak = fmaxf(fmaxf(mr, mg), mb);
      if (peak > 1.0f) { const float inv = 1.0f / peak; mr *= inv; mg *= inv; mb *= inv; }
    }
    float o[4] = {powf(fmaxf(mr, 0.0f), invGamma), powf(fmaxf(mg, 0.0f), invGamma),
                  powf(fmaxf(mb, 0.0f), invGamma), c[3]};
    for (int k = 0; k < 3; k++) if (o[k] > 1.0f) o[k] = 1.0f;
    memcpy(&dst[i * 4], o, sizeof(o));
  }
}

// Camera view transform, Renderer::applyCameraTransform (renderer.cpp:24-28):
// rotate by -angle, then translate by -location.  Row-vector convention
// p_view = [p 1] * M, whose 3x3 block is R = Ry(ay) Rx(ax) Rz(az) (degrees,
// active right-handed rotations) and whose last row is -(location * R); that
// is, p_view = R^T (p - location).  The order of the three axis rotations
// lives in the graphics-module submodule, which the reference tree does not
// vendor; single-axis angles (the sample scenes') do not depend on it.  The
// products run in a fixed order without contraction (this file is built with
// -ffp-contract=off), so view-space vertices are bit-identical to the
// device's, and angle 0 reduces to p - location exactly.
struct ViewM {
  float m[16];
};

static ViewM cameraView(const rg_camera& c) {
  const float d2r = 3.14159265358979323846f / 180.0f;
  const float ax = c.angle[0] * d2r, ay = c.angle[1] * d2r, az = c.angle[2] * d2r;
  const double cx = std::cos(ax), sx = std::sin(ax), cy = std::cos(ay), sy = std::sin(ay), cz = std::cos(az),
               sz = std::sin(az);
  const double Rx[3][3] = {{1, 0, 0}, {0, cx, -sx}, {0, sx, cx}};
  const double Ry[3][3] = {{cy, 0, sy}, {0, 1, 0}, {-sy, 0, cy}};
  const double Rz[3][3] = {{cz, -sz, 0}, {sz, cz, 0}, {0, 0, 1}};
  double T[3][3], R[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      T[i][j] = 0;
      for (int k = 0; k < 3; k++) T[i][j] += Ry[i][k] * Rx[k][j];
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      R[i][j] = 0;
      for (int k = 0; k < 3; k++) R[i][j] += T[i][k] * Rz[k][j];
    }
  ViewM M;
  memset(M.m, 0, sizeof(M.m));
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) M.m[i * 4 + j] = (float)R[i][j];
  for (int j = 0; j < 3; j++) {
    const float t = c.location[0] * M.m[j] + c.location[1] * M.m[4 + j] + c.location[2] * M.m[8 + j];
    M.m[12 + j] = -t;
  }
  M.m[15] = 1.0f;
  return M;
}

static V3 viewPoint(const ViewM& M, const float* p) {
  float o[3];
  for (int j = 0; j < 3; j++) o[j] = ((p[0] * M.m[j] + p[1] * M.m[4 + j]) + p[2] * M.m[8 + j]) + M.m[12 + j];
  return V3(o[0], o[1], o[2]);
}

// Directions by the rotation block, renormalised (R is orthonormal, so it is
// its own inverse transpose).
static V3 viewDir(const ViewM& M, const float* p) {
  float o[3];
  for (int j = 0; j < 3; j++) o[j] = (p[0] * M.m[j] + p[1] * M.m[4 + j]) + p[2] * M.m[8 + j];
  const float l = sqrtf((o[0] * o[0] + o[1] * o[1]) + o[2] * o[2]);
  return l > 0.0f ? V3(o[0] / l, o[1] / l, o[2] / l) : V3(o[0], o[1], o[2]);
}

// Scene::buildEnvmapCDF, equirectangular part (scene.cpp:414-463): per-row
// running sums of luminance x sin(theta) over raw texels (no sRGB decode),
// each row normalised to a conditional CDF, a marginal CDF over the row sums,
// sequential float sums in file order.
static void buildEnvmapCDF(Scene& s) {
  const Texture& T = s.textures[s.envTex];
  const int W = T.w, H = T.h;
  if (W <= 0 || H <= 0) return;
  s.envW = W;
  s.envH = H;
  std::vector<float> rowWeight(H, 0.0f);
  s.envCond.assign((size_t)H * (W + 1), 0.0f);
  for (int y = 0; y < H; y++) {
    const float v = (y + 0.5f) / (float)H;
    const float sinTheta = sinf((float)M_PI * v);
    float rowSum = 0.0f;
    for (int x = 0; x < W; x++) {
      const float* c = &T.rgba[((size_t)y * W + x) * 4];
      const float lum = fmaxf(0.0f, 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]);
      rowSum += lum * sinTheta;
      s.envCond[(size_t)y * (W + 1) + (x + 1)] = rowSum;
    }
    rowWeight[y] = rowSum;
  }
  for (int y = 0; y < H; y++) {
    if (rowWeight[y] > 0.0f) {
      const float inv = 1.0f / rowWeight[y];
      for (int x = 1; x <= W; x++) s.envCond[(size_t)y * (W + 1) + x] *= inv;
    }
  }
  s.envMarg.assign(H + 1, 0.0f);
  for (int y = 0; y < H; y++) s.envMarg[y + 1] = s.envMarg[y] + rowWeight[y];
  s.envTotal = s.envMarg[H];
  if (s.envTotal > 0.0f) {
    const float inv = 1.0f / s.envTotal;
    for (int y = 0; y <= H; y++) s.envMarg[y] *= inv;
  }
}

// Scene::buildEnvmapCDF, cubemap part (scene.cpp:343-410): per face, running
// row sums of luminance x the texel's solid-angle Jacobian 1/(s^2+t^2+1)^1.5,
// rows normalised to conditional CDFs, a per-face marginal over rows and a CDF
// over the face totals; raw texels, sequential float sums.
static void buildCubeCDF(Scene& s) {
  const int W = s.textures[s.envFace[0]].w, H = s.textures[s.envFace[0]].h;
  if (W <= 0 || H <= 0) return;
  s.envCubeW = W;
  s.cubeMargFace.assign(7, 0.0f);
  s.cubeMargY.assign((size_t)6 * (H + 1), 0.0f);
  s.cubeCond.assign((size_t)6 * H * (W + 1), 0.0f);
  float faceWeights[6] = {0, 0, 0, 0, 0, 0};
  for (int f = 0; f < 6; f++) {
    const Texture& T = s.textures[s.envFace[f]];
    std::vector<float> rowWeight(H, 0.0f);
    for (int y = 0; y < H; y++) {
      float* cond = &s.cubeCond[((size_t)f * H + y) * (W + 1)];
      cond[0] = 0.0f;
      float rowSum = 0.0f;
      const float t = 1.0f - (y + 0.5f) * (2.0f / (float)H);
      for (int x = 0; x < W; x++) {
        const float sx = (x + 0.5f) * (2.0f / (float)W) - 1.0f;
        const float denom = sx * sx + t * t + 1.0f;
        const float jac = 1.0f / (denom * sqrtf(denom));
        const float* c = &T.rgba[((size_t)y * W + x) * 4];
        const float lum = fmaxf(0.0f, 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]);
        rowSum += lum * jac;
        cond[x + 1] = rowSum;
      }
      if (rowSum > 0.0f) {
        const float inv = 1.0f / rowSum;
        for (int x = 1; x <= W; x++) cond[x] *= inv;
      }
      rowWeight[y] = rowSum;
    }
    float* my = &s.cubeMargY[(size_t)f * (H + 1)];
    my[0] = 0.0f;
    for (int y = 0; y < H; y++) my[y + 1] = my[y] + rowWeight[y];
    const float faceTotal = my[H];
    faceWeights[f] = faceTotal;
    if (faceTotal > 0.0f) {
      const float inv = 1.0f / faceTotal;
      for (int y = 0; y <= H; y++) my[y] *= inv;
    }
  }
  float total = 0.0f;
  for (int f = 0; f < 6; f++) total += faceWeights[f];
  s.envCubeTotal = total;
  if (total > 0.0f) {
    const float inv = 1.0f / total;
    float acc = 0.0f;
    s.cubeMargFace[0] = 0.0f;
    for (int f = 0; f < 6; f++) {
      acc += faceWeights[f];
      s.cubeMargFace[f + 1] = acc * inv;
    }
  }
}

static Scene* buildScene(const rg_scene_desc* d, int bins) {
  Scene* s = new Scene();
  const int nt = d->num_triangles;
  const ViewM view = cameraView(d->camera);
  s->camLoc = V3(d->camera.location[0], d->camera.location[1], d->camera.location[2]);
  s->fov = d->camera.field_of_view;
  s->viewNear = d->camera.view_near;
  s->viewFar = d->camera.view_far;
  s->dof = d->camera.depth_of_field;
  s->aperture = d->camera.aperture;
  s->blades = d->camera.aperture_blades;
  s->apertureRot = d->camera.aperture_rotation;
  s->exposure = d->camera.exposure;
  s->mats.resize(d->num_materials);
  for (int i = 0; i < d->num_materials; i++) {
    const rg_material& m = d->materials[i];
    Material& o = s->mats[i];
    o.color = C3(m.color[0], m.color[1], m.color[2]);
    o.glossy = m.glossy; o.roughness = m.roughness; o.transparency = m.transparency;
    o.refraction = m.refraction; o.ior = m.refraction_ratio; o.chroma = m.chroma_dispersion;
    o.metallic = m.metallic; o.aniso = m.anisotropy; o.anisoRot = m.aniso_rotation;
    o.emission = m.emission; o.spotRange = m.spot_range; o.texture = m.texture;
    o.tiling[0] = m.tex_tiling[0]; o.tiling[1] = m.tex_tiling[1];
  }
  // media: prepare() + bake() (medium.cpp:18-101); only the cone (cone mode)
  // and the path points (path mode) are baked into camera space
  auto cap = [](int n) { return n > 64 ? 64 : n; };
  s->media.resize(d->num_media);
  for (int i = 0; i < d->num_media; i++) {
    const rg_medium& m = d->media[i];
    Medium& o = s->media[i];
    const float dn = fmaxf(0.0f, m.density);
    o.sigma_s_eff = C3(m.sigma_s[0], m.sigma_s[1], m.sigma_s[2]) * dn;
    o.sigma_e_eff = C3(m.sigma_e[0], m.sigma_e[1], m.sigma_e[2]) * dn;
    const C3 sa = C3(m.sigma_a[0], m.sigma_a[1], m.sigma_a[2]) * dn;
    o.sigma_t = sa + o.sigma_s_eff;
    o.hero = (o.sigma_t.x + o.sigma_t.y + o.sigma_t.z) * (1.0f / 3.0f);
    o.g = m.g;
    o.density = m.density;
    o.mode = (m.emission_mode == 1 || m.emission_mode == 2) ? m.emission_mode : 0;
    o.field = m.density_field == 1 ? 1 : 0;
    o.tMaxHero = o.field ? o.hero * fmaxf(0.0f, m.noise_amplitude * 1.0f + m.noise_bias) : o.hero;
    const float al2 = m.cone_axis[0] * m.cone_axis[0] + m.cone_axis[1] * m.cone_axis[1] + m.cone_axis[2] * m.cone_axis[2];
    V3 axN(0.0f, 0.0f, -1.0f);
    if (al2 > 1e-12f) {
      const float inv = 1.0f / sqrtf(al2);
      axN = V3(m.cone_axis[0] * inv, m.cone_axis[1] * inv, m.cone_axis[2] * inv);
    }
    o.coneOriginR = V3(m.cone_origin[0], m.cone_origin[1], m.cone_origin[2]);
    o.coneAxisR = axN;
    if (o.mode == 1) {
      o.coneOriginR = viewPoint(view, m.cone_origin);
      float av[3];
      for (int j = 0; j < 3; j++) av[j] = (axN.x * view.m[j] + axN.y * view.m[4 + j]) + axN.z * view.m[8 + j];
      const float vl2 = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
      if (vl2 > 1e-12f) {
        const float inv = 1.0f / sqrtf(vl2);
        o.coneAxisR = V3(av[0] * inv, av[1] * inv, av[2] * inv);
      }
    }
    o.coneLength = m.cone_length; o.coneRadius = m.cone_radius;
    o.coneInner = C3(m.cone_inner[0], m.cone_inner[1], m.cone_inner[2]);
    o.coneOuter = C3(m.cone_outer[0], m.cone_outer[1], m.cone_outer[2]);
    o.coneIntensity = m.cone_intensity; o.conePeakAxial = m.cone_peak_axial;
    o.conePeakSharpness = m.cone_peak_sharpness; o.coneSamples = cap(m.cone_emission_samples);
    o.pathCount = m.num_path_points > 0 ? m.num_path_points : 0;
    if (o.mode == 2)
      for (int k = 0; k < o.pathCount; k++) {
        const rg_medium_path_point& q = m.path_points[k];
        o.pathPointsR.push_back(PathPt{viewPoint(view, q.p), q.radius, q.t});
      }
    o.pathInner = C3(m.path_inner[0], m.path_inner[1], m.path_inner[2]);
    o.pathOuter = C3(m.path_outer[0], m.path_outer[1], m.path_outer[2]);
    o.pathIntensity = m.path_intensity; o.pathFalloffPower = m.path_falloff_power;
    o.pathSamples = cap(m.path_emission_samples);
    o.noiseFrequency = m.noise_frequency; o.noiseOctaves = cap(m.noise_octaves); o.noiseGain = m.noise_gain;
    o.noiseLacunarity = m.noise_lacunarity; o.noiseAmplitude = m.noise_amplitude; o.noiseBias = m.noise_bias;
    o.noiseOffset = V3(m.noise_offset[0], m.noise_offset[1], m.noise_offset[2]);
    o.hazeOn = m.heat_haze != 0;
    o.iorAmplitude = m.ior_amplitude; o.iorFrequency = m.ior_frequency; o.iorOctaves = cap(m.ior_octaves);
    o.iorGain = m.ior_gain; o.iorLacunarity = m.ior_lacunarity; o.iorMarchSteps = cap(m.ior_march_steps);
    o.iorOffset = V3(m.ior_offset[0], m.ior_offset[1], m.ior_offset[2]);
    o.iorFalloff = m.ior_falloff;
  }
  // inactive media are dropped by readMedium (sceneloader.cpp:325-333)
  auto live = [&](int m) { return m >= 0 && m < d->num_media && s->media[m].active() ? m : -1; };
  s->globalMedium = live(d->global_medium);
  s->objMat.resize(d->num_objects);
  s->objMedium.resize(d->num_objects);
  for (int i = 0; i < d->num_objects; i++) {
    s->objMat[i] = d->objects[i].material;
    s->objMedium[i] = live(d->objects[i].interior_medium);
    // emissive-volume registration (rayrenderer.cpp:180-206)
    const int mi = s->objMedium[i];
    if (mi >= 0) {
      const Medium& M = s->media[mi];
      if ((M.mode == 1 && M.coneIntensity > 0.0f) || (M.mode == 0 && !Medium::isZero3(M.sigma_e_eff)))
        s->vols.push_back(VolLight{mi, viewPoint(view, d->objects[i].location)});
    }
  }
  s->meshObj.assign(d->mesh_object, d->mesh_object + d->num_meshes);
  s->meshTris.assign(d->num_meshes, {});
  s->objMeshes.assign(d->num_objects, {});
  for (int i = 0; i < d->num_meshes; i++) s->objMeshes[s->meshObj[i]].push_back(i);
  s->tris.resize(nt);
  for (int i = 0; i < nt; i++) {
    Tri& t = s->tris[i];
    const float* p = &d->positions[(size_t)i * 9];
    const float* n = &d->normals[(size_t)i * 9];
    t.v1 = viewPoint(view, p); t.v2 = viewPoint(view, p + 3); t.v3 = viewPoint(view, p + 6);
    t.n1 = viewDir(view, n); t.n2 = viewDir(view, n + 3); t.n3 = viewDir(view, n + 6);
    for (int k = 0; k < 6; k++) t.uv[k] = d->uvs ? d->uvs[(size_t)i * 6 + k] : 0.0f;
    // precalc: raycommon.cpp:128-149
    const V3 pd = cross(t.v2 - t.v1, t.v3 - t.v2);
    t.tia = 1.0f / length(cross(t.v1 - t.v2, t.v1 - t.v3));
    t.npd = normalize(pd);
    t.area = 0.5f * length(cross(t.v2 - t.v1, t.v3 - t.v1));
    t.bmin = V3(fminf(t.v1.x, fminf(t.v2.x, t.v3.x)), fminf(t.v1.y, fminf(t.v2.y, t.v3.y)), fminf(t.v1.z, fminf(t.v2.z, t.v3.z)));
    t.bmax = V3(fmaxf(t.v1.x, fmaxf(t.v2.x, t.v3.x)), fmaxf(t.v1.y, fmaxf(t.v2.y, t.v3.y)), fmaxf(t.v1.z, fmaxf(t.v2.z, t.v3.z)));
    t.mesh = d->tri_mesh[i];
    t.obj = s->meshObj[t.mesh];
    s->meshTris[t.mesh].push_back(i);
  }
  // light registration: rayrenderer.cpp:333-353
  for (int i = 0; i < d->num_objects; i++) {
    const Material& m = s->mats[s->objMat[i]];
    if (m.emission > 0.0f && !s->objMeshes[i].empty()) s->areaLights.push_back(i);
  }
  for (int i = 0; i < d->num_point_lights; i++) {
    const rg_point_light& pl = d->point_lights[i];
    PointLight o;
    o.pos = viewPoint(view, pl.position);
    o.normal = viewDir(view, pl.normal);
    o.mat = pl.material;
    s->points.push_back(o);
  }
  for (int i = 0; i < d->num_textures; i++) {
    Texture T;
    T.w = d->textures[i].width; T.h = d->textures[i].height; T.hdr = d->textures[i].is_hdr;
    T.rgba.assign(d->textures[i].rgba, d->textures[i].rgba + (size_t)T.w * T.h * 4);
    s->textures.push_back(std::move(T));
  }
  const bool eq = d->has_envmap && d->envmap_texture >= 0 && d->envmap_texture < d->num_textures;
  bool cube = d->envmap_cube != 0;
  for (int f = 0; cube && f < 6; f++) cube = d->envmap_cube_faces[f] >= 0 && d->envmap_cube_faces[f] < d->num_textures;
  if (eq || cube) {
    s->envIntensity = d->envmap_intensity;
    const float yaw = d->envmap_rotation * (float)(M_PI / 180.0);
    s->envCosY = cosf(yaw);
    s->envSinY = sinf(yaw);
  }
  if (eq) {
    s->envTex = d->envmap_texture;
    buildEnvmapCDF(*s);
  }
  if (cube) {
    s->envCube = true;
    for (int f = 0; f < 6; f++) s->envFace[f] = d->envmap_cube_faces[f];
    buildCubeCDF(*s);
  }
  buildBVH(*s, bins);
  return s;
}

}  // namespace orc

// ------------------------------------------------------------------ C API ----
using namespace orc;

struct orc_settings {
  int32_t width, height, spp, shader, antialias, color_sampling, denoise, denoise_levels;
  float sigma_color, sigma_normal, sigma_depth, denoise_intensity, firefly_clamp;
  int32_t adaptive, adaptive_base, adaptive_mode;
  float adaptive_threshold;
  float world_color[3];
  float back_color[4];
  uint32_t seed;
  int32_t max_depth, rr_depth, light_pick_fix, threads, mix_tree;
};

extern "C" {

void* orc_scene_create(const rg_scene_desc* d, int32_t bins) { return buildScene(d, bins > 1 ? bins : 16); }
void orc_scene_destroy(void* s) { delete (Scene*)s; }
int32_t orc_bvh_nodes(void* s) { return (int32_t)((Scene*)s)->nodes.size(); }

// Ray-batch closest hit: out_tuv n*3, out_prim n (DFS triangle id or -1).
void orc_closest(void* sp, const float* rays, int32_t n, float* out_tuv, int32_t* out_prim) {
  const Scene& s = *(Scene*)sp;
  for (int i = 0; i < n; i++) {
    const Ray r{V3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]), V3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5])};
    HitInfo h;
    intersectClosest(s, r, h);
    out_prim[i] = h.tri;
    out_tuv[i * 3] = h.t; out_tuv[i * 3 + 1] = h.u; out_tuv[i * 3 + 2] = h.v;
  }
}
// Brute-force closest hit over every triangle in DFS order (tie-break check).
void orc_closest_brute(void* sp, const float* rays, int32_t n, float* out_tuv, int32_t* out_prim) {
  const Scene& s = *(Scene*)sp;
  for (int i = 0; i < n; i++) {
    const Ray r{V3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]), V3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5])};
    HitInfo h;
    for (size_t k = 0; k < s.tris.size(); k++) intersectClosestTri(s.tris[k], (int)k, r, h);
    out_prim[i] = h.tri;
    out_tuv[i * 3] = h.t; out_tuv[i * 3 + 1] = h.u; out_tuv[i * 3 + 2] = h.v;
  }
}
void orc_any(void* sp, const float* rays, const float* tmax, int32_t n, int32_t pred, uint8_t* out) {
  const Scene& s = *(Scene*)sp;
  for (int i = 0; i < n; i++) {
    const Ray r{V3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]), V3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5])};
    out[i] = intersectAny(s, r, tmax[i], pred) ? 1 : 0;
  }
}

// Full render. Outputs (any may be NULL): sum/sumsq W*H*3 doubles, counts W*H,
// hdr W*H*4 floats (mean*exposure, clamped >= 0, denoised if enabled), ldr W*H*4.
int32_t orc_render(void* sp, const orc_settings* st, double* out_sum, double* out_sumsq, int32_t* out_n,
                   float* out_hdr, float* out_ldr, float* out_normal, float* out_albedo, float* out_depth) {
  Scene& s = *(Scene*)sp;
  Settings& S = s.st;
  S.W = st->width; S.H = st->height; S.spp = st->spp; S.shader = st->shader; S.aa = st->antialias;
  S.colorSampling = st->color_sampling; S.denoise = st->denoise; S.levels = st->denoise_levels;
  S.sigC = st->sigma_color; S.sigN = st->sigma_normal; S.sigD = st->sigma_depth;
  S.intensity = st->denoise_intensity; S.clampMax = st->firefly_clamp;
  S.adaptive = st->adaptive; S.adaptiveBase = st->adaptive_base; S.adaptiveMode = st->adaptive_mode;
  S.adaptiveThreshold = st->adaptive_threshold;
  S.worldColor = C3(st->world_color[0], st->world_color[1], st->world_color[2]);
  for (int k = 0; k < 4; k++) S.backColor[k] = st->back_color[k];
  S.seed = st->seed; S.maxDepth = st->max_depth; S.rrDepth = st->rr_depth;
  S.lightFix = st->light_pick_fix; S.threads = st->threads; S.mixTree = st->mix_tree;
  if (S.shader == 4 || S.shader < 0 || S.shader > 5) return RG_ERR_UNSUPPORTED;
  Image img;
  render(s, img);
  const size_t np = (size_t)S.W * S.H;
  if (out_sum) memcpy(out_sum, img.sum.data(), np * 3 * sizeof(double));
  if (out_sumsq) memcpy(out_sumsq, img.sumSq.data(), np * 3 * sizeof(double));
  if (out_n) memcpy(out_n, img.n.data(), np * sizeof(int32_t));
  if (out_normal) memcpy(out_normal, img.normal.data(), np * 3 * sizeof(float));
  if (out_albedo) memcpy(out_albedo, img.albedo.data(), np * 3 * sizeof(float));
  if (out_depth) memcpy(out_depth, img.depth.data(), np * sizeof(float));
  if (out_hdr || out_ldr) {
    std::vector<float> hdr(np * 4), rgb(np * 3);
    for (size_t i = 0; i < np; i++) {
      const float invN = img.n[i] > 0 ? 1.0f / (float)img.n[i] : 0.0f;
      for (int k = 0; k < 3; k++) rgb[i * 3 + k] = fmaxf((float)img.sum[i * 3 + k] * invN * s.exposure, 0.0f);
    }
    if (S.denoise) {
      std::vector<float> out(np * 3);
      denoise(S.W, S.H, rgb.data(), img.normal.data(), img.depth.data(), img.albedo.data(), img.albedoA.data(),
              S.levels, S.sigC, S.sigN, S.sigD, S.intensity, out.data());
      rgb.swap(out);
    }
    for (size_t i = 0; i < np; i++) {
      for (int k = 0; k < 3; k++) hdr[i * 4 + k] = rgb[i * 3 + k];
      hdr[i * 4 + 3] = 1.0f;
    }
    if (out_hdr) memcpy(out_hdr, hdr.data(), np * 4 * sizeof(float));
    if (out_ldr) tonemap(S.W, S.H, hdr.data(), out_ldr);
  }
  return RG_OK;
}

void orc_denoise(int32_t w, int32_t h, const float* color, const float* normal, const float* depth,
                 const float* albedo, const float* albedo_alpha, int32_t levels, float sc, float sn, float sd,
                 float intensity, float* out) {
  denoise(w, h, color, normal, depth, albedo, albedo_alpha, levels, sc, sn, sd, intensity, out);
}
void orc_tonemap(int32_t w, int32_t h, const float* hdr, float* ldr) { tonemap(w, h, hdr, ldr); }
void orc_bloom(int32_t w, int32_t h, float* hdr, float threshold, float strength, float radius, float size_aspect,
               float curve) {
  bloom(w, h, hdr, threshold, strength, radius, size_aspect, curve);
}

// RNG probes (shared specification with the device code).
float orc_lds(uint32_t x, uint32_t y, uint32_t width, uint32_t sample, uint32_t seed, int32_t dim) {
  Ctx c; c.begin(x, y, width, sample, seed); return c.lds(dim);
}
float orc_prng(uint32_t x, uint32_t y, uint32_t width, uint32_t sample, uint32_t seed, int32_t vertex, int32_t slot) {
  Ctx c; c.begin(x, y, width, sample, seed); return c.prng(vertex, slot);
}
// Analytic helpers for known-answer tests.
float orc_phase_pdf(float g, float cosTheta) {
  Medium m{}; m.g = g; return m.phasePdf(V3(0, 0, 1), V3(sqrtf(fmaxf(0.0f, 1 - cosTheta * cosTheta)), 0, cosTheta));
}
void orc_sample_phase(float g, float u1, float u2, float* out3) {
  Medium m{}; m.g = g; const V3 d = m.samplePhase(V3(0, 0, 1), u1, u2);
  out3[0] = d.x; out3[1] = d.y; out3[2] = d.z;
}

// Probes of the standalone helpers, one row per input, in the layout of the
// reference harness (oracle/ref_harness.cpp ref_bsdf_probe):
//   0 sampleGGXVNDF (Ve xyz, ax, ay, u1, u2) -> H xyz; 1 smithG1 (w xyz, ax, ay);
//   2 fresnelSchlick (cos, ior); 3 refract (d xyz, n xyz, ior) -> xyz;
//   4 buildTangentFrame (n xyz) -> t xyz, b xyz
void orc_bsdf_probe(int32_t which, const float* in, int32_t n, float* out) {
  for (int32_t i = 0; i < n; ++i) {
    if (which == 0) {
      const float* a = in + (size_t)i * 7;
      const V3 h = sampleGGXVNDF(V3(a[0], a[1], a[2]), a[3], a[4], a[5], a[6]);
      out[i * 3] = h.x; out[i * 3 + 1] = h.y; out[i * 3 + 2] = h.z;
    } else if (which == 1) {
      const float* a = in + (size_t)i * 5;
      out[i] = smithG1Aniso(V3(a[0], a[1], a[2]), a[3], a[4]);
    } else if (which == 2) {
      out[i] = Tracer::fresnelSchlick(in[i * 2], in[i * 2 + 1]);
    } else if (which == 3) {
      const float* a = in + (size_t)i * 7;
      const V3 d = Tracer::refract(V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]), a[6]);
      out[i * 3] = d.x; out[i * 3 + 1] = d.y; out[i * 3 + 2] = d.z;
    } else if (which == 4) {
      V3 t, b;
      buildTangentFrame(V3(in[i * 3], in[i * 3 + 1], in[i * 3 + 2]), t, b);
      float* o = out + (size_t)i * 6;
      o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = b.x; o[4] = b.y; o[5] = b.z;
    }
  }
}
// cosineWeightedDirection / ldsPointInTriangle on LDS dimensions dim, dim + 1
// of pixel (x, y), sample `sample` (seed 1: the reference's scramble).
void orc_cosine_direction(int32_t x, int32_t y, int32_t sample, int32_t dim, const float* normal, float* out3) {
  Ctx c; c.begin((uint32_t)x, (uint32_t)y, 1u << 16, (uint32_t)sample, 1u);
  const V3 d = cosineWeightedDirection(V3(normal[0], normal[1], normal[2]), c.lds(dim), c.lds(dim + 1));
  out3[0] = d.x; out3[1] = d.y; out3[2] = d.z;
}
void orc_point_in_triangle(int32_t x, int32_t y, int32_t sample, int32_t dim, const float* t9, float* out3) {
  Ctx c; c.begin((uint32_t)x, (uint32_t)y, 1u << 16, (uint32_t)sample, 1u);
  const V3 p = ldsPointInTriangle(V3(t9[0], t9[1], t9[2]), V3(t9[3], t9[4], t9[5]), V3(t9[6], t9[7], t9[8]),
                                  c.lds(dim), c.lds(dim + 1));
  out3[0] = p.x; out3[1] = p.y; out3[2] = p.z;
}
// The flattened view-space triangles in DFS order (positions and vertex
// normals, n x 9 each).
void orc_view_triangles(void* sp, float* pos, float* nrm) {
  const Scene& s = *static_cast<Scene*>(sp);
  for (size_t i = 0; i < s.tris.size(); ++i) {
    const Tri& t = s.tris[i];
    const V3 v[6] = {t.v1, t.v2, t.v3, t.n1, t.n2, t.n3};
    for (int k = 0; k < 3; ++k) {
      pos[i * 9 + k * 3] = v[k].x; pos[i * 9 + k * 3 + 1] = v[k].y; pos[i * 9 + k * 3 + 2] = v[k].z;
      nrm[i * 9 + k * 3] = v[3 + k].x; nrm[i * 9 + k * 3 + 1] = v[3 + k].y; nrm[i * 9 + k * 3 + 2] = v[3 + k].z;
    }
  }
}
int32_t orc_num_triangles(void* sp) { return (int32_t)static_cast<Scene*>(sp)->tris.size(); }

// Environment-map probes for the tests: n view-space directions (n x 3).
// radiance: n x 3 (sampleEnvironment); pdf: n (envmapDirectionPdf);
// sample: u n x 2 -> dir n x 3 + pdf n (sampleEnvmapDirection).
void orc_env_eval(void* sp, const float* dirs, int32_t n, float* out_rgb, float* out_pdf) {
  const Scene& s = *static_cast<Scene*>(sp);
  Ctx c{};
  Tracer t(s, c);
  for (int i = 0; i < n; i++) {
    const V3 d(dirs[i * 3], dirs[i * 3 + 1], dirs[i * 3 + 2]);
    const C3 L = t.sampleEnvironment(d);
    out_rgb[i * 3] = L.x; out_rgb[i * 3 + 1] = L.y; out_rgb[i * 3 + 2] = L.z;
    out_pdf[i] = t.envmapDirectionPdf(d);
  }
}
void orc_env_sample(void* sp, const float* u, int32_t n, float* out_dir, float* out_pdf) {
  const Scene& s = *static_cast<Scene*>(sp);
  Ctx c{};
  Tracer t(s, c);
  for (int i = 0; i < n; i++) {
    V3 d;
    float pdf;
    t.sampleEnvmapDirection(u[i * 2], u[i * 2 + 1], d, pdf);
    out_dir[i * 3] = d.x; out_dir[i * 3 + 1] = d.y; out_dir[i * 3 + 2] = d.z;
    out_pdf[i] = pdf;
  }
}

// Medium fields of medium `m` at camera-space points: n x 5 (density, emission rgb, ior).
void orc_medium_eval(void* sp, int32_t m, const float* pts, int32_t n, float* out) {
  const Medium& M = static_cast<Scene*>(sp)->media[m];
  for (int i = 0; i < n; i++) {
    const V3 p(pts[i * 3], pts[i * 3 + 1], pts[i * 3 + 2]);
    const C3 e = M.emissionAt(p);
    out[i * 5] = M.densityAt(p);
    out[i * 5 + 1] = e.x; out[i * 5 + 2] = e.y; out[i * 5 + 3] = e.z;
    out[i * 5 + 4] = M.iorAt(p);
  }
}
// Heat-haze bending of rays n x 7 (origin, direction, length) -> n x 6.
void orc_medium_bend(void* sp, int32_t m, const float* rays, int32_t n, float* out) {
  const Medium& M = static_cast<Scene*>(sp)->media[m];
  for (int i = 0; i < n; i++) {
    const float* r = rays + (size_t)i * 7;
    const Ray b = M.bendRay(Ray{V3(r[0], r[1], r[2]), V3(r[3], r[4], r[5])}, r[6]);
    out[i * 6] = b.o.x; out[i * 6 + 1] = b.o.y; out[i * 6 + 2] = b.o.z;
    out[i * 6 + 3] = b.d.x; out[i * 6 + 4] = b.d.y; out[i * 6 + 5] = b.d.z;
  }
}
// Probes of medium `m` in the layout of the reference harness
// (oracle/ref_harness.cpp ref_medium_probe): 0 transmittance (d) -> rgb;
// 1 sampleFreeFlight (u) -> t; 2 samplePhase (wo xyz, u1, u2) -> xyz;
// 3 phasePdf (wo xyz, wi xyz) -> pdf; 4 fields (p xyz) -> density, emission
// rgb, ior; 5 bendRay (o xyz, d xyz, length) -> o xyz, d xyz.
void orc_medium_probe(void* sp, int32_t m, int32_t which, const float* in, int32_t n, float* out) {
  const Medium& M = static_cast<Scene*>(sp)->media[m];
  for (int32_t i = 0; i < n; i++) {
    if (which == 0) {
      const C3 c = M.transmittance(in[i]);
      out[i * 3] = c.x; out[i * 3 + 1] = c.y; out[i * 3 + 2] = c.z;
    } else if (which == 1) {
      out[i] = M.sampleFreeFlight(in[i]);
    } else if (which == 2) {
      const float* a = in + (size_t)i * 5;
      const V3 d = M.samplePhase(V3(a[0], a[1], a[2]), a[3], a[4]);
      out[i * 3] = d.x; out[i * 3 + 1] = d.y; out[i * 3 + 2] = d.z;
    } else if (which == 3) {
      const float* a = in + (size_t)i * 6;
      out[i] = M.phasePdf(V3(a[0], a[1], a[2]), V3(a[3], a[4], a[5]));
    } else if (which == 4) {
      orc_medium_eval(sp, m, in + (size_t)i * 3, 1, out + (size_t)i * 5);
    } else if (which == 5) {
      orc_medium_bend(sp, m, in + (size_t)i * 7, 1, out + (size_t)i * 6);
    }
  }
}
// n volume-light NEE draws at one camera-space point (sample index i, vertex 0
// of pixel (0, 0)): direction, solid-angle pdf, radiance and success flag.
void orc_volume_nee(void* sp, const float* hit, const float* normal, int32_t n, uint32_t seed, float* out_dir,
                    float* out_pdf, float* out_le, uint8_t* out_ok) {
  const Scene& s = *static_cast<Scene*>(sp);
  for (int i = 0; i < n; i++) {
    Ctx c{};
    c.begin(0, 0, 1, (uint32_t)i, seed);
    Tracer t(s, c);
    V3 d; float pdf = 0.0f; C3 le;
    const bool ok = t.sampleVolumeLightForNEE(V3(hit[0], hit[1], hit[2]), V3(normal[0], normal[1], normal[2]), 0, d,
                                              pdf, le);
    out_dir[i * 3] = d.x; out_dir[i * 3 + 1] = d.y; out_dir[i * 3 + 2] = d.z;
    out_pdf[i] = pdf;
    out_le[i * 3] = le.x; out_le[i * 3 + 1] = le.y; out_le[i * 3 + 2] = le.z;
    out_ok[i] = ok ? 1 : 0;
  }
}
int32_t orc_num_volume_lights(void* sp) { return (int32_t)static_cast<Scene*>(sp)->vols.size(); }

}  // extern "C"
