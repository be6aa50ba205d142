// rg_trace.cu - wavefront kernels of the shader-5 path tracer.
//
// The reference traces one sample at a time with a recursive
// tracePath -> shade -> {Diffuse,Glossy,Refraction,Transparency}Shader ->
// tracePath loop (rayrenderer.cpp:1596-1864, :2776-2896, bsdf.cpp:54-610).
// Here every bounce of a whole wave of paths is one kernel sequence:
//   generate -> [extend -> shade -> connect(A) -> connect(B)] x depth -> accumulate
// Rays live in SoA float4 queues (128-bit loads), the shade kernel compacts
// the surviving paths into the next queue with warp ballots plus one atomic
// per warp, and NEE shadow rays go to two shadow queues (area lights /
// point lights) whose visibility kernels add the contribution to the path.
// The mix shader picks one lobe per vertex with probability proportional to
// its weight (the reference evaluates every lobe); all other estimator rules
// (MIS weights, back-face rules, Russian roulette on the reference's
// throughput, depth cap, media) follow the reference line by line.
#include <cuda_fp16.h>

#include "rg_device.cuh"
#include "rg_medium.cuh"
#include "rg_trace.cuh"
#include "rg_traverse.cuh"

namespace rg {

// ------------------------------------------------------------ helpers ----
__device__ __forceinline__ int warpPush(int* counter, bool want) {
  const unsigned act = __activemask();
  const unsigned m = __ballot_sync(act, want);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (m) {
    const int leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(counter, __popc(m));
    base = __shfl_sync(act, base, leader);
  }
  return want ? base + __popc(m & ((1u << lane) - 1u)) : -1;
}

__device__ __forceinline__ void warpAddStat(unsigned long long* dst, uint32_t v) {
  const unsigned act = __activemask();
  unsigned long long s = v;
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(act, s, o);
  const int leader = __ffs(act) - 1;
  if ((int)(threadIdx.x & 31) == leader && s) atomicAdd(dst, s);
}

// raycommon.h:82-85
__device__ __forceinline__ V3 surfaceOrigin(V3 hit, V3 dir, V3 n) {
  const float side = dot(dir, n) >= 0.0f ? 1.0f : -1.0f;
  return hit + n * (side * kSurfaceThickness);
}

// raycommon.cpp:94-115
__device__ __forceinline__ V3 cosineWeightedDirection(V3 n, float r1, float r2) {
  const float theta = acosf(sqrtf(1.0f - r1));
  const float phi = 2.0f * kPi * r2;
  float st, ct, sp, cp;
  sincosf(theta, &st, &ct);
  sincosf(phi, &sp, &cp);
  V3 tangent = fabsf(n.x) > fabsf(n.y) ? normalize(cross(v3(0, 1, 0), n)) : normalize(cross(v3(1, 0, 0), n));
  const V3 bit = cross(n, tangent);
  return normalize(tangent * (st * cp) + bit * (st * sp) + n * ct);
}

// Uniform direction on the sphere flipped into n's hemisphere (stand-in for
// ugm randomRayInHemisphere, which is not vendored).
__device__ __forceinline__ V3 randomRayInHemisphere(V3 n, float u1, float u2) {
  const float z = 1.0f - 2.0f * u1;
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  float s, c;
  sincosf(2.0f * kPi * u2, &s, &c);
  V3 d = v3(r * c, r * s, z);
  if (dot(d, n) < 0.0f) d = -d;
  return d;
}

// buildTangentFrame: bsdf.cpp:129-135
__device__ __forceinline__ void buildTangentFrame(V3 n, V3& t, V3& b) {
  const V3 up = fabsf(n.y) > 0.99f ? v3(1, 0, 0) : v3(0, 1, 0);
  t = normalize(cross(up, n));
  b = cross(n, t);
}

// smithG1 for anisotropic GGX in the local frame: bsdf.cpp:164-170
__device__ __forceinline__ float smithG1(V3 w, float ax, float ay) {
  if (w.z <= 0.0f) return 0.0f;
  const float ax2 = (ax * w.x) * (ax * w.x), ay2 = (ay * w.y) * (ay * w.y);
  const float lambda = 0.5f * (sqrtf(1.0f + (ax2 + ay2) / (w.z * w.z)) - 1.0f);
  return 1.0f / (1.0f + lambda);
}

// sampleGGXVNDF (Heitz 2018): bsdf.cpp:139-161; Ve is the local view direction
__device__ __forceinline__ V3 sampleGGXVNDF(V3 Ve, float ax, float ay, float u1, float u2) {
  const V3 Vh = normalize(v3(ax * Ve.x, ay * Ve.y, Ve.z));
  const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
  const V3 T1 = lensq > 0.0f ? v3(-Vh.y, Vh.x, 0.0f) * (1.0f / sqrtf(lensq)) : v3(1, 0, 0);
  const V3 T2 = cross(Vh, T1);
  const float rr = sqrtf(u1);
  float sphi, cphi;
  sincosf(2.0f * kPi * u2, &sphi, &cphi);
  const float t1 = rr * cphi;
  float t2 = rr * sphi;
  const float sw = 0.5f * (1.0f + Vh.z);
  t2 = (1.0f - sw) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + sw * t2;
  const V3 Nh = T1 * t1 + T2 * t2 + Vh * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2));
  return normalize(v3(ax * Nh.x, ay * Nh.y, fmaxf(0.0f, Nh.z)));
}

// fresnelSchlick: bsdf.cpp:32-37
__device__ __forceinline__ float fresnelSchlick(float cosTheta, float ior) {
  float r0 = (1.0f - ior) / (1.0f + ior);
  r0 = r0 * r0;
  const float mm = 1.0f - cosTheta;
  return r0 + (1.0f - r0) * (mm * mm) * (mm * mm) * mm;
}

// refract: bsdf.cpp:39-52 (total internal reflection -> reflect)
__device__ __forceinline__ V3 refractDir(V3 d, V3 n, float ior) {
  const V3 nl = dot(d, n) < 0.0f ? n : -n;
  const bool into = dot(nl, n) > 0.0f;
  const float rr = into ? 1.0f / ior : ior;
  const float c = dot(d, nl);
  const float tt = 1.0f - rr * rr * (1.0f - c * c);
  if (tt < 0.0f) return reflect(d, n);
  return normalize(d * rr - n * ((into ? 1.0f : -1.0f) * (c * rr + sqrtf(tt))));
}

// ldsPointInTriangle: raycommon.cpp:117-122 (u, w: two LDS draws)
__device__ __forceinline__ V3 ldsPointInTriangle(V3 v1, V3 v2, V3 v3, float u, float w) {
  if (u + w > 1.0f) {
    u = 1.0f - u;
    w = 1.0f - w;
  }
  return v1 + (v2 - v1) * u + (v3 - v1) * w;
}

// sampleFreeFlight: medium.cpp:475-480 (hero: the mean of sigma_t)
__device__ __forceinline__ float sampleFreeFlight(float hero, float u) {
  if (hero <= 0.0f) return 1e30f;
  const float xi = fminf(0.9999999f, fmaxf(0.0f, u));
  return -logf(1.0f - xi) / hero;
}

// Henyey-Greenstein samplePhase around the travel direction wo: medium.cpp:496-517,
// with coordSystem (:482-494)
__device__ __forceinline__ V3 samplePhaseHG(V3 wo, float g, float u1, float u2) {
  float cosTheta;
  if (fabsf(g) < 1e-3f) {
    cosTheta = 1.0f - 2.0f * u1;
  } else {
    const float sq = (1.0f - g * g) / (1.0f - g + 2.0f * g * u1);
    cosTheta = (1.0f + g * g - sq * sq) / (2.0f * g);
  }
  const float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - cosTheta * cosTheta));
  float sp, cp;
  sincosf(2.0f * kPi * u2, &sp, &cp);
  V3 t1;
  if (fabsf(wo.x) > fabsf(wo.y)) {
    const float inv = 1.0f / sqrtf(wo.x * wo.x + wo.z * wo.z);
    t1 = v3(-wo.z * inv, 0.0f, wo.x * inv);
  } else {
    const float inv = 1.0f / sqrtf(wo.y * wo.y + wo.z * wo.z);
    t1 = v3(0.0f, wo.z * inv, -wo.y * inv);
  }
  const V3 t2 = cross(wo, t1);
  return normalize(t1 * (sinTheta * cp) + t2 * (sinTheta * sp) + wo * cosTheta);
}

// Henyey-Greenstein phasePdf: medium.cpp:519-525
__device__ __forceinline__ float phasePdfHG(V3 wo, V3 wi, float g) {
  const float cosT = dot(wo, wi);
  const float den = 1.0f + g * g - 2.0f * g * cosT;
  return (1.0f - g * g) * (1.0f / (4.0f * kPi)) / (den * sqrtf(fmaxf(1e-8f, den)));
}

__device__ __forceinline__ float srgbToLinear(float c) {  // texture.cpp:204-207
  if (c <= 0.04045f) return c * (1.0f / 12.92f);
  return powf((c + 0.055f) * (1.0f / 1.055f), 2.4f);
}

// Texture::sample: texture.cpp:210-241
__device__ V3 texSample(const DevScene& S, int tex, float u, float v) {
  const DevTexture T = S.textures[tex];
  if (T.width <= 0 || T.height <= 0) return v3(0, 0, 0);
  if (!(u == u) || !(v == v)) return v3(0, 0, 0);
  float fu = u - floorf(u), fv = v - floorf(v);
  if (fu < 0.0f || fu >= 1.0f) fu = 0.0f;
  if (fv < 0.0f || fv >= 1.0f) fv = 0.0f;
  const int x = min(max((int)(fu * T.width), 0), T.width - 1);
  const int y = min(max((int)(fv * T.height), 0), T.height - 1);
  const float4 p = __ldg(T.texels + (size_t)y * T.width + x);
  V3 c = v3(p.x, p.y, p.z);
  if (!T.isHdr) c = v3(srgbToLinear(c.x), srgbToLinear(c.y), srgbToLinear(c.z));
  return c;
}

struct Hit {
  V3 p;        // hit point
  V3 n;        // interpolated shading normal
  V3 gn;       // ti.normalizedpd
  float uvx, uvy;
  int mesh;
  int prim;
};

__device__ __forceinline__ Hit loadHit(const DevScene& S, int prim, V3 o, V3 d, float t, float u, float v) {
  Hit h;
  const float4* ts = S.triShade + (size_t)prim * 3;
  const float4 a = __ldg(ts), b = __ldg(ts + 1), c = __ldg(ts + 2);
  const V3 n1 = v3(a.x, a.y, a.z), n2 = v3(a.w, b.x, b.y), n3 = v3(b.z, b.w, c.x);
  const float w = 1.0f - u - v;
  h.n = normalize(n1 * w + n2 * u + n3 * v);
  h.gn = v3(c.y, c.z, c.w);
  h.p = o + d * t;
  h.mesh = __float_as_int(__ldg(&S.triVerts[(size_t)prim * 3].w));
  h.prim = prim;
  h.uvx = h.uvy = 0.0f;
  if (S.triUV) {
    const float2 t1 = S.triUV[(size_t)prim * 3], t2 = S.triUV[(size_t)prim * 3 + 1], t3 = S.triUV[(size_t)prim * 3 + 2];
    h.uvx = t1.x * w + t2.x * u + t3.x * v;
    h.uvy = t1.y * w + t2.y * u + t3.y * v;
  }
  return h;
}

__device__ __forceinline__ V3 matColor(const DevMaterial& m) { return v3(m.cr, m.cg, m.cb); }
__device__ __forceinline__ V3 albedoOf(const DevScene& S, const DevMaterial& m, const Hit& h) {
  V3 a = matColor(m);
  if (m.texture >= 0) a = a * texSample(S, m.texture, h.uvx * m.tileU, h.uvy * m.tileV);
  return a;
}

// An area-light sample (the pick in traceAreaLight / sampleAreaLightForNEE,
// rayrenderer.cpp:1916-2036).
struct LightSample {
  V3 p;        // point on the emitter
  V3 ln;       // interpolated (unnormalised) emitter normal
  float area;  // triangles in the mesh * triangle area
  V3 Le;
};

__device__ bool pickAreaLight(const DevScene& S, const Rng& rng, int v, int lightObj, LightSample& ls) {
  const int2 om = S.lightObjMeshes[lightObj];
  if (om.y <= 0) return false;
  const int mesh = S.lightMeshList[om.x + pickIndex(rng.prng(v, S_MESH), om.y)];
  const int2 mt = S.lightMeshTris[mesh];
  if (mt.y <= 0) return false;
  const int k = mt.x + pickIndex(rng.prng(v, S_TRI), mt.y);
  const float4* lt = S.lightTris + (size_t)k * 6;
  const float4 a = __ldg(lt), b = __ldg(lt + 1), c = __ldg(lt + 2);
  const float4 na = __ldg(lt + 3), nb = __ldg(lt + 4), nc = __ldg(lt + 5);
  const V3 v1 = xyz(a), v2 = xyz(b), v3_ = xyz(c);
  ls.p = ldsPointInTriangle(v1, v2, v3_, rng.lds(rng.neeDim(v)), rng.lds(rng.neeDim(v) + 1));
  // calcVertexInterpolation(tri, p): rayrenderer.cpp:2337-2352
  const V3 f1 = v1 - ls.p, f2 = v2 - ls.p, f3 = v3_ - ls.p;
  const V3 c1 = cross(f2, f3), c2 = cross(f3, f1), c3 = cross(f1, f2);
  const float a1 = sqrtf(dot(c1, c1)) * a.w, a2 = sqrtf(dot(c2, c2)) * a.w, a3 = sqrtf(dot(c3, c3)) * a.w;
  ls.ln = xyz(na) * a1 + xyz(nb) * a2 + xyz(nc) * a3;
  ls.area = (float)mt.y * b.w;
  const DevMaterial& m = S.mats[S.objMat[lightObj]];
  ls.Le = matColor(m) * m.emission;
  return true;
}

struct Shadow {
  bool on;
  V3 o, d;
  float tmax;
  V3 c;
};

// traceAreaLight (rayrenderer.cpp:1916-1984) up to the shadow test; the
// contribution is deferred to the shadow ray.  `w` multiplies the result.
__device__ void traceAreaLight(const DevScene& S, const DevRender& R, const Rng& rng, int v, V3 hit, V3 n, V3 w,
                               Shadow& sh) {
  const int N = S.numAreaLights;
  if (N <= 0) return;
  const int lo = S.areaLightObj[pickIndex(rng.prng(v, S_LIGHT), N)];
  LightSample ls;
  if (!pickAreaLight(S, rng, v, lo, ls)) return;
  const V3 lr = ls.p - hit;
  const V3 ld = normalize(lr);
  const float dObj = dot(ld, n);
  if (dObj <= 0.0f) return;
  const float dLight = dot(-ld, ls.ln);
  if (dLight <= 0.0f) return;
  const float lf = R.lightFix ? (float)N : 1.0f;
  const float r2 = dot(lr, lr);
  const float pl = r2 / (dLight * ls.area) / lf;
  const float pb = dObj / kPi;
  const float wl = pl * pl / (pl * pl + pb * pb);
  sh.on = true;
  sh.o = surfaceOrigin(hit, lr, n);
  sh.d = lr;
  sh.tmax = 0.99999f;
  sh.c = w * ls.Le * (dObj * dLight * ls.area / (kPi * r2) * wl * lf);
}

// tracePointLight (rayrenderer.cpp:2205-2269) up to the shadow test.
__device__ void tracePointLight(const DevScene& S, int idx, V3 hit, V3 n, V3 w, Shadow& sh) {
  const DevPointLight P = S.points[idx];
  const V3 lr = v3(P.px, P.py, P.pz) - hit;
  const V3 ldir = normalize(lr);
  const float dObj = dot(ldir, n);
  float dLight = dot(ldir, v3(P.nx, P.ny, P.nz));
  if (!(dObj > 0.0f)) return;
  const DevMaterial& m = S.mats[P.material];
  if (m.spotRange > 0.0f) {
    const float spotDot = cosf(m.spotRange * 0.5f * (180.0f / kPi));
    const float e0 = fmaxf(spotDot - 0.1f, 0.0f), e1 = fminf(spotDot + 0.1f, 1.0f);
    float x = (dLight - e0) / (e1 - e0);
    x = fminf(fmaxf(x, 0.0f), 1.0f);
    dLight = dLight * (x * x * (3.0f - 2.0f * x));
  } else {
    dLight = fabsf(dObj);
  }
  if (!(dLight > 0.0f)) return;
  const float da = 1.0f / dot(lr, lr);
  const float lum = m.emission * dLight * da;
  V3 col = matColor(m) * lum;
  col = v3(fminf(fmaxf(col.x, 0.0f), 1.0f), fminf(fmaxf(col.y, 0.0f), 1.0f), fminf(fmaxf(col.z, 0.0f), 1.0f));
  sh.on = true;
  sh.o = surfaceOrigin(hit, lr, n);
  sh.d = lr;
  sh.tmax = 0.99999f;
  sh.c = w * col;
}

// traceLight (rayrenderer.cpp:2271-2293): one area light + one point light.
__device__ void traceLight(const DevScene& S, const DevRender& R, const Rng& rng, int v, V3 hit, V3 n, V3 w,
                           Shadow& a, Shadow& b) {
  traceAreaLight(S, R, rng, v, hit, n, w, a);
  const int np = S.numPointLights;
  if (np > 0) tracePointLight(S, np == 1 ? 0 : pickIndex(rng.prng(v, S_POINT), np), hit, n, w, b);
}

// sampleAreaLightForNEE (rayrenderer.cpp:1986-2036) up to the shadow test.
__device__ bool sampleAreaLightForNEE(const DevScene& S, const DevRender& R, const Rng& rng, int v, V3 hit, V3 n,
                                      V3& dir, float& pdf, V3& Le, Shadow& sh) {
  const int N = S.numAreaLights;
  if (N <= 0) return false;
  const int lo = S.areaLightObj[pickIndex(rng.prng(v, S_LIGHT), N)];
  LightSample ls;
  if (!pickAreaLight(S, rng, v, lo, ls)) return false;
  const V3 lr = ls.p - hit;
  dir = normalize(lr);
  const float cObj = dot(dir, n);
  if (cObj <= 0.0f) return false;
  const float cLight = dot(-dir, ls.ln);
  if (cLight <= 0.0f) return false;
  const float lf = R.lightFix ? (float)N : 1.0f;
  pdf = dot(lr, lr) / (cLight * ls.area) / lf;
  Le = ls.Le;
  sh.o = surfaceOrigin(hit, lr, n);
  sh.d = lr;
  sh.tmax = 0.99999f;
  return true;
}

// ---- equirectangular environment map ----------------------------------------
// Directions are view space, as in the reference (the map turns with the
// camera).  Lookups go through Texture::sample; the importance-sampling grid
// and its CDFs (Scene::buildEnvmapCDF) are built at scene set-up.  These are
// kept out of line (only scenes with an environment map reach them) and read
// the scene through its copy in the job table (global memory), with scalar
// arguments and by-value results, so the shade kernel keeps no local frame.
constexpr float kInv2Pi = (float)(0.5 / 3.14159265358979323846);
constexpr float kInvPi = (float)(1.0 / 3.14159265358979323846);
constexpr float kPi2 = (float)(3.14159265358979323846 * 3.14159265358979323846);

__device__ __forceinline__ bool envSampling(const DevScene* S) {
  return S->envTex >= 0 && S->envW > 0 && S->envTotal > 0.0f;
}
__device__ __forceinline__ bool cubeSampling(const DevScene* S) { return S->envCubeW > 0 && S->envCubeTotal > 0.0f; }

// Cubemap face and face-local (s, t) of a rotated direction (OpenGL
// convention, rayrenderer.cpp:1311-1333).
__device__ __forceinline__ int cubeFace(float rx, float ry, float rz, float& sc, float& tc, float& ma) {
  const float ax = fabsf(rx), ay = fabsf(ry), az = fabsf(rz);
  if (ax >= ay && ax >= az) {
    ma = ax;
    if (rx > 0) { sc = -rz; tc = ry; return 0; }
    sc = rz; tc = ry; return 1;
  }
  if (ay >= ax && ay >= az) {
    ma = ay;
    if (ry > 0) { sc = rx; tc = rz; return 2; }
    sc = rx; tc = -rz; return 3;
  }
  ma = az;
  if (rz > 0) { sc = rx; tc = ry; return 4; }
  sc = -rx; tc = ry; return 5;
}

__device__ __forceinline__ float cubeTexelLum(const DevScene* S, int face, int x, int y) {
  const float4 c = __ldg(S->textures[S->envFace[face]].texels + (size_t)y * S->envCubeW + x);
  return fmaxf(0.0f, 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z);
}

__device__ __forceinline__ float envTexelLum(const DevScene* S, int x, int y) {
  const float4 c = __ldg(S->textures[S->envTex].texels + (size_t)y * S->envW + x);
  return fmaxf(0.0f, 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z);
}

// sampleEnvironment (rayrenderer.cpp:1299-1348): the cubemap when present, else
// the equirectangular map
__device__ __noinline__ V3 envRadiance(const DevScene* S, V3 dir) {
  if (!S->envOn) return v3(0, 0, 0);
  const V3 d = normalize(dir);
  const float rx = d.x * S->envCosY - d.z * S->envSinY;
  const float rz = d.x * S->envSinY + d.z * S->envCosY;
  if (S->envCube) {
    float sc, tc, ma;
    const int face = cubeFace(rx, d.y, rz, sc, tc, ma);
    const float u = 0.5f * (sc / ma + 1.0f);
    const float v = 0.5f * (1.0f - tc / ma);
    return texSample(*S, S->envFace[face], u, v) * S->envIntensity;
  }
  const float u = 0.5f + atan2f(rz, rx) * kInv2Pi;
  const float v = 0.5f - asinf(fminf(fmaxf(d.y, -1.0f), 1.0f)) * kInvPi;
  return texSample(*S, S->envTex, u, v) * S->envIntensity;
}

// envmapDirectionPdf (rayrenderer.cpp:1521-1573)
__device__ __noinline__ float envPdf(const DevScene* S, V3 dir) {
  const V3 d = normalize(dir);
  const float rx = d.x * S->envCosY - d.z * S->envSinY;
  const float rz = d.x * S->envSinY + d.z * S->envCosY;
  if (cubeSampling(S)) {
    float sc, tc, ma;
    const int face = cubeFace(rx, d.y, rz, sc, tc, ma);
    if (ma <= 0.0f) return 0.0f;
    const float u = 0.5f * (sc / ma + 1.0f);
    const float v = 0.5f * (1.0f - tc / ma);
    const int W = S->envCubeW;
    const int x = min(max((int)(u * W), 0), W - 1);
    const int y = min(max((int)(v * W), 0), W - 1);
    return cubeTexelLum(S, face, x, y) * (float)(W * W) / (4.0f * S->envCubeTotal);
  }
  if (!envSampling(S)) return 0.0f;
  const int W = S->envW, H = S->envH;
  const float u = 0.5f + atan2f(rz, rx) * kInv2Pi;
  const float v = 0.5f - asinf(fminf(fmaxf(d.y, -1.0f), 1.0f)) * kInvPi;
  const int x = min(max((int)(u * W), 0), W - 1);
  const int y = min(max((int)(v * H), 0), H - 1);
  const float lum = envTexelLum(S, x, y);
  const float sinTheta = sinf(kPi * v);
  if (sinTheta <= 0.0f) return 0.0f;
  const float pdfUV = (lum * sinTheta) / S->envTotal;
  return pdfUV * (float)(W * H) / (2.0f * kPi2 * sinTheta);
}

// searchCDF (rayrenderer.cpp:1353-1362): largest i with cdf[i] <= u, in [0, n-1]
__device__ __forceinline__ int searchCDF(const float* __restrict__ cdf, int n, float u) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(cdf + mid + 1) <= u) lo = mid + 1;
    else hi = mid;
  }
  return lo < n ? lo : n - 1;
}

struct EnvSample {
  V3 dir;
  float pdf;  // 0: no sample
  V3 Li;
};

// sampleEnvmapDirection, equirectangular branch (rayrenderer.cpp:1426-1482),
// plus the radiance toward the sample (the NEE part of sampleEnvmapForNEE,
// rayrenderer.cpp:2038-2065, before its front-facing and shadow tests).
__device__ __noinline__ EnvSample envSample(const DevScene* S, float u0, float u1) {
  EnvSample r;
  r.dir = v3(0, 1, 0);
  r.pdf = 0.0f;
  r.Li = v3(0, 0, 0);
  if (cubeSampling(S)) {  // face, row, texel (rayrenderer.cpp:1384-1433)
    const int W = S->envCubeW, H = W;
    const int face = searchCDF(S->cubeMargFace, 6, u0);
    const float faceLo = __ldg(S->cubeMargFace + face), faceSpan = __ldg(S->cubeMargFace + face + 1) - faceLo;
    const float u0r = faceSpan > 0.0f ? (u0 - faceLo) / faceSpan : 0.5f;
    const float* marY = S->cubeMargY + (size_t)face * (H + 1);
    const int y = searchCDF(marY, H, u0r);
    const float yLo = __ldg(marY + y), ySpan = __ldg(marY + y + 1) - yLo;
    const float yFrac = ySpan > 0.0f ? (u0r - yLo) / ySpan : 0.5f;
    const float* condX = S->cubeCond + ((size_t)face * H + y) * (W + 1);
    const int x = searchCDF(condX, W, u1);
    const float xLo = __ldg(condX + x), xSpan = __ldg(condX + x + 1) - xLo;
    const float xFrac = xSpan > 0.0f ? (u1 - xLo) / xSpan : 0.5f;
    const float sc = 2.0f * ((x + xFrac) / (float)W) - 1.0f, tc = 1.0f - 2.0f * ((y + yFrac) / (float)H);
    V3 l;  // cubeFaceDir (rayrenderer.cpp:1367-1376)
    switch (face) {
      case 0: l = v3(1.0f, tc, -sc); break;
      case 1: l = v3(-1.0f, tc, sc); break;
      case 2: l = v3(sc, 1.0f, tc); break;
      case 3: l = v3(sc, -1.0f, -tc); break;
      case 4: l = v3(sc, tc, 1.0f); break;
      default: l = v3(-sc, tc, -1.0f); break;
    }
    r.dir = normalize(v3(l.x * S->envCosY + l.z * S->envSinY, l.y, -l.x * S->envSinY + l.z * S->envCosY));
    r.pdf = cubeTexelLum(S, face, x, y) * (float)(W * H) / (4.0f * S->envCubeTotal);
    if (r.pdf > 0.0f) r.Li = envRadiance(S, r.dir);
    return r;
  }
  if (!envSampling(S)) return r;
  const int W = S->envW, H = S->envH;
  const int y = searchCDF(S->envMarg, H, u0);
  const float* row = S->envCond + (size_t)y * (W + 1);
  const int x = searchCDF(row, W, u1);
  const float yPrev = __ldg(S->envMarg + y), ySpan = __ldg(S->envMarg + y + 1) - yPrev;
  const float xPrev = __ldg(row + x), xSpan = __ldg(row + x + 1) - xPrev;
  const float yFrac = ySpan > 0.0f ? (u0 - yPrev) / ySpan : 0.5f;
  const float xFrac = xSpan > 0.0f ? (u1 - xPrev) / xSpan : 0.5f;
  const float u = (x + xFrac) / (float)W;
  const float v = (y + yFrac) / (float)H;
  const float phi = (u - 0.5f) * 2.0f * kPi;
  const float theta = (0.5f - v) * kPi;
  const float cosT = cosf(theta);
  const float dx = cosT * cosf(phi), dy = sinf(theta), dz = cosT * sinf(phi);
  r.dir = normalize(v3(dx * S->envCosY + dz * S->envSinY, dy, -dx * S->envSinY + dz * S->envCosY));
  const float lum = envTexelLum(S, x, y);
  const float sinTheta = sinf(kPi * v);
  if (sinTheta <= 0.0f) return r;
  const float pdfUV = (lum * sinTheta) / S->envTotal;
  r.pdf = pdfUV * (float)(W * H) / (2.0f * kPi2 * sinTheta);
  if (r.pdf > 0.0f) r.Li = envRadiance(S, r.dir);
  return r;
}

// sampleEnvmapForNEE (rayrenderer.cpp:2038-2065) up to the shadow test: an
// unbounded shadow ray (tmax 1e30) with the point/env occluders, queue C.
__device__ __forceinline__ bool envNEE(const DevScene* S, const Rng& rng, int v, V3 hit, V3 n, EnvSample& e,
                                       Shadow& sh) {
  if (!envSampling(S) && !cubeSampling(S)) return false;
  e = envSample(S, rng.prng(v, S_ENV0), rng.prng(v, S_ENV1));
  if (e.pdf <= 0.0f || dot(e.dir, n) <= 0.0f) return false;
  sh.o = surfaceOrigin(hit, e.dir, n);
  sh.d = e.dir;
  sh.tmax = 1e30f;
  return true;
}

// Radiance of a ray that left the scene, with the BSDF-side MIS weight against
// environment NEE when the last bounce advertised a pdf (rayrenderer.cpp:1619-1630).
__device__ __noinline__ V3 envMiss(const DevScene* S, V3 d, float bsdfPdf) {
  V3 env = envRadiance(S, d);
  if (bsdfPdf > 0.0f) {
    const float e = envPdf(S, d);
    const float b2 = bsdfPdf * bsdfPdf, e2 = e * e;
    env = env * ((b2 + e2 > 0.0f) ? b2 / (b2 + e2) : 1.0f);
  }
  return env;
}

// ------------------------------------------------------------ kernels ----
// Segment of the wave holding path p (segments are few; linear scan after a
// binary search on the path prefix).
__device__ __forceinline__ int segmentOfPath(const DevWave& W, int p) {
  int lo = 0, hi = W.numSegments - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (W.segs[mid].pathBase <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}
__device__ __forceinline__ int segmentOfPixel(const DevWave& W, int t) {
  int lo = 0, hi = W.numSegments - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (W.segs[mid].pixBase <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ int dimBaseOf(const DevRender& R) { return (R.dof >= 0.001f && R.aperture > 0.0f) ? 4 : 2; }

// accumulatePixelSamples ray generation (rayrenderer.cpp:847-934).
__device__ void primaryRay(const DevRender& R, const Rng& rng, int x, int y, V3& o, V3& d) {
  const float vs = R.viewScale;
  const float dx = ((float)x + 0.5f - R.halfW) * vs;
  const float dy = -((float)y + 0.5f - R.halfH) * vs;
  const float jx = rng.lds(0), jy = rng.lds(1);
  const float jxo = R.aa ? (jx - 0.5f) : 0.0f, jyo = R.aa ? (jy - 0.5f) : 0.0f;
  if (R.dof >= 0.001f && R.aperture > 0.0f) {
    const float pxDx = dx + jxo * vs, pxDy = dy - jyo * vs;
    const V3 fp = v3(pxDx * R.dof, pxDy * R.dof, -R.dof);
    const float du = rng.lds(2), dv = rng.lds(3);
    float ox, oy;
    if (R.blades >= 3) {
      const int N = R.blades;
      const float u0 = du * (float)N;
      const int wedge = (int)fminf((float)(N - 1), floorf(u0));
      float s = u0 - (float)wedge, t = dv;
      if (s + t > 1.0f) { s = 1.0f - s; t = 1.0f - t; }
      const float step = 2.0f * kPi / (float)N;
      const float a0 = R.apertureRot + step * (float)wedge, a1 = a0 + step;
      ox = (cosf(a0) * s + cosf(a1) * t) * R.aperture;
      oy = (sinf(a0) * s + sinf(a1) * t) * R.aperture;
    } else {
      const float a = 2.0f * du - 1.0f, b = 2.0f * dv - 1.0f;
      float r, phi;
      if (a == 0.0f && b == 0.0f) { r = 0.0f; phi = 0.0f; }
      else if (a * a > b * b) { r = a; phi = (kPi / 4.0f) * (b / a); }
      else { r = b; phi = (kPi / 2.0f) - (kPi / 4.0f) * (a / b); }
      ox = r * cosf(phi) * R.aperture;
      oy = r * sinf(phi) * R.aperture;
    }
    o = v3(ox, oy, 0.0f);
    d = normalize(fp - o);
  } else {
    o = v3(0, 0, 0);
    d = normalize(v3(dx + jxo * vs, dy - jyo * vs, -1.0f));
  }
}

__global__ void __launch_bounds__(256) k_generate(const DevJob* __restrict__ jobs, const DevWave* __restrict__ Wp,
                                                  DevQueues Q) {
  const DevWave W = *Wp;
  const int numPaths = W.numPaths;
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < Q.maxIter * kCountersPerIter; i += blockDim.x) Q.counters[i] = 0;
    __syncthreads();
    if (threadIdx.x == 0) Q.counters[C_RAYS] = numPaths;
  }
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < numPaths; p += gridDim.x * blockDim.x) {
    const DevSegment seg = W.segs[segmentOfPath(W, p)];
    const int local = p - seg.pathBase;
    const int i = local % seg.numPixels, sl = local / seg.numPixels;
    const int pixel = seg.pixelList ? seg.pixelList[seg.pixelOffset + i] : seg.pixelOffset + i;
    const DevJob& J = jobs[seg.slot];
    const DevRender& R = J.R;
    const int x = pixel % R.width, y = pixel / R.width;
    const uint32_t sample = (uint32_t)(J.cnt[pixel] + sl);
    Rng rng;
    rng.init(x, y, R.width, sample, R.seed, dimBaseOf(R));
    V3 o, d;
    primaryRay(R, rng, x, y, o, d);
    const uint32_t medFlag = (uint32_t)(J.S.globalMedium + 1) << F_MED_SHIFT;
    Q.rayO[0][p] = make_float4(o.x, o.y, o.z, __int_as_float(p));
    Q.rayD[0][p] = make_float4(d.x, d.y, d.z, __int_as_float(seg.slot));
    Q.pathT[0][p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    Q.pathR[0][p] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(F_EYE | medFlag));
    Q.pathPS[0][p] = make_int2(pixel, (int)sample);
    Q.pathL[p] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));
  }
}

// Closest hit for the iteration's queue; persistent warps fetch 32 rays at a time.
__global__ void __launch_bounds__(128) k_extend(const DevJob* __restrict__ jobs, DevQueues Q, int iter) {
  const int count = Q.counters[iter * kCountersPerIter + C_RAYS];
  int* fetch = &Q.counters[iter * kCountersPerIter + C_FETCH_EXT];
  const float4* __restrict__ rO = Q.rayO[iter & 1];
  const float4* __restrict__ rD = Q.rayD[iter & 1];
  const int lane = threadIdx.x & 31;
  uint32_t nodes = 0, tris = 0, rays = 0;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(fetch, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= count) break;
    const int q = base + lane;
    if (q < count) {
      const float4 a = rO[q], b = rD[q];
      const DevScene& S = jobs[__float_as_int(b.w)].S;
      const ClosestHit h = traceClosest2(S, xyz(a), xyz(b), nodes, tris);
      Q.hits[q] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
      rays++;
    }
  }
  warpAddStat(&Q.stats[0], nodes);
  warpAddStat(&Q.stats[1], tris);
  warpAddStat(&Q.stats[4], rays);
}

// Shadow-ray visibility; unoccluded contributions are added to the path.
__global__ void __launch_bounds__(128) k_connect(const DevJob* __restrict__ jobs, DevQueues Q, int iter, int which) {
  const int count = Q.counters[iter * kCountersPerIter + shadowCountSlot(which)];
  int* fetch = &Q.counters[iter * kCountersPerIter + shadowFetchSlot(which)];
  const float4* __restrict__ sO = Q.shO[which];
  const float4* __restrict__ sD = Q.shD[which];
  const float4* __restrict__ sC = Q.shC[which];
  const uint32_t occ = shadowOccluder(which);
  const int lane = threadIdx.x & 31;
  uint32_t nodes = 0, tris = 0, rays = 0;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(fetch, 32);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= count) break;
    const int q = base + lane;
    if (q < count) {
      const float4 a = sO[q], b = sD[q];
      const float4 c = sC[q];
      const DevScene& S = jobs[__float_as_int(c.w)].S;
      rays++;
      if (!traceAny2(S, xyz(a), xyz(b), b.w, occ, nodes, tris)) {
        const int pid = __float_as_int(a.w);
        float4 l = Q.pathL[pid];
        l.x += c.x; l.y += c.y; l.z += c.z;
        Q.pathL[pid] = l;
      }
    }
  }
  warpAddStat(&Q.stats[2], nodes);
  warpAddStat(&Q.stats[3], tris);
  warpAddStat(&Q.stats[5], rays);
}

// ---- 8-wide traversal kernels with per-lane ray refill ----------------------
// Persistent warps (Aila & Laine's persistent threads with ray refill, with
// the triangle postponing of Ylitie et al.'s compressed wide BVH traversal):
// * a lane whose ray finished is refilled once enough lanes of its warp are
//   idle (warp ballot + one atomic per warp);
// * every step a lane either intersects one node or tests one triangle; a
//   lane with pending triangles pushes them as a triangle group and keeps
//   descending unless enough lanes of the warp have triangles to test, so the
//   warp runs mostly one kind of step at a time.
// Stack entries: node group (childBase, hits | imask << 8) or triangle group
// (triBase | 0x80000000, triangle mask).
// Refill and triangle-vote thresholds, per traversal kind (closest hit /
// shadow rays); build-time overridable (-D) for sweeps.
#ifndef RG_REFILL_IDLE_CLOSEST
#define RG_REFILL_IDLE_CLOSEST 8
#endif
#ifndef RG_REFILL_IDLE_ANY
#define RG_REFILL_IDLE_ANY 8
#endif
#ifndef RG_TRI_VOTES_CLOSEST
#define RG_TRI_VOTES_CLOSEST 4
#endif
#ifndef RG_TRI_VOTES_ANY
#define RG_TRI_VOTES_ANY 4
#endif
constexpr int kRefillIdle = RG_REFILL_IDLE_CLOSEST;  // refill once this many lanes are idle
#ifndef RG_SHARED_STACK
#define RG_SHARED_STACK 8
#endif
constexpr int kSharedStack = RG_SHARED_STACK;  // traversal stack entries kept in shared memory (the rest in local)
constexpr int kTraceBlock = 128;   // block size of the persistent traversal kernels
constexpr int kTriVotes = RG_TRI_VOTES_CLOSEST;  // lanes with triangles needed to run a triangle step (swept: 2-4 best, 10 -1.6%)

template <bool ANY, bool MULTI>
__device__ __forceinline__ void traverseWave8(const DevScene& S0, const DevJob* __restrict__ jobs, int count, int* fetch, const float4* __restrict__ rO,
                                              const float4* __restrict__ rD, uint32_t occ, float4* __restrict__ hitsOut,
                                              const float4* __restrict__ contrib, float4* __restrict__ pathL,
                                              uint32_t& nodes, uint32_t& tris, uint32_t& rays) {
  const int lane = threadIdx.x & 31;
  const unsigned ltMask = (1u << lane) - 1u;
  int q = -1;  // -1: needs a ray, -2: none left
  V3 o = v3(0, 0, 0), d = v3(0, 0, 1), inv = v3(0, 0, 0);
  uint32_t oct = 0;
  float tmax = 0.0f, hu = 0.0f, hv = 0.0f;
  int prim = -1, pid = 0;
  uint32_t gInner = 0, gImask = 0, tMask = 0;
  int gBase = 0, tBase = 0, sp = 0, steps = 0;
  // traversal stack: entries [0, kSharedStack) in shared memory, entry-major so a
  // warp at one depth touches consecutive words; deeper entries in local memory
  __shared__ uint2 sStack[kSharedStack > 0 ? kSharedStack : 1][kTraceBlock];
  uint2 lStack[kStack8 - kSharedStack];
  auto push = [&](uint2 e) {
    if (sp < kSharedStack) sStack[sp][threadIdx.x] = e;
    else lStack[sp - kSharedStack] = e;
    sp++;
  };
  auto pop = [&]() -> uint2 {
    --sp;
    return sp < kSharedStack ? sStack[sp][threadIdx.x] : lStack[sp - kSharedStack];
  };
  const float4* nodesP = nullptr;
  const float4* trisP = nullptr;
  int numNodes = 0;
  int* errP = nullptr;
  for (;;) {
    // ---- refill idle lanes
    const bool need = q == -1;
    const unsigned needMask = __ballot_sync(0xffffffffu, need);
    if (needMask) {
      const int leader = __ffs(needMask) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(fetch, __popc(needMask));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        const int idx = base + __popc(needMask & ltMask);
        if (idx < count) {
          q = idx;
          const float4 a = rO[q], b = rD[q];
          o = xyz(a);
          d = xyz(b);
          int slot;
          if (ANY) {
            tmax = b.w;
            pid = __float_as_int(a.w);
            slot = __float_as_int(contrib[q].w);
          } else {
            tmax = kMaxRayDistance;
            slot = __float_as_int(b.w);
          }
          if (MULTI) {
            const DevScene& S = jobs[slot].S;
            nodesP = S.nodes8;
            trisP = S.triVerts;
            numNodes = S.numNodes8;
            errP = S.error;
          } else {
            nodesP = S0.nodes8;
            trisP = S0.triVerts;
            numNodes = S0.numNodes8;
            errP = S0.error;
          }
          prim = -1;
          hu = hv = 0.0f;
          inv = safeInv(d);
          oct = rayOctant(inv);
          gBase = 0;
          gImask = 1u;          // the root as a one-child group
          gInner = 1u << oct;   // slot 0 at priority position 0 ^ oct
          tMask = 0;
          sp = 0;
          steps = 0;
          rays++;
        } else {
          q = -2;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, q >= 0) == 0) break;
    // ---- traversal steps until enough lanes are idle
    for (;;) {
      const bool alive = q >= 0;
      int result = 0;  // 1: finished (closest: hit record, any: unoccluded), 2: occluded
      if (alive && tMask == 0 && gInner == 0) {
        if (sp == 0) {
          result = 1;
        } else {
          const uint2 e = pop();
          if (e.x & 0x80000000u) {
            tBase = (int)(e.x & 0x7fffffffu);
            tMask = e.y;
          } else {
            gBase = (int)e.x;
            gInner = e.y & 0xffu;
            gImask = e.y >> 8;
          }
        }
      }
      const bool hasTri = alive && result == 0 && tMask != 0;
      const int triVotes = __popc(__ballot_sync(0xffffffffu, hasTri));
      if (alive && result == 0) {
        const bool doTri = hasTri && (gInner == 0 || triVotes >= (ANY ? RG_TRI_VOTES_ANY : kTriVotes));
        if (doTri) {
          // up to two triangles per step: a triangle step costs about half a node
          // step, so two keep the triangle and node branches of a divergent warp
          // closer in length (swept: 1 / 2 / 3 / 4 per step)
#pragma unroll 1
         for (int rep = 0; rep < 2 && tMask && result == 0; rep++) {
          const int i = __ffs(tMask) - 1;
          tMask &= tMask - 1u;
          const int tk = tBase + i;
          const float4* tp = trisP + (size_t)tk * 3;
          const float4 b = ldTri4(tp + 1);
          if (!ANY || (__float_as_uint(b.w) & occ)) {
            const float4 a = ldTri4(tp), c = ldTri4(tp + 2);
            tris++;
            if (ANY) {
              if (mtAny(o, d, xyz(a), xyz(b), xyz(c), tmax)) result = 2;
            } else {
              ClosestHit h;
              h.t = tmax;
              h.u = hu;
              h.v = hv;
              if (mtClosest(o, d, xyz(a), xyz(b), xyz(c), h)) {
                tmax = h.t;
                hu = h.u;
                hv = h.v;
                prim = tk;
              }
            }
          }
         }
        } else {
          // node step (pending triangles are postponed onto the stack)
          if (hasTri) {
            if (sp < kStack8) push(make_uint2((uint32_t)tBase | 0x80000000u, tMask));
            else atomicCAS(errP, 0, kErrStackOverflow);
            tMask = 0;
          }
          const int pos = 31 - __clz(gInner);
          gInner &= ~(1u << pos);
          const int slot = pos ^ (int)oct;
          const int node = gBase + __popc(gImask & ((1u << slot) - 1u));
          if (gInner) {
            if (sp < kStack8) push(make_uint2((uint32_t)gBase, gInner | (gImask << 8)));
            else atomicCAS(errP, 0, kErrStackOverflow);
          }
          if (node >= numNodes || ++steps > c_traversalStepCap) {
            atomicCAS(errP, 0, kErrTraversalSteps);
            result = ANY ? 2 : 1;
          } else {
            const Node8Hit g = intersectNode8(nodesP + (size_t)node * kNode8Vec, o, inv, tmax, oct);
            nodes++;
            gInner = g.inner;
            gImask = g.imask;
            gBase = g.childBase;
            tMask = g.tris;
            tBase = g.triBase;
            const int nslot = (31 - __clz(gInner)) ^ (int)oct;
            const int nnode = gBase + __popc(gImask & ((1u << nslot) - 1u));
            // closest hit: the node this group visits next into L1 while the warp's other
            // lanes finish their step (for shadow rays it measured slower)
            if (!ANY && gInner && nnode < numNodes) {
              const char* np = reinterpret_cast<const char*>(nodesP + (size_t)nnode * kNode8Vec);
              asm volatile("prefetch.global.L1 [%0];" ::"l"(np));
              asm volatile("prefetch.global.L1 [%0];" ::"l"(np + 128));
              asm volatile("prefetch.global.L1 [%0];" ::"l"(np + 207));
            }
          }
        }
      }
      if (result != 0) {
        if (ANY) {
          if (result == 1) {
            const float4 c = contrib[q];
            float4 l = pathL[pid];
            l.x += c.x;
            l.y += c.y;
            l.z += c.z;
            pathL[pid] = l;
          }
        } else {
          hitsOut[q] = make_float4(tmax, hu, hv, __int_as_float(prim));
        }
        q = -1;
      }
      const unsigned idle = __ballot_sync(0xffffffffu, q == -1);
      const unsigned live = __ballot_sync(0xffffffffu, q >= 0);
      if (live == 0 || __popc(idle) >= (ANY ? RG_REFILL_IDLE_ANY : kRefillIdle)) break;
    }
  }
}

// Resident blocks per SM of the traversal kernels (8: 64 registers), build-time
// overridable (-D) for sweeps.
#ifndef RG_TRACE_MIN_BLOCKS
#define RG_TRACE_MIN_BLOCKS 8
#endif
#ifndef RG_CONNECT_MIN_BLOCKS
#define RG_CONNECT_MIN_BLOCKS RG_TRACE_MIN_BLOCKS
#endif
template <bool MULTI>
__global__ void __launch_bounds__(128, RG_TRACE_MIN_BLOCKS) k_extend8(DevScene S0, const DevJob* __restrict__ jobs, DevQueues Q, int iter) {
  const int count = Q.counters[iter * kCountersPerIter + C_RAYS];
  uint32_t nodes = 0, tris = 0, rays = 0;
  traverseWave8<false, MULTI>(S0, jobs, count, &Q.counters[iter * kCountersPerIter + C_FETCH_EXT], Q.rayO[iter & 1],
                       Q.rayD[iter & 1], 0u, Q.hits, nullptr, nullptr, nodes, tris, rays);
  warpAddStat(&Q.stats[0], nodes);
  warpAddStat(&Q.stats[1], tris);
  warpAddStat(&Q.stats[4], rays);
}

template <bool MULTI>
__global__ void __launch_bounds__(128, RG_CONNECT_MIN_BLOCKS) k_connect8(DevScene S0, const DevJob* __restrict__ jobs, DevQueues Q, int iter,
                                                  int which) {
  const int count = Q.counters[iter * kCountersPerIter + shadowCountSlot(which)];
  uint32_t nodes = 0, tris = 0, rays = 0;
  traverseWave8<true, MULTI>(S0, jobs, count, &Q.counters[iter * kCountersPerIter + shadowFetchSlot(which)],
                      Q.shO[which], Q.shD[which], shadowOccluder(which), nullptr, Q.shC[which], Q.pathL, nodes,
                      tris, rays);
  warpAddStat(&Q.stats[2], nodes);
  warpAddStat(&Q.stats[3], tris);
  warpAddStat(&Q.stats[5], rays);
}

// Shading class of a material: the branch its surface vertices take in the
// shade kernel (emitter, diffuse, rough glossy, mirror, refraction,
// transparency, mixed lobes; 7 = miss), the key of the kernel's sort.
constexpr int kTriMatIndex = (1 << 28) - 1;
__device__ __forceinline__ int materialClass(const DevMaterial& m) {
  const float gl = m.glossy, rf = m.refraction;
  if (m.emission > 0.0f) return 0;
  if (m.transparency > 0.001f) return 5;
  if (gl <= 0.00001f && rf <= 0.00001f) return 1;
  if (rf <= 0.00001f && gl >= 1.0f - 0.00001f) return m.roughness < 1e-3f ? 3 : 2;
  if (gl <= 0.00001f && rf >= 1.0f - 0.00001f) return 4;
  return 6;
}

__global__ void k_triMaterial(DevScene S, int n, int* __restrict__ triMat) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int mesh = __float_as_int(S.triVerts[(size_t)i * 3].w);
  const int mat = S.objMat[S.meshObj[mesh]];
  triMat[i] = (materialClass(S.mats[mat]) << 28) | (mat & kTriMatIndex);
}

void launchTriMaterial(const DevScene& S, int n, int* triMat, cudaStream_t st) {
  k_triMaterial<<<(n + 255) / 256, 256, 0, st>>>(S, n, triMat);
}

// One path vertex (RayBSDFShaderProvider::shade + lobes + tracePath's medium branch).
// MULTI = false: one job whose scene and render constants come in as kernel
// parameters (constant bank); MULTI = true: per-ray job slot into the table.
// ENV = false drops the environment-map code (misses, environment NEE) for
// scenes without one; MEDL selects the participating-medium code: 0 none,
// 1 homogeneous media, 2 procedural media (fBm density with delta tracking,
// cone / path emission, heat haze) and volume-light NEE.  Scenes without
// those features run a smaller kernel (instruction fetch is this kernel's
// main stall).
template <bool MULTI, bool ENV, int MEDL>
__global__ void __launch_bounds__(256) k_shade(DevScene S0, DevRender R0, const DevJob* __restrict__ jobs, DevQueues Q,
                                               int iter) {
  const int count = Q.counters[iter * kCountersPerIter + C_RAYS];
  const int inB = iter & 1, outB = (iter + 1) & 1;
  // Each block iteration takes 512 consecutive queue entries (two per thread)
  // and shades them grouped by the branch their hit takes (a counting sort in
  // shared memory), so that a warp mostly runs one lobe: incoherent bounces
  // otherwise leave a third of the lanes active and the kernel waiting on
  // instruction fetch.  Classes: 0 emitter, 1 diffuse, 2 rough glossy,
  // 3 mirror, 4 refraction, 5 transparency, 6 mixed lobes, 7 miss.  The bins and
  // the order are double buffered by iteration, which leaves three block
  // barriers per iteration.
  constexpr int kBins = 8, kPer = 2, kWin = 256 * kPer;
  __shared__ int sBin[2][kBins];
  __shared__ int sOrder[2][kWin];
  if (threadIdx.x < 2 * kBins) sBin[threadIdx.x / kBins][threadIdx.x % kBins] = 0;
  __syncthreads();
  int buf = 0;
  for (int base = blockIdx.x * kWin; base < count; base += gridDim.x * kWin, buf ^= 1) {
    {
      int key[kPer], rank[kPer];
#pragma unroll
      for (int h = 0; h < kPer; ++h) {
        const int q0 = base + h * 256 + threadIdx.x;
        key[h] = kBins - 1;
        if (q0 < count) {
          const int prim0 = __float_as_int(Q.hits[q0].w);
          if (prim0 >= 0) {
            const DevScene& Sk = MULTI ? jobs[__float_as_int(Q.rayD[inB][q0].w)].S : S0;
            key[h] = __ldg(&Sk.triMat[prim0]) >> 28;
          }
        }
        // sBin[buf] was zeroed, and this buffer's order last read, before the previous
        // iteration's second barrier
        rank[h] = atomicAdd(&sBin[buf][key[h]], 1);
      }
      __syncthreads();
      if (threadIdx.x < 32) {  // exclusive scan of the bins
        const int c = threadIdx.x < kBins ? sBin[buf][threadIdx.x] : 0;
        int incl = c;
#pragma unroll
        for (int o = 1; o < kBins; o <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, incl, o);
          if ((int)threadIdx.x >= o) incl += t;
        }
        if (threadIdx.x < kBins) sBin[buf][threadIdx.x] = incl - c;
      } else if (threadIdx.x < 32 + kBins) {
        sBin[buf ^ 1][threadIdx.x - 32] = 0;  // every thread is past the previous iteration's reads
      }
      __syncthreads();
#pragma unroll
      for (int h = 0; h < kPer; ++h) sOrder[buf][sBin[buf][key[h]] + rank[h]] = base + h * 256 + threadIdx.x;
      __syncthreads();
    }
    for (int h = 0; h < kPer; ++h) {
      const int q = sOrder[buf][threadIdx.x + h * 256];
      const bool valid = q < count;
      Shadow shA, shB, shE, shV;  // area light / point light / environment / volume light
      shA.on = false;
      shB.on = false;
      shE.on = false;
      shV.on = false;
      bool cont = false;
      V3 no = v3(0, 0, 0), nd = v3(0, 0, 0);
      int pid = 0, slot = 0;
      float4 outT = make_float4(0, 0, 0, 0), outR = make_float4(0, 0, 0, 0);  // state of the continuing path
      int2 outPS = make_int2(0, 0);
      if (valid) {
        const float4 ro = Q.rayO[inB][q], rd = Q.rayD[inB][q];
        pid = __float_as_int(ro.w);
        slot = __float_as_int(rd.w);
        const DevScene S = MULTI ? jobs[slot].S : S0;
        const DevRender R = MULTI ? jobs[slot].R : R0;
        const V3 o = xyz(ro), d = xyz(rd);
        const float4 hq = Q.hits[q];
        const int prim = __float_as_int(hq.w);
        const float4 PT = Q.pathT[inB][q], PR = Q.pathR[inB][q], PL = Q.pathL[pid];
        V3 beta = xyz(PT);
        float bsdfPdf = PT.w;
        V3 rrT = xyz(PR);
        uint32_t flags = __float_as_uint(PR.w);
        V3 L = xyz(PL);
        const int vraw = __float_as_int(PL.w);
        const int v = vraw & kVtxMask;
        int vflags = vraw & ~kVtxMask;
        bool eye = (flags & F_EYE) != 0;
        int passes = (int)(flags & F_PASSES_MASK);
        int chroma = (int)((flags & F_CHROMA_MASK) >> F_CHROMA_SHIFT) - 1;
        int med = (int)((flags & F_MED_MASK) >> F_MED_SHIFT) - 1;
        if (eye && prim < 0) vflags |= kVtxEyeNoHit;
        const int2 ps = Q.pathPS[inB][q];
        const int x = ps.x % R.width, y = ps.x / R.width;
        Rng rng;
        rng.init(x, y, R.width, (uint32_t)ps.y, R.seed, dimBaseOf(R));
        bool done = false;
        bool silhouette = false;
        // ---- participating medium on the segment (tracePath, rayrenderer.cpp:1612-1863)
        const bool medActive = MEDL > 0 && med >= 0 && S.media[med].active;
        if (MEDL == 2 && medActive && S.media[med].haze) {
          // heat haze (rayrenderer.cpp:1645-1660): march to the next surface bending
          // the ray, then continue from the bent ray in the outer (global) medium.
          // A heat-haze global medium bends once and the path goes on without a
          // medium (the reference recurses without end there).
          const float maxT = prim >= 0 ? hq.x : kRayMaxDistance;
          const med::Ray6 bent = med::bendRay(S.media + med, o, d, fminf(maxT, 1000.0f));
          const int outer = S.globalMedium;
          med = (outer >= 0 && S.media[outer].haze) ? -1 : outer;
          cont = true;
          no = bent.o;
          nd = bent.d;
        } else if (medActive) {
          const DevMedium* Mg = S.media + med;
          const DevMedium M = *Mg;
          const bool het = MEDL == 2 && M.field != 0;
          const float maxT = prim >= 0 ? hq.x : kRayMaxDistance;
          float tF, dens = 1.0f;
          bool scat;
          if (het) {  // delta tracking (medium.cpp:406-441)
            const med::Collision col = med::deltaTrack(Mg, o, d, maxT, rng, v);
            scat = col.hit;
            tF = col.hit ? col.t : maxT;
            dens = col.density;
          } else {
            tF = sampleFreeFlight(M.hero, rng.prng(v, S_FLIGHT));
            scat = tF < maxT;
          }
          const float el = scat ? tF : maxT;
          if (MEDL == 2) {
            L = L + beta * med::emissionIntegral(&jobs[slot].S, Mg, o, d, el, rng, v);
          } else if (el > 0.0f) {
            auto ew = [](float st, float dd) { return st < 1e-6f ? dd : (1.0f - expf(-st * dd)) / st; };
            L = L + beta * v3(M.ser * ew(M.str, el), M.seg * ew(M.stg, el), M.seb * ew(M.stb, el));
          }
          if (scat) {
            V3 sw = v3(0, 0, 0);
            if (het) {  // sigma_s(p) / sigma_t_max: the rejection walk carries the decay
              const float inv = M.tMaxHero > 0.0f ? 1.0f / M.tMaxHero : 0.0f;
              sw = v3(M.ssr * dens * inv, M.ssg * dens * inv, M.ssb * dens * inv);
            } else {
              const float pHero = M.hero * expf(-M.hero * tF);
              if (pHero > 0.0f)
                sw = v3(M.ssr * expf(-M.str * tF) / pHero, M.ssg * expf(-M.stg * tF) / pHero, M.ssb * expf(-M.stb * tF) / pHero);
            }
            const int passesS = eye ? 1 : passes + 1;
            if ((sw.x == 0.0f && sw.y == 0.0f && sw.z == 0.0f) || passesS > R.maxDepth) {
              done = true;
            } else {
              const V3 pos = o + d * tF;
              const V3 proxy = -d;
              V3 lDir, Le;
              float pl;
              auto phaseTo = [&](V3 w) { return phasePdfHG(-d, w, M.g); };
              if (sampleAreaLightForNEE(S, R, rng, v, pos, proxy, lDir, pl, Le, shA) && pl > 0.0f) {
                shA.on = true;
                shA.c = beta * sw * Le * (phaseTo(lDir) / pl);
              }
              if (ENV && S.envOn) {  // environment NEE at the scatter point (rayrenderer.cpp:1757-1761)
                EnvSample e;
                if (envNEE(&jobs[slot].S, rng, v, pos, proxy, e, shE)) {
                  shE.on = true;
                  shE.c = beta * sw * e.Li * (phaseTo(e.dir) / e.pdf);
                }
              }
              if (MEDL == 2 && S.numVolLights > 0) {  // volume-light NEE (rayrenderer.cpp:1763-1767)
                const med::VolSample vs = med::sampleVolumeLight(&jobs[slot].S, rng, v, pos, proxy);
                if (vs.ok && vs.pdf > 0.0f) {
                  shV.on = true;
                  shV.o = vs.so;
                  shV.d = vs.sd;
                  shV.tmax = 0.99999f;
                  shV.c = beta * sw * vs.Le * (phaseTo(vs.dir) / vs.pdf);
                }
              }
              const V3 ndir = samplePhaseHG(d, M.g, rng.prng(v, S_PHASE0), rng.prng(v, S_PHASE1));
              const V3 rrBase = eye ? v3(1, 1, 1) : rrT;
              float rrW = 1.0f;
              bool killed = false;
              if (passesS >= R.rrDepth) {
                float qq = maxc(rrBase * sw);
                qq = fminf(kRRMax, fmaxf(kRRMin, qq));
                if (rng.prng(v, S_MEDRR) >= qq) killed = true;
                else rrW = 1.0f / qq;
              }
              if (killed) {
                done = true;
              } else {
                beta = beta * sw * rrW;
                rrT = rrBase;
                if (eye) chroma = -1;
                bsdfPdf = 0.0f;
                passes = passesS;
                eye = false;
                cont = true;
                no = pos + normalize(ndir) * kSurfaceThickness;  // ThicknessRay
                nd = ndir;
              }
            }
          } else {
            const float surv = het ? 0.0f : expf(-M.hero * maxT);  // delta tracking: weight 1 (rayrenderer.cpp:1815-1822)
            if (surv > 0.0f)
              beta = beta * v3(expf(-M.str * maxT) / surv, expf(-M.stg * maxT) / surv, expf(-M.stb * maxT) / surv);
            if (prim < 0) {
              if (ENV && S.envOn) L = L + beta * envMiss(&jobs[slot].S, d, bsdfPdf);  // rayrenderer.cpp:1852-1863
              done = true;
            }
            silhouette = true;
          }
        } else if (prim < 0) {
          // environment miss (rayrenderer.cpp:1619-1630; the eye ray has no pdf, so no weight)
          if (ENV && S.envOn) L = L + beta * envMiss(&jobs[slot].S, d, bsdfPdf);
          done = true;
        }
        // ---- surface vertex (RayBSDFShaderProvider::shade, rayrenderer.cpp:2776-2896)
        if (!done && !cont) {
          Hit h = loadHit(S, prim, o, d, hq.x, hq.y, hq.z);
          if (silhouette) {  // rayrenderer.cpp:1842-1846
            const V3 geomN = dot(h.gn, d) <= 0.0f ? h.gn : -h.gn;
            if (dot(d, h.n) > 0.0f && dot(d, geomN) < 0.0f) h.n = geomN;
          }
          const int obj = S.meshObj[h.mesh];
          const DevMaterial m = S.mats[__ldg(&S.triMat[prim]) & kTriMatIndex];
          const V3 gN = dot(h.gn, h.n) >= 0.0f ? h.gn : -h.gn;  // geomNormal, bsdf.cpp:27-30
          const float lf = R.lightFix ? (float)S.numAreaLights : 1.0f;
          int lobe = -1;  // 0 diffuse 1 glossy 2 refraction 3 transparency
          if (m.emission > 0.0f) {
            V3 e = matColor(m) * m.emission;
            if (!eye && bsdfPdf > 0.0f) {
              const float cosL = -dot(d, h.n);
              if (cosL <= 0.0f) e = v3(0, 0, 0);
              else {
                const V3 dv = h.p - o;
                const float r2 = dot(dv, dv);
                const float4 e1 = __ldg(&S.triVerts[(size_t)prim * 3 + 1]), e2 = __ldg(&S.triVerts[(size_t)prim * 3 + 2]);
                const V3 cr = cross(xyz(e1), xyz(e2));
                const float area = 0.5f * sqrtf(dot(cr, cr)) * (float)S.meshTriCount[h.mesh];
                const float pl = r2 / (cosL * area) / lf;
                e = e * (bsdfPdf * bsdfPdf / (bsdfPdf * bsdfPdf + pl * pl));
              }
            }
            L = L + beta * e;
            done = true;
          } else {
            bool backTransparency = false;
            if (dot(d, h.n) > 0.0f) {
              if (m.transparency > 0.001f) {
                if (!eye && passes + 1 <= R.maxDepth) {
                  backTransparency = true;
                  passes = passes + 1;
                  chroma = -1;
                  bsdfPdf = 0.0f;
                  lobe = 3;
                } else {
                  done = true;
                }
              } else if (m.refraction < 0.001f && m.glossy > 0.001f) {
                done = true;
              }
            }
            if (!done && !backTransparency) {
              if (!eye) {
                if (passes + 1 >= R.maxDepth) {  // depth cap: direct light only
                  if (1.0f - m.glossy - m.refraction > 0.00001f) {
                    const V3 col = R.colorSampling ? albedoOf(S, m, h) : v3(0, 0, 0);
                    traceLight(S, R, rng, v, h.p, h.n, beta * col, shA, shB);
                  }
                  done = true;
                } else {
                  passes = passes + 1;
                  if (passes >= R.rrDepth) {
                    float qq = maxc(rrT);
                    qq = fminf(kRRMax, fmaxf(kRRMin, qq));
                    if (rng.prng(v, S_RR) >= qq) done = true;
                    else beta = beta * (1.0f / qq);
                  }
                  if (!done) lobe = m.transparency > 0.001f ? 3 : 4;
                }
              } else {
                passes = 0;
                rrT = v3(1, 1, 1);
                chroma = -1;
                bsdfPdf = 0.0f;
                if (m.transparency > 0.01f) {
                  // mix * (1 - t) + transparency: pick transparency with probability t
                  lobe = rng.prng(v, S_EYETR) < m.transparency ? 3 : 4;
                  if (lobe == 3) beta = beta * (1.0f / m.transparency);
                } else {
                  lobe = 4;
                }
              }
            }
            if (!done && lobe == 4) {  // MixShader (bsdf.cpp:579-610), one lobe selected
              const float wv[3] = {1.0f - m.glossy - m.refraction, m.glossy, m.refraction};
              float sum = 0.0f;
              for (int k = 0; k < 3; k++) if (wv[k] > 0.00001f) sum += wv[k];
              if (sum > 0.0f) {
                const float u = rng.prng(v, S_LOBE) * sum;
                float acc = 0.0f;
                for (int k = 0; k < 3; k++) {
                  if (!(wv[k] > 0.00001f)) continue;
                  lobe = k;
                  acc += wv[k];
                  if (u < acc) break;
                }
                beta = beta * sum;
                rrT = rrT * wv[lobe];
              } else {
                done = true;
              }
            }
            if (!done && lobe == 0) {  // DiffuseShader (bsdf.cpp:54-108)
              const V3 albedo = R.colorSampling ? albedoOf(S, m, h) : v3(1, 1, 1);
              const int d0 = rng.dirDim(v);
              const V3 dir = cosineWeightedDirection(h.n, rng.lds(d0), rng.lds(d0 + 1));
              traceLight(S, R, rng, v, h.p, h.n, beta * albedo, shA, shB);
              bsdfPdf = fmaxf(0.0f, dot(dir, h.n)) * (1.0f / kPi);
              if (ENV && S.envOn) {  // traceEnvmapLight (rayrenderer.cpp:1484-1519)
                EnvSample e;
                if (envNEE(&jobs[slot].S, rng, v, h.p, h.n, e, shE)) {
                  // the MIS partner is this vertex's own sampled-direction pdf, as passed at bsdf.cpp:86-88
                  const float w = bsdfPdf > 0.0f ? e.pdf * e.pdf / (e.pdf * e.pdf + bsdfPdf * bsdfPdf) : 1.0f;
                  shE.on = true;
                  shE.c = beta * albedo * e.Li * (dot(e.dir, h.n) * w / (kPi * e.pdf));
                }
              }
              if (MEDL == 2 && S.numVolLights > 0) {  // volume-light NEE, no MIS (bsdf.cpp:91-101)
                const med::VolSample vs = med::sampleVolumeLight(&jobs[slot].S, rng, v, h.p, h.n);
                const float cosL = vs.ok && vs.pdf > 0.0f ? fmaxf(0.0f, dot(vs.dir, h.n)) : 0.0f;
                if (cosL > 0.0f) {
                  shV.on = true;
                  shV.o = vs.so;
                  shV.d = vs.sd;
                  shV.tmax = 0.99999f;
                  shV.c = beta * albedo * vs.Le * (cosL * (1.0f / kPi) / vs.pdf);
                }
              }
              beta = beta * albedo;
              rrT = rrT * albedo;
              cont = true;
              no = surfaceOrigin(h.p, dir, gN);
              nd = dir;
            } else if (!done && lobe == 1) {  // GlossyShader (bsdf.cpp:173-374)
              V3 albedo = matColor(m);
              if (R.colorSampling && m.texture >= 0) albedo = albedoOf(S, m, h);
              const V3 F0 = m.metallic >= 1.0f ? albedo : (albedo * m.metallic + v3(0.04f, 0.04f, 0.04f) * (1.0f - m.metallic));
              auto schlick = [&](float VdotH) {
                const float a1 = fmaxf(0.0f, 1.0f - VdotH);
                const float a5 = a1 * a1 * a1 * a1 * a1;
                return F0 + (v3(1, 1, 1) - F0) * a5;
              };
              if (m.roughness < 1e-3f) {
                V3 r = reflect(d, h.n);
                if (dot(r, gN) <= 0.0f) r = reflect(d, gN);
                const V3 F = schlick(fmaxf(0.0f, -dot(d, h.n)));
                beta = beta * F;
                rrT = rrT * F;
                bsdfPdf = 0.0f;
                cont = true;
                no = surfaceOrigin(h.p, r, gN);
                nd = r;
              } else {
                V3 t, b;
                buildTangentFrame(h.n, t, b);
                if (fabsf(m.anisoRot) > 0.0f) {
                  float sa, ca;
                  sincosf(m.anisoRot * (kPi / 180.0f), &sa, &ca);
                  const V3 t2 = t * ca + b * sa, b2 = b * ca - t * sa;
                  t = t2;
                  b = b2;
                }
                const float aniso = fmaxf(-0.99f, fminf(0.99f, m.aniso));
                const float r2 = m.roughness * m.roughness;
                const float ax = fmaxf(1e-3f, r2 * (1.0f - aniso));
                const float ay = fmaxf(1e-3f, r2 * (1.0f + aniso));
                const V3 Vw = -d;
                const V3 Vl = v3(dot(Vw, t), dot(Vw, b), dot(Vw, h.n));
                if (Vl.z <= 0.0f) {
                  done = true;
                } else {
                  const float G1v = smithG1(Vl, ax, ay);
                  // evalGlossy (bsdf.cpp:260-280): f*cos_L and the VNDF pdf toward dw
                  auto evalGlossy = [&](V3 dw, V3& fCos, float& pb) {
                    const V3 Ll = v3(dot(dw, t), dot(dw, b), dot(dw, h.n));
                    if (Ll.z <= 0.0f) return false;
                    V3 Hl = Vl + Ll;
                    const float hl2 = dot(Hl, Hl);
                    if (hl2 <= 0.0f) return false;
                    Hl = Hl * (1.0f / sqrtf(hl2));
                    const float VdotH = fmaxf(0.0f, dot(Vl, Hl));
                    if (Hl.z <= 0.0f || VdotH <= 0.0f) return false;
                    const float hx = Hl.x / ax, hy = Hl.y / ay;
                    const float den = hx * hx + hy * hy + Hl.z * Hl.z;
                    const float D = 1.0f / (kPi * ax * ay * den * den);
                    fCos = schlick(VdotH) * (D * G1v * smithG1(Ll, ax, ay) / (4.0f * Vl.z));
                    pb = G1v * D / (4.0f * Vl.z);
                    return true;
                  };
                  // area-light NEE with MIS (bsdf.cpp:271-284)
                  V3 lDir, Le, fCos;
                  float pl, pb;
                  if (sampleAreaLightForNEE(S, R, rng, v, h.p, h.n, lDir, pl, Le, shA) && evalGlossy(lDir, fCos, pb)) {
                    shA.on = true;
                    shA.c = beta * Le * fCos * (pl * pl / (pl * pl + pb * pb) / pl);
                  }
                  // environment NEE with MIS (bsdf.cpp:302-314)
                  if (ENV && S.envOn) {
                    EnvSample e;
                    if (envNEE(&jobs[slot].S, rng, v, h.p, h.n, e, shE) && evalGlossy(e.dir, fCos, pb)) {
                      shE.on = true;
                      shE.c = beta * e.Li * fCos * (e.pdf * e.pdf / (e.pdf * e.pdf + pb * pb) / e.pdf);
                    }
                  }
                  // volume-light NEE, no MIS (bsdf.cpp:316-328)
                  if (MEDL == 2 && S.numVolLights > 0) {
                    const med::VolSample vs = med::sampleVolumeLight(&jobs[slot].S, rng, v, h.p, h.n);
                    if (vs.ok && vs.pdf > 0.0f && evalGlossy(vs.dir, fCos, pb)) {
                      shV.on = true;
                      shV.o = vs.so;
                      shV.d = vs.sd;
                      shV.tmax = 0.99999f;
                      shV.c = beta * vs.Le * fCos * (1.0f / vs.pdf);
                    }
                  }
                  // VNDF sample (bsdf.cpp:139-161, 319-373)
                  const float u1 = rng.prng(v, S_VNDF0), u2 = rng.prng(v, S_VNDF1);
                  const V3 H = sampleGGXVNDF(Vl, ax, ay, u1, u2);
                  const V3 Ll = H * (2.0f * dot(Vl, H)) - Vl;
                  if (Ll.z <= 0.0f) {
                    done = true;
                  } else {
                    const V3 Lw = t * Ll.x + b * Ll.y + h.n * Ll.z;
                    if (dot(Lw, gN) <= 0.0f) {
                      done = true;
                    } else {
                      const V3 F = schlick(fmaxf(0.0f, dot(Vl, H)));
                      const V3 wgt = F * smithG1(Ll, ax, ay);
                      const float hx = H.x / ax, hy = H.y / ay;
                      const float den = hx * hx + hy * hy + H.z * H.z;
                      const float D = 1.0f / (kPi * ax * ay * den * den);
                      bsdfPdf = G1v * D / (4.0f * Vl.z);
                      beta = beta * wgt;
                      rrT = rrT * wgt;
                      cont = true;
                      no = surfaceOrigin(h.p, Lw, gN);
                      nd = Lw;
                    }
                  }
                }
              }
            } else if (!done && lobe == 2) {  // RefractionShader (bsdf.cpp:376-483)
              const float cosTheta = fabsf(dot(d, h.n));
              float ior = m.ior;
              V3 mask = v3(1, 1, 1);
              if (m.chroma > 0.0f) {
                bool first = false;
                if (chroma < 0) {
                  chroma = (int)fminf(2.0f, floorf(rng.prng(v, S_CHROMA) * 3.0f));
                  first = true;
                }
                if (chroma == 0) ior = m.ior * (1.0f - m.chroma);
                else if (chroma == 2) ior = m.ior * (1.0f + m.chroma);
                if (first) mask = chroma == 0 ? v3(3, 0, 0) : (chroma == 1 ? v3(0, 3, 0) : v3(0, 0, 3));
              }
              const float F = fresnelSchlick(cosTheta, ior);
              const bool pickReflect = rng.prng(v, S_FRESNEL) < F;
              V3 dir = pickReflect ? reflect(d, h.n) : refractDir(d, h.n, ior);
              if (m.roughness > 0.0f)
                dir = normalize(dir + randomRayInHemisphere(h.n, rng.prng(v, S_HEMI0), rng.prng(v, S_HEMI1)) * m.roughness);
              if (pickReflect && dot(dir, gN) <= 0.0f) dir = reflect(d, gN);
              const float dIn = dot(d, h.n), dOut = dot(dir, h.n);
              if (dIn * dOut > 0.0f) {
                if (dIn < 0.0f) { const int im = S.objMedium[obj]; if (im >= 0) med = im; }
                else med = S.globalMedium;
              }
              const V3 col = matColor(m);
              beta = beta * col * mask;
              rrT = rrT * col;
              bsdfPdf = 0.0f;
              cont = true;
              no = surfaceOrigin(h.p, dir, gN);
              nd = dir;
            } else if (!done && lobe == 3) {  // TransparencyShader (bsdf.cpp:513-546)
              const float tr = m.transparency;
              beta = beta * tr;
              rrT = rrT * tr;
              if (dot(d, h.n) < 0.0f) { const int im = S.objMedium[obj]; if (im >= 0) med = im; }
              else med = S.globalMedium;
              cont = true;
              no = surfaceOrigin(h.p, d, gN);
              nd = d;
            }
            if (!done && cont) eye = false;
          }
        }
        // write back the path state
        flags = (flags & ~(F_PASSES_MASK | F_CHROMA_MASK | F_MED_MASK | F_EYE)) | ((uint32_t)passes & F_PASSES_MASK) |
                ((uint32_t)(chroma + 1) << F_CHROMA_SHIFT) | ((uint32_t)(med + 1) << F_MED_SHIFT) | (eye ? F_EYE : 0u);
        outT = make_float4(beta.x, beta.y, beta.z, bsdfPdf);
        outR = make_float4(rrT.x, rrT.y, rrT.z, __uint_as_float(flags));
        outPS = ps;
        Q.pathL[pid] = make_float4(L.x, L.y, L.z, __int_as_float(((v + 1) & kVtxMask) | vflags));
        if (!cont) {
          no = v3(0, 0, 0);
        }
      }
      // queue pushes (warp-aggregated); the path state goes with the next ray
      const int qslot = warpPush(&Q.counters[(iter + 1) * kCountersPerIter + C_RAYS], cont && (iter + 1) < Q.maxIter);
      if (qslot >= 0) {
        Q.rayO[outB][qslot] = make_float4(no.x, no.y, no.z, __int_as_float(pid));
        Q.rayD[outB][qslot] = make_float4(nd.x, nd.y, nd.z, __int_as_float(slot));
        Q.pathT[outB][qslot] = outT;
        Q.pathR[outB][qslot] = outR;
        Q.pathPS[outB][qslot] = outPS;
      }
      const int sa = warpPush(&Q.counters[iter * kCountersPerIter + C_SHA], shA.on);
      if (sa >= 0) {
        Q.shO[0][sa] = make_float4(shA.o.x, shA.o.y, shA.o.z, __int_as_float(pid));
        Q.shD[0][sa] = make_float4(shA.d.x, shA.d.y, shA.d.z, shA.tmax);
        Q.shC[0][sa] = make_float4(shA.c.x, shA.c.y, shA.c.z, __int_as_float(slot));
      }
      const int sb = warpPush(&Q.counters[iter * kCountersPerIter + C_SHB], shB.on);
      if (sb >= 0) {
        Q.shO[1][sb] = make_float4(shB.o.x, shB.o.y, shB.o.z, __int_as_float(pid));
        Q.shD[1][sb] = make_float4(shB.d.x, shB.d.y, shB.d.z, shB.tmax);
        Q.shC[1][sb] = make_float4(shB.c.x, shB.c.y, shB.c.z, __int_as_float(slot));
      }
      if (ENV) {
        const int se = warpPush(&Q.counters[iter * kCountersPerIter + C_SHC], shE.on);
        if (se >= 0) {
          Q.shO[2][se] = make_float4(shE.o.x, shE.o.y, shE.o.z, __int_as_float(pid));
          Q.shD[2][se] = make_float4(shE.d.x, shE.d.y, shE.d.z, shE.tmax);
          Q.shC[2][se] = make_float4(shE.c.x, shE.c.y, shE.c.z, __int_as_float(slot));
        }
      }
      if (MEDL == 2) {
        const int sv = warpPush(&Q.counters[iter * kCountersPerIter + C_SHD], shV.on);
        if (sv >= 0) {
          Q.shO[3][sv] = make_float4(shV.o.x, shV.o.y, shV.o.z, __int_as_float(pid));
          Q.shD[3][sv] = make_float4(shV.d.x, shV.d.y, shV.d.z, shV.tmax);
          Q.shC[3][sv] = make_float4(shV.c.x, shV.c.y, shV.c.z, __int_as_float(slot));
        }
      }
    }
  }
}

// ---- shader ids 0-3 (one thread per path; rayrenderer.h:456-474, lambert.cpp:14-65)
__device__ float calcAO(const DevScene& S, const DevRender& R, const Rng& rng, int v, V3 hit, V3 n, float dist,
                        uint32_t& nodes, uint32_t& tris) {
  float sum = 0.0f;
  const int N = R.aoSamples;
  for (int i = 0; i < N; i++) {
    const int d0 = rng.dimBase + 4 * v + 4 + 2 * i;
    const V3 dir = cosineWeightedDirection(n, rng.lds(d0), rng.lds(d0 + 1));
    const V3 o = hit + normalize(dir) * kSurfaceThickness;
    if (!traceAny(S, o, dir, dist, kOccAO, nodes, tris)) sum += fmaxf(dot(dir, n), 0.0f);
  }
  return sum / (float)N;
}

__device__ V3 lambertLights(const DevScene& S, const DevRender& R, const Rng& rng, int v, V3 hit, V3 n,
                            uint32_t& nodes, uint32_t& tris) {
  V3 acc = v3(0, 0, 0);
  Shadow a;
  a.on = false;
  traceAreaLight(S, R, rng, v, hit, n, v3(1, 1, 1), a);
  if (a.on && !traceAny(S, a.o, a.d, a.tmax, kOccArea, nodes, tris)) acc = acc + a.c;
  for (int i = 0; i < S.numPointLights; i++) {
    Shadow b;
    b.on = false;
    tracePointLight(S, i, hit, n, v3(1, 1, 1), b);
    if (b.on && !traceAny(S, b.o, b.d, b.tmax, kOccPoint, nodes, tris)) acc = acc + b.c;
  }
  return acc + v3(R.worldR, R.worldG, R.worldB);
}

__global__ void __launch_bounds__(128) k_simple(const DevJob* __restrict__ jobs, const DevWave* __restrict__ Wp,
                                                DevQueues Q) {
  const DevWave W = *Wp;
  const int numPaths = W.numPaths;
  uint32_t nodes = 0, tris = 0;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < numPaths; p += gridDim.x * blockDim.x) {
    const DevSegment seg = W.segs[segmentOfPath(W, p)];
    const int local = p - seg.pathBase;
    const int li = local % seg.numPixels, sl = local / seg.numPixels;
    const int pixel = seg.pixelList ? seg.pixelList[seg.pixelOffset + li] : seg.pixelOffset + li;
    const DevScene& S = jobs[seg.slot].S;
    const DevRender& R = jobs[seg.slot].R;
    const int x = pixel % R.width, y = pixel / R.width;
    const uint32_t sample = (uint32_t)(jobs[seg.slot].cnt[pixel] + sl);
    Rng rng;
    rng.init(x, y, R.width, sample, R.seed, dimBaseOf(R));
    V3 o, d;
    primaryRay(R, rng, x, y, o, d);
    // tracePath through transparent surfaces, accumulating (color, weight)
    V3 total = v3(0, 0, 0), w = v3(1, 1, 1);
    bool eyeHit = false;
    for (int depth = 0, v = 0; depth < R.maxDepth; depth++, v++) {
      const ClosestHit ch = traceClosest(S, o, d, nodes, tris);
      if (ch.prim < 0) {
        // traceEyeRay's miss and tracePath's miss without BSDF parameters (rayrenderer.cpp:1292, 1619)
        if (S.envOn) total = total + w * envRadiance(&S, d);
        break;
      }
      if (depth == 0) eyeHit = true;
      const Hit h = loadHit(S, ch.prim, o, d, ch.t, ch.u, ch.v);
      const DevMaterial m = S.mats[S.objMat[S.meshObj[h.mesh]]];
      if (R.shader == 0) {
        const V3 Ld = normalize(v3(1, 1, 1));
        const float c = 0.1f + fmaxf(dot(Ld, h.n), 0.0f);
        total = total + w * c;
        break;
      }
      if (R.shader == 1) {
        const float a = fminf(fmaxf(calcAO(S, R, rng, v, h.p, h.n, kRayMaxDistance, nodes, tris), 0.0f), 1.0f);
        total = total + w * a;
        break;
      }
      if (m.emission > 0.0f) {
        total = total + w * matColor(m) * m.emission;
        break;
      }
      const V3 light = lambertLights(S, R, rng, v, h.p, h.n, nodes, tris) * 0.3f;
      V3 col;
      float through = 0.0f;
      if (R.shader == 2) {
        col = light;
        if (R.colorSampling) col = col * albedoOf(S, m, h);
        if (m.transparency > 0.0f) {
          col = matColor(m) * (light + v3(0.5f, 0.5f, 0.5f)) * (1.0f - m.transparency);
          through = m.transparency;
        }
      } else {
        col = light * 0.2f + light * 0.8f * calcAO(S, R, rng, v, h.p, h.n, 2.0f, nodes, tris);
        if (R.colorSampling) col = col * albedoOf(S, m, h);
        if (m.transparency > 0.0f) through = m.transparency;
      }
      total = total + w * col;
      if (through <= 0.0f || depth + 1 >= R.maxDepth) break;
      w = w * through;
      o = h.p + normalize(d) * kSurfaceThickness;  // ThicknessRay(hit, inray.dir)
    }
    Q.pathL[p] = make_float4(total.x, total.y, total.z, __int_as_float(eyeHit ? 0 : kVtxEyeNoHit));
  }
  warpAddStat(&Q.stats[0], nodes);
  warpAddStat(&Q.stats[1], tris);
}

// Per-sample clamp and accumulation into the pixel sums (rayrenderer.cpp:936-951).
__global__ void __launch_bounds__(256) k_accumulate(const DevJob* __restrict__ jobs, const DevWave* __restrict__ Wp,
                                                    DevQueues Q) {
  const DevWave W = *Wp;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < W.numPixelsTotal; t += gridDim.x * blockDim.x) {
    const DevSegment seg = W.segs[segmentOfPixel(W, t)];
    const int i = t - seg.pixBase;
    const int pixel = seg.pixelList ? seg.pixelList[seg.pixelOffset + i] : seg.pixelOffset + i;
    const DevJob& J = jobs[seg.slot];
    const DevRender& R = J.R;
    float sr = 0, sg = 0, sb = 0, qr = 0, qg = 0, qb = 0;
    for (int s = 0; s < seg.samples; s++) {
      const int p = seg.pathBase + s * seg.numPixels + i;
      const float4 l = Q.pathL[p];
      const bool noHit = (__float_as_int(l.w) & kVtxEyeNoHit) != 0;
      float r = l.x, g = l.y, b = l.z;
      if (noHit && r == 0.0f && g == 0.0f && b == 0.0f) { r = R.backR; g = R.backG; b = R.backB; }
      r = fmaxf(r, 0.0f); g = fmaxf(g, 0.0f); b = fmaxf(b, 0.0f);
      if (R.clampMax > 0.0f) { r = fminf(r, R.clampMax); g = fminf(g, R.clampMax); b = fminf(b, R.clampMax); }
      sr += r; sg += g; sb += b;
      qr += r * r; qg += g * g; qb += b * b;
    }
    float4 a = J.sum[pixel], c = J.sumSq[pixel];
    a.x += sr; a.y += sg; a.z += sb;
    c.x += qr; c.y += qg; c.z += qb;
    J.sum[pixel] = a;
    J.sumSq[pixel] = c;
    J.cnt[pixel] += seg.samples;
  }
}

// AOV guides from the pixel-centre primary ray (rayrenderer.cpp:819-844).
__global__ void k_aov(DevScene S, DevRender R, __half* __restrict__ normal, __half* __restrict__ albedo,
                      __half* __restrict__ albedoA, __half* __restrict__ depth) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= R.width * R.height) return;
  const int x = i % R.width, y = i / R.width;
  const float dx = ((float)x + 0.5f - R.halfW) * R.viewScale;
  const float dy = -((float)y + 0.5f - R.halfH) * R.viewScale;
  const V3 d = normalize(v3(dx, dy, -1.0f));
  uint32_t nodes = 0, tris = 0;
  const ClosestHit ch = traceClosest(S, v3(0, 0, 0), d, nodes, tris);
  if (ch.prim >= 0) {
    const Hit h = loadHit(S, ch.prim, v3(0, 0, 0), d, ch.t, ch.u, ch.v);
    const DevMaterial m = S.mats[S.objMat[S.meshObj[h.mesh]]];
    normal[i * 3] = __float2half(h.n.x * 0.5f + 0.5f);
    normal[i * 3 + 1] = __float2half(h.n.y * 0.5f + 0.5f);
    normal[i * 3 + 2] = __float2half(h.n.z * 0.5f + 0.5f);
    albedo[i * 3] = __float2half(m.cr);
    albedo[i * 3 + 1] = __float2half(m.cg);
    albedo[i * 3 + 2] = __float2half(m.cb);
    albedoA[i] = __float2half(1.0f);
    float dd = sqrtf(sqrtf(dot(h.p, h.p)) / R.viewFar);
    depth[i] = __float2half(1.0f - fminf(fmaxf(dd, 0.0f), 1.0f));
  } else {
    normal[i * 3] = normal[i * 3 + 1] = normal[i * 3 + 2] = __float2half(0.5f);
    albedo[i * 3] = __float2half(R.backR);
    albedo[i * 3 + 1] = __float2half(R.backG);
    albedo[i * 3 + 2] = __float2half(R.backB);
    albedoA[i] = __float2half(0.0f);
    depth[i] = __float2half(0.0f);
  }
}

// Ray-batch queries (parity API).
__global__ void k_queryClosest(DevScene S, const float* __restrict__ rays, int n, float* __restrict__ tuv,
                               int* __restrict__ prim) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t nodes = 0, tris = 0;
  const V3 o = v3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]);
  const V3 d = v3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
  const ClosestHit h = traceClosest(S, o, d, nodes, tris);
  tuv[i * 3] = h.t;
  tuv[i * 3 + 1] = h.u;
  tuv[i * 3 + 2] = h.v;
  prim[i] = h.prim >= 0 ? S.triOrig[h.prim] : -1;
}

__global__ void k_queryAny(DevScene S, const float* __restrict__ rays, const float* __restrict__ tmax, int n,
                           uint32_t occ, uint8_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t nodes = 0, tris = 0;
  const V3 o = v3(rays[i * 6], rays[i * 6 + 1], rays[i * 6 + 2]);
  const V3 d = v3(rays[i * 6 + 3], rays[i * 6 + 4], rays[i * 6 + 5]);
  out[i] = traceAny(S, o, d, tmax[i], occ, nodes, tris) ? 1 : 0;
}

// Medium field queries (rg_medium_eval / rg_medium_bend).  The scene copy
// sits in the job table so the field functions read it from global memory.
__global__ void k_mediumEval(const DevJob* __restrict__ jobs, int medium, const float* __restrict__ pts, int n,
                             float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevScene* S = &jobs[0].S;
  const DevMedium* M = S->media + medium;
  const V3 p = v3(pts[i * 3], pts[i * 3 + 1], pts[i * 3 + 2]);
  const V3 e = med::emissionAt(S, M, p);
  out[i * 5 + 0] = med::densityAt(M, p);
  out[i * 5 + 1] = e.x;
  out[i * 5 + 2] = e.y;
  out[i * 5 + 3] = e.z;
  out[i * 5 + 4] = med::iorAt(M, p.x, p.y, p.z);
}

__global__ void k_mediumBend(const DevJob* __restrict__ jobs, int medium, const float* __restrict__ rays, int n,
                             float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DevMedium* M = jobs[0].S.media + medium;
  const float* r = rays + (size_t)i * 7;
  const med::Ray6 b = med::bendRay(M, v3(r[0], r[1], r[2]), v3(r[3], r[4], r[5]), r[6]);
  out[i * 6 + 0] = b.o.x;
  out[i * 6 + 1] = b.o.y;
  out[i * 6 + 2] = b.o.z;
  out[i * 6 + 3] = b.d.x;
  out[i * 6 + 4] = b.d.y;
  out[i * 6 + 5] = b.d.z;
}

// ------------------------------------------------------------ launchers ----
// Resident blocks per SM for the persistent traversal kernels.
int residentBlocks(int kernel, int width) {
  int perSM = 0;
  if (kernel == 0) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, width == 8 ? (const void*)k_extend8<true> : (const void*)k_extend, 128, 0);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, width == 8 ? (const void*)k_connect8<true> : (const void*)k_connect, 128, 0);
  return perSM < 1 ? 1 : perSM;
}

void launchGenerate(const DevJob* jobs, const DevWave* W, const DevQueues& Q, int grid, cudaStream_t st) {
  k_generate<<<grid, 256, 0, st>>>(jobs, W, Q);
}
void launchExtend(const DevScene* single, const DevJob* jobs, int width, const DevQueues& Q, int iter, int grid,
                  cudaStream_t st) {
  if (width == 8) {
    if (single) k_extend8<false><<<grid, kTraceBlock, 0, st>>>(*single, jobs, Q, iter);
    else k_extend8<true><<<grid, kTraceBlock, 0, st>>>(DevScene{}, jobs, Q, iter);
  } else {
    k_extend<<<grid, 128, 0, st>>>(jobs, Q, iter);
  }
}
void launchShade(const DevScene* single, const DevRender* singleR, const DevJob* jobs, const DevQueues& Q, int iter,
                 int grid, cudaStream_t st, int multiMediaLevel) {
  if (!single) {
    if (multiMediaLevel >= 2) k_shade<true, true, 2><<<grid, 256, 0, st>>>(DevScene{}, DevRender{}, jobs, Q, iter);
    else k_shade<true, true, 1><<<grid, 256, 0, st>>>(DevScene{}, DevRender{}, jobs, Q, iter);
    return;
  }
  const bool env = single->envOn != 0;
  const int ml = single->mediaLevel;
  if (!env) {
    if (ml == 0) k_shade<false, false, 0><<<grid, 256, 0, st>>>(*single, *singleR, jobs, Q, iter);
    else if (ml == 1) k_shade<false, false, 1><<<grid, 256, 0, st>>>(*single, *singleR, jobs, Q, iter);
    else k_shade<false, false, 2><<<grid, 256, 0, st>>>(*single, *singleR, jobs, Q, iter);
  } else {
    if (ml == 0) k_shade<false, true, 0><<<grid, 256, 0, st>>>(*single, *singleR, jobs, Q, iter);
    else if (ml == 1) k_shade<false, true, 1><<<grid, 256, 0, st>>>(*single, *singleR, jobs, Q, iter);
    else k_shade<false, true, 2><<<grid, 256, 0, st>>>(*single, *singleR, jobs, Q, iter);
  }
}
void launchConnect(const DevScene* single, const DevJob* jobs, int width, const DevQueues& Q, int iter, int which,
                   int grid, cudaStream_t st) {
  if (width == 8) {
    if (single) k_connect8<false><<<grid, kTraceBlock, 0, st>>>(*single, jobs, Q, iter, which);
    else k_connect8<true><<<grid, kTraceBlock, 0, st>>>(DevScene{}, jobs, Q, iter, which);
  } else {
    k_connect<<<grid, 128, 0, st>>>(jobs, Q, iter, which);
  }
}
void launchSimple(const DevJob* jobs, const DevWave* W, const DevQueues& Q, int grid, cudaStream_t st) {
  k_simple<<<grid, 128, 0, st>>>(jobs, W, Q);
}
void launchAccumulate(const DevJob* jobs, const DevWave* W, const DevQueues& Q, int grid, cudaStream_t st) {
  k_accumulate<<<grid, 256, 0, st>>>(jobs, W, Q);
}
void launchAov(const DevScene& S, const DevRender& R, __half* normal, __half* albedo, __half* albedoA, __half* depth,
               cudaStream_t st) {
  const int n = R.width * R.height;
  k_aov<<<(n + 127) / 128, 128, 0, st>>>(S, R, normal, albedo, albedoA, depth);
}
// Sampling-helper probes: each row runs one of the device functions the shade
// kernel uses, on the row's inputs (layouts in rg_probe_sampling's header).
__global__ void k_probeSampling(int which, const float* __restrict__ in, int n, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto put3 = [&](float* o, V3 v) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
  };
  auto rngOf = [&](const float* a) {
    Rng r;
    r.init((uint32_t)a[0], (uint32_t)a[1], 1u << 16, (uint32_t)a[2], 1u, 0);
    return r;
  };
  switch (which) {
    case 0: {
      const float* a = in + (size_t)i * 7;
      put3(out + (size_t)i * 3, sampleGGXVNDF(v3(a[0], a[1], a[2]), a[3], a[4], a[5], a[6]));
      break;
    }
    case 1: {
      const float* a = in + (size_t)i * 5;
      out[i] = smithG1(v3(a[0], a[1], a[2]), a[3], a[4]);
      break;
    }
    case 2:
      out[i] = fresnelSchlick(in[i * 2], in[i * 2 + 1]);
      break;
    case 3: {
      const float* a = in + (size_t)i * 7;
      put3(out + (size_t)i * 3, refractDir(v3(a[0], a[1], a[2]), v3(a[3], a[4], a[5]), a[6]));
      break;
    }
    case 4: {
      const float* a = in + (size_t)i * 3;
      V3 t, b;
      buildTangentFrame(v3(a[0], a[1], a[2]), t, b);
      put3(out + (size_t)i * 6, t);
      put3(out + (size_t)i * 6 + 3, b);
      break;
    }
    case 5: {
      const float* a = in + (size_t)i * 7;
      const Rng r = rngOf(a);
      const int dim = (int)a[3];
      put3(out + (size_t)i * 3, cosineWeightedDirection(v3(a[4], a[5], a[6]), r.lds(dim), r.lds(dim + 1)));
      break;
    }
    case 6: {
      const float* a = in + (size_t)i * 13;
      const Rng r = rngOf(a);
      const int dim = (int)a[3];
      put3(out + (size_t)i * 3, ldsPointInTriangle(v3(a[4], a[5], a[6]), v3(a[7], a[8], a[9]), v3(a[10], a[11], a[12]),
                                                  r.lds(dim), r.lds(dim + 1)));
      break;
    }
    case 7: {
      const float* a = in + (size_t)i * 4;
      out[i] = rngOf(a).lds((int)a[3]);
      break;
    }
    case 8: {
      const float* a = in + (size_t)i * 6;
      put3(out + (size_t)i * 3, samplePhaseHG(v3(a[0], a[1], a[2]), a[3], a[4], a[5]));
      break;
    }
    case 9: {
      const float* a = in + (size_t)i * 7;
      out[i] = phasePdfHG(v3(a[0], a[1], a[2]), v3(a[3], a[4], a[5]), a[6]);
      break;
    }
    case 10:
      out[i] = sampleFreeFlight(in[i * 2], in[i * 2 + 1]);
      break;
    default:
      break;
  }
}

bool setTraversalStepCap(int cap) {
  const int v = cap > 0 ? cap : kMaxTraversalSteps;
  return cudaMemcpyToSymbol(c_traversalStepCap, &v, sizeof(v)) == cudaSuccess;
}

void launchProbeSampling(int which, const float* in, int n, float* out, cudaStream_t st) {
  k_probeSampling<<<(n + 127) / 128, 128, 0, st>>>(which, in, n, out);
}

void launchQueryClosest(const DevScene& S, const float* rays, int n, float* tuv, int* prim, cudaStream_t st) {
  if (n > 0) k_queryClosest<<<(n + 127) / 128, 128, 0, st>>>(S, rays, n, tuv, prim);
}
void launchQueryAny(const DevScene& S, const float* rays, const float* tmax, int n, uint32_t occ, uint8_t* out,
                    cudaStream_t st) {
  if (n > 0) k_queryAny<<<(n + 127) / 128, 128, 0, st>>>(S, rays, tmax, n, occ, out);
}
void launchMediumQuery(const DevJob* jobs, int medium, bool bend, const float* in, int n, float* out, cudaStream_t st) {
  if (n <= 0) return;
  if (bend) k_mediumBend<<<(n + 127) / 128, 128, 0, st>>>(jobs, medium, in, n, out);
  else k_mediumEval<<<(n + 127) / 128, 128, 0, st>>>(jobs, medium, in, n, out);
}

}  // namespace rg
