// rg_device.cuh - device data layout, vector math and the counter-based RNG
// of the B200 wavefront tracer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace rg {

// ------------------------------------------------------------ constants ----
constexpr float kPi = 3.14159265358979323846f;
constexpr float kSurfaceThickness = 0.0001f;  // SURFACE_THICKNESS, raycommon.h:21
constexpr float kMaxRayDistance = 1.0e6f;     // MAX_RAY_DISTANCE, raycommon.h:34
constexpr float kRayMaxDistance = 100.0f;     // RAY_MAX_DISTANCE, rayrenderer.h:48
constexpr float kRRMin = 0.05f, kRRMax = 0.95f;  // rayrenderer.cpp:44-45
constexpr int kMaxLeaf = 8;                   // triangles per leaf in the device BVH
constexpr int kMaxMediumCount = 64;           // cap on a medium's octaves, strata and march steps
constexpr int kStackSize = 64;
// 8-wide BVH node: a header float4 (child base, triangle base, 8 meta bytes) and the
// float planes of the 8 child boxes, per axis 8 lo then 8 hi values (12 float4);
// the node stride in float4 is build-time overridable (-D) for sweeps (>= 13)
#ifndef RG_NODE8_VEC
#define RG_NODE8_VEC 13
#endif
constexpr int kNode8Vec = RG_NODE8_VEC;
static_assert(kNode8Vec >= 13, "an 8-wide node holds 13 float4");

// occluder classes (bit per shadow-ray predicate)
constexpr uint32_t kOccArea = 1u;   // transparency < 0.01 && emission <= 0   (rayrenderer.cpp:1956-1959)
constexpr uint32_t kOccPoint = 2u;  // emission <= 0 && (transparency < 0.01 || refraction > 0.1) (:2211-2215)
constexpr uint32_t kOccAO = 4u;     // transparency < 0.01                    (:2388-2390)
constexpr uint32_t kOccAll = 8u;
constexpr uint32_t kOccVol = 16u;   // emission <= 0 && transparency < 0.01 && refraction <= 0.1 (:2167-2171)

// -------------------------------------------------------------- structs ----
struct DevMaterial {
  float cr, cg, cb;
  float glossy, roughness, transparency, refraction, ior;
  float chroma, metallic, aniso, anisoRot;
  float emission, spotRange;
  int texture;
  float tileU, tileV;
  float pad;
};

// A participating medium in camera space (HomogeneousMedium after prepare()
// and bake(), medium.cpp:18-101).  The first twelve words are all the
// homogeneous branch reads.
struct DevMedium {
  float ssr, ssg, ssb;   // sigma_s * density
  float ser, seg, seb;   // sigma_e * density
  float str, stg, stb;   // sigma_t
  float hero, g;
  int active;            // isActive(), medium.h:226-234
  int mode;              // emission mode: 0 constant, 1 cone, 2 path
  int field;             // density field: 0 none, 1 fBm
  int haze;              // isHeatHaze(), medium.h:240-242
  int hazeOn;            // the heatHaze switch alone (iorAt's test)
  float tMaxHero;        // sigma_t_max_hero: delta-tracking majorant
  float densityScale;    // max(0, density)
  // cone (coneOriginR / coneAxisR: camera space)
  float cox, coy, coz, cax, cay, caz;
  float coneLength, coneRadius;
  float cir, cig, cib, cor, cog, cob;
  float coneIntensity, conePeakAxial, conePeakSharpness;
  int coneSamples;
  // path tube (points in DevScene::pathPts, camera space)
  int pathFirst, pathCount;
  float pir, pig, pib, por, pog, pob;
  float pathIntensity, pathFalloff;
  int pathSamples;
  // fBm density
  float nFreq;
  int nOct;
  float nGain, nLac, nAmp, nBias, nox, noy, noz;
  // heat haze
  float iAmp, iFreq;
  int iOct;
  float iGain, iLac;
  int iSteps;
  float iox, ioy, ioz, iFalloff;
};

// A path-tube control point: (p.xyz, radius) and (t, 0, 0, 0).
struct DevPathPoint {
  float4 pr;
  float4 t;
};

// An emissive volume sampled by volume-light NEE (EmissiveVolumeSource,
// rayrenderer.cpp:180-206): its medium and, for constant-mode media, the
// owning object's location in camera space.
struct DevVolLight {
  int medium;
  float ax, ay, az;
};

struct DevPointLight {
  float px, py, pz;      // view space
  float nx, ny, nz;
  int material;
  int pad;
};

struct DevTexture {
  const float4* texels;
  int width, height, isHdr, pad;
};

// Everything the kernels read about the scene.  Triangle arrays are in BVH
// leaf order; `triOrig` maps back to the DFS triangle id.
struct DevScene {
  const float4* nodes;        // 4 float4 per BVH2 node (two child boxes + refs)
  int numNodes;
  int rootIsLeaf;             // whole scene in one leaf: rootLeafRef holds it
  int rootLeafRef;
  const float4* triVerts;     // 3 float4 per triangle: (v1, mesh bits) (e1, occluder bits) (e2, 0)
  const float4* triShade;     // 3 float4: (n1.xyz, n2.x) (n2.yz, n3.xy) (n3.z, gn.xyz)
  const float2* triUV;        // 3 float2 per triangle (NULL when the scene has no textures)
  const int* triOrig;
  const int* triMat;          // per triangle (leaf order): shading class << 28 | material index
  int numTris;
  const int* meshObj;         // mesh -> object
  const int* meshTriCount;    // mesh -> triangle count (areaLightSampledArea)
  const int* objMat;          // object -> material
  const int* objMedium;       // object -> interior medium (-1 none)
  const DevMaterial* mats;
  const DevMedium* media;
  int numMedia;
  int globalMedium;
  int numAreaLights;
  const int* areaLightObj;    // area light -> object
  const int2* lightObjMeshes; // object -> (first, count) in lightMeshList (light objects only)
  const int* lightMeshList;   // flattened mesh ids
  const int2* lightMeshTris;  // mesh -> (first, count) in lightTris (light meshes only)
  const float4* lightTris;    // 6 float4 per emitter triangle: (v1,ti.a) (v2,area) (v3,0) (n1,0) (n2,0) (n3,0)
  int numPointLights;
  const DevPointLight* points;
  const DevTexture* textures;
  int numTextures;
  int* error;                 // device error word (first error code wins)
  const float4* nodes8;       // 5 float4 per 8-wide compressed node (when bvhWidth == 8)
  int numNodes8;
  int bvhWidth;               // 2 or 8
  // equirectangular environment map, looked up by view-space direction
  int envTex;                 // texture index, -1 none
  int envW, envH;             // importance-sampling grid (the texture size); 0 when not sampled
  float envIntensity, envCosY, envSinY, envTotal;
  const float* envMarg;       // H+1 marginal CDF over rows
  const float* envCond;       // H x (W+1) conditional CDFs
  int envOn;                  // an environment (equirectangular or cubemap) is present
  int envCube;                // cubemap faces present: lookups use them
  int envFace[6];             // face textures +X -X +Y -Y +Z -Z
  int envCubeW;               // face size of the cubemap CDF, 0 when not sampled
  float envCubeTotal;
  const float* cubeMargFace;  // 7: CDF over the faces
  const float* cubeMargY;     // 6 x (W+1) per-face CDFs over rows
  const float* cubeCond;      // 6 x W x (W+1) per-row CDFs
  // procedural media and volume lights
  const DevPathPoint* pathPts;
  const DevVolLight* volLights;
  int numVolLights;
  int mediaLevel;             // 0 no active medium, 1 homogeneous only, 2 procedural / volume lights
};

// device error codes
constexpr int kErrTraversalSteps = 1;   // traversal exceeded its step bound
constexpr int kErrStackOverflow = 2;    // traversal stack full
constexpr int kErrLeafRange = 3;        // leaf outside the triangle array
constexpr int kErrPartition = 4;        // BVH build scatter outside a child range
constexpr int kMaxTraversalSteps = 1 << 22;

// Render-wide constants for the trace kernels.
struct DevRender {
  int width, height;
  float viewScale;            // 2 tan(fov/2) / H
  float halfW, halfH;
  float dof, aperture;        // aperture = 1/camera.aperture (0 when disabled)
  int blades;
  float apertureRot;          // radians
  float exposure;
  float viewFar;
  int aa;
  int colorSampling;
  int shader;
  int maxDepth, rrDepth;
  int lightFix;
  uint32_t seed;
  float clampMax;
  float backR, backG, backB;
  float worldR, worldG, worldB;
  int aoSamples;              // settings.samples (calcAO loop count)
};

// One render job resident on the device: its scene, render constants and
// accumulation buffers.  Kernels index a table of jobs by slot; the ray and
// shadow queues carry the slot of every ray.
struct DevJob {
  DevScene S;
  DevRender R;
  float4* sum;
  float4* sumSq;
  int* cnt;                   // samples per pixel so far (= next sample index)
  int pad[2];
};

// A wave is a list of segments; segment k holds paths
// [pathBase, pathBase + numPixels * samples) of job `slot`:
//   path = pathBase + s * numPixels + i, pixel = pixelList ? pixelList[pixelOffset + i] : pixelOffset + i,
//   sample = cnt[pixel] + s.
struct DevSegment {
  int slot;
  int numPixels;
  int samples;
  int pathBase;
  int pixelOffset;
  int pixBase;                // prefix sum of numPixels over the wave's segments
  const int* pixelList;
};

struct DevWave {
  int numSegments;
  int numPaths;
  int numPixelsTotal;
  int pad;
  const DevSegment* segs;
};

// Wavefront buffers.
struct DevQueues {
  float4* rayO[2];            // (origin, path id bits)
  float4* rayD[2];            // (dir, job slot bits)
  float4* hits;               // (t, u, v, prim bits) per queue slot
  // Path state that travels with its ray, in queue order (entry q of buffer b
  // belongs to ray q of rayO[b] / rayD[b]): the shade kernel reads it where it
  // reads the ray and writes it where it pushes the next ray, so no gather by
  // path id is needed for it.
  float4* pathT[2];           // (beta rgb, bsdfPdf)
  float4* pathR[2];           // (rrT rgb, flags bits)
  int2* pathPS[2];            // (pixel, sample)
  // By path id: the radiance that shadow rays add to and the accumulation reads.
  float4* pathL;              // (L rgb, vertex count | kVtxEyeNoHit bits)
  float4* shO[4];             // shadow queues A (area) / B (point) / C (environment) / D (volume): (origin, path id bits)
  float4* shD[4];             // (dir, tmax)
  float4* shC[4];             // (contribution rgb, job slot bits)
  int* counters;              // per-iteration counters, zeroed by the generate kernel
  unsigned long long* stats;  // [0] nodes closest [1] tris closest [2] nodes shadow [3] tris shadow [4] closest rays [5] shadow rays
  int* error;                 // first device error code
  int capacity;
  int maxIter;
};

// counters layout: [k*kCountersPerIter + c] for iteration k
enum CounterSlot {
  C_RAYS = 0, C_FETCH_EXT = 1, C_SHA = 2, C_SHB = 3, C_FETCH_SHA = 4, C_FETCH_SHB = 5, C_FETCH_SHADE = 6,
  C_SHC = 7, C_FETCH_SHC = 8, C_SHD = 9, C_FETCH_SHD = 10
};
constexpr int kCountersPerIter = 12;
// shadow queue `which` (0 area, 1 point, 2 environment, 3 volume) -> its counter slots
__host__ __device__ inline int shadowCountSlot(int which) {
  return which == 0 ? C_SHA : (which == 1 ? C_SHB : (which == 2 ? C_SHC : C_SHD));
}
__host__ __device__ inline int shadowFetchSlot(int which) {
  return which == 0 ? C_FETCH_SHA : (which == 1 ? C_FETCH_SHB : (which == 2 ? C_FETCH_SHC : C_FETCH_SHD));
}
// occluder class of shadow queue `which`; point lights and the environment share one
__host__ __device__ inline uint32_t shadowOccluder(int which) {
  return which == 0 ? kOccArea : (which == 3 ? kOccVol : kOccPoint);
}

// path flags (pathR.w)
constexpr uint32_t F_PASSES_MASK = 0xFFu;
constexpr uint32_t F_CHROMA_SHIFT = 8;       // 0 = none, 1..3 = channel+1
constexpr uint32_t F_CHROMA_MASK = 0x300u;
constexpr uint32_t F_MED_SHIFT = 12;         // medium + 1 (0 = none), 10 bits
constexpr uint32_t F_MED_MASK = 0x3FF000u;
constexpr uint32_t F_EYE = 1u << 24;         // next event is the eye vertex
constexpr uint32_t F_EYE_NOHIT = 1u << 25;   // eye ray hit no triangle
// pathL.w: the path's vertex count in the low bits, and this flag when the eye
// ray hit no triangle (the accumulation then shows the background colour)
constexpr int kVtxMask = (1 << 24) - 1;
constexpr int kVtxEyeNoHit = 1 << 30;

// ------------------------------------------------------------------ math ----
struct V3 {
  float x, y, z;
};
__host__ __device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__host__ __device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__host__ __device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__host__ __device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__host__ __device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float maxc(V3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
__device__ __forceinline__ V3 normalize(V3 a) {
  const float l = sqrtf(dot(a, a));
  return l > 0.0f ? v3(a.x / l, a.y / l, a.z / l) : a;
}
__device__ __forceinline__ V3 reflect(V3 d, V3 n) { return d - n * (dot(d, n) * 2.0f); }
__device__ __forceinline__ V3 xyz(float4 f) { return v3(f.x, f.y, f.z); }

// Non-contracted (round-to-nearest, no FMA) forms used where device results
// must match the CPU oracle bit for bit (triangle tests, scene transform).
__device__ __forceinline__ V3 sub_rn(V3 a, V3 b) { return v3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)); }
__device__ __forceinline__ float dot_rn(V3 a, V3 b) {
  return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
// FMA forms with a fixed evaluation order, mirrored exactly by the CPU oracle:
//   dot(a, b)   = fma(a.z, b.z, fma(a.y, b.y, a.x * b.x))
//   cross(a, b) = (fma(a.y, b.z, -(a.z * b.y)), fma(a.z, b.x, -(a.x * b.z)), fma(a.x, b.y, -(a.y * b.x)))
__device__ __forceinline__ float dot_f(V3 a, V3 b) {
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, __fmul_rn(a.x, b.x)));
}
__device__ __forceinline__ V3 cross_f(V3 a, V3 b) {
  return v3(__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
            __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ V3 cross_rn(V3 a, V3 b) {
  return v3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)), __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// ------------------------------------------------------------------- RNG ----
// Shared specification with the CPU oracle:
//   lds(dim)        dims < 16: Halton (radicalInverse(sample+1, prime[dim]),
//                   raycommon.cpp:48-61) + Cranley-Patterson offset
//                   hashPixel(dim, 0, hashPixel(x, y, seed-1)) (raycommon.cpp:71-87);
//                   dims >= 16: prng(vertex = dim, slot 63)
//   prng(v, slot)   pcg4d(pixel, sample, v<<6 | slot, seed).x >> 8, * 2^-24
__host__ __device__ __forceinline__ uint32_t hashPixel(uint32_t x, uint32_t y, uint32_t salt) {
  uint32_t v = x * 73856093u ^ y * 19349663u ^ salt * 83492791u;
  v ^= v >> 16; v *= 0x7feb352du;
  v ^= v >> 15; v *= 0x846ca68bu;
  v ^= v >> 16;
  return v;
}
__host__ __device__ __forceinline__ uint32_t pcg4d_x(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  uint32_t v0 = a * 1664525u + 1013904223u, v1 = b * 1664525u + 1013904223u;
  uint32_t v2 = c * 1664525u + 1013904223u, v3_ = d * 1664525u + 1013904223u;
  v0 += v1 * v3_; v1 += v2 * v0; v2 += v0 * v1; v3_ += v1 * v2;
  v0 ^= v0 >> 16; v1 ^= v1 >> 16; v2 ^= v2 >> 16; v3_ ^= v3_ >> 16;
  v0 += v1 * v3_; v1 += v2 * v0; v2 += v0 * v1; v3_ += v1 * v2;
  return v0;
}

template <int BASE>
__device__ __forceinline__ float radicalInverseT(uint32_t i) {
  const float invBase = 1.0f / (float)BASE;
  float invBaseN = 1.0f;
  uint64_t rev = 0;
  while (i > 0) {
    const uint32_t next = i / BASE;
    const uint32_t digit = i - next * BASE;
    rev = rev * BASE + digit;
    invBaseN = __fmul_rn(invBaseN, invBase);
    i = next;
  }
  const float v = __fmul_rn((float)rev, invBaseN);
  return v < 1.0f ? v : 0.9999999f;
}

__device__ __forceinline__ float radicalInverseDim(uint32_t i, int dim) {
  switch (dim) {
    case 0: return radicalInverseT<2>(i);
    case 1: return radicalInverseT<3>(i);
    case 2: return radicalInverseT<5>(i);
    case 3: return radicalInverseT<7>(i);
    case 4: return radicalInverseT<11>(i);
    case 5: return radicalInverseT<13>(i);
    case 6: return radicalInverseT<17>(i);
    case 7: return radicalInverseT<19>(i);
    case 8: return radicalInverseT<23>(i);
    case 9: return radicalInverseT<29>(i);
    case 10: return radicalInverseT<31>(i);
    case 11: return radicalInverseT<37>(i);
    case 12: return radicalInverseT<41>(i);
    case 13: return radicalInverseT<43>(i);
    case 14: return radicalInverseT<47>(i);
    default: return radicalInverseT<53>(i);
  }
}

enum Slot {
  S_LOBE = 0, S_LIGHT = 1, S_MESH = 2, S_TRI = 3, S_VNDF0 = 4, S_VNDF1 = 5, S_RR = 6,
  S_FRESNEL = 7, S_CHROMA = 8, S_HEMI0 = 9, S_HEMI1 = 10, S_POINT = 11, S_ENV0 = 12,
  S_ENV1 = 13, S_FLIGHT = 14, S_PHASE0 = 15, S_PHASE1 = 16, S_MEDRR = 17, S_EYETR = 18,
  S_DTSTEP = 19, S_DTACC = 20, S_EMIS = 21, S_VOLPICK = 22, S_VOLU = 23,
  S_LDS = 63
};

struct Rng {
  uint32_t pixel, sample, seed, scramble;
  int dimBase;
  __device__ __forceinline__ void init(uint32_t x, uint32_t y, uint32_t width, uint32_t s, uint32_t sd, int base) {
    pixel = y * width + x;
    sample = s;
    seed = sd;
    scramble = hashPixel(x, y, sd - 1u);
    dimBase = base;
  }
  __device__ __forceinline__ float prng(int v, int slot) const {
    const uint32_t h = pcg4d_x(pixel, sample, ((uint32_t)v << 6) | (uint32_t)slot, seed);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
  }
  // k-th draw of a repeated use at vertex v (delta-tracking steps, emission
  // strata); k = 0 is prng(v, slot).
  __device__ __forceinline__ float prngk(int v, int slot, int k) const {
    const uint32_t h = pcg4d_x(pixel, sample, ((uint32_t)k << 16) | ((uint32_t)v << 6) | (uint32_t)slot, seed);
    return (float)(h >> 8) * (1.0f / 16777216.0f);
  }
  __device__ __forceinline__ float lds(int dim) const {
    if (dim >= 16) return prng(dim, S_LDS);
    const float v = radicalInverseDim(sample + 1u, dim);
    const uint32_t h = hashPixel((uint32_t)dim, 0u, scramble);
    const float off = (float)(h >> 8) * (1.0f / 16777216.0f);
    float w = __fadd_rn(v, off);
    if (w >= 1.0f) w = __fsub_rn(w, 1.0f);
    return w;
  }
  __device__ __forceinline__ int dirDim(int v) const { return dimBase + 4 * v; }
  __device__ __forceinline__ int neeDim(int v) const { return dimBase + 4 * v + 2; }
};

__device__ __forceinline__ int pickIndex(float u, int n) {
  const int i = (int)(u * (float)n);
  return i < n - 1 ? i : n - 1;
}

__device__ __forceinline__ void setError(int* err, int code) { atomicCAS(err, 0, code); }

}  // namespace rg
