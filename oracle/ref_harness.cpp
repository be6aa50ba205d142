// ref_harness.cpp - TEST INFRASTRUCTURE ONLY.
//
// Runs the reference renderer's own hot-path code, compiled unchanged from
// its sources (src/raygen/bvh.cpp, raycommon.cpp, medium.cpp, bsdf.cpp of the
// RayGen project) against the clean-room math stand-in in oracle/ref_shim/,
// and exposes it through a small C interface.  tests/golden/make_ref_golden.py
// uses it to write golden vectors that pin both the CPU oracle (rg_oracle.cpp)
// and the B200 kernels to the reference's own outputs:
//   * TriangleBVH::build / intersectClosest / intersectAny (bvh.cpp:76-285,
//     bvh.h:63-101) over RenderMeshTriangle (raycommon.cpp:128-235);
//   * the Halton / Cranley-Patterson sampler (raycommon.cpp:35-92),
//     cosineWeightedDirection (:94-115) and ldsPointInTriangle (:117-122);
//   * fresnelSchlick, refract, buildTangentFrame, sampleGGXVNDF, smithG1
//     (bsdf.cpp:32-52, 129-170);
//   * HomogeneousMedium: prepare, transmittance, sampleFreeFlight,
//     samplePhase, phasePdf, densityAt, emissionAt, iorAt, bendRay
//     (medium.cpp:18-123, 128-404, 475-525).
// The build recipe is oracle/Makefile's `ref` target; the library goes to
// oracle/_ref/ and is never shipped, linked into, or loaded by the product.
//
// Nothing the probes call needs the renderer class; its member functions that
// bsdf.cpp's shaders reference are defined below only so the library links,
// and abort if ever reached.  randomValue() (ugm, not vendored) reads a
// caller-supplied stream of uniforms.

#include <cstdlib>
#include <vector>

// bsdf.cpp keeps its GGX helpers in an anonymous namespace: the harness
// compiles the whole file as part of this translation unit to reach them.
#include "bsdf.cpp"

namespace {
thread_local const float* g_stream = nullptr;
thread_local int g_streamLen = 0;
thread_local int g_streamPos = 0;
}  // namespace

namespace ugm {
float randomValue() {
  if (g_stream && g_streamPos < g_streamLen) return g_stream[g_streamPos++];
  return 0.5f;
}
// Unused by the probes (the reference's hemisphere sampler is not vendored).
vec3 randomRayInHemisphere(const vec3& normal) {
  const float u1 = randomValue(), u2 = randomValue();
  const float z = 1.0f - 2.0f * u1;
  const float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
  const float phi = 2.0f * (float)M_PI * u2;
  vec3 d = vec3(r * cosf(phi), r * sinf(phi), z);
  return dot(d, normal) < 0.0f ? -d : d;
}
}  // namespace ugm

namespace raygen {
// Out-of-line members declared by the reference headers and defined in files
// the harness does not compile.
SceneObject::~SceneObject() {}
Mesh::~Mesh() {}
[[noreturn]] static void unreachable() { std::abort(); }
color4f Texture::sample(const vec2&) const { unreachable(); }
color3 RayRenderer::tracePath(const Ray&, void*) const { unreachable(); }
color3 RayRenderer::traceLight(const vec3&, const vec3&) const { unreachable(); }
color3 RayRenderer::traceEnvmapLight(const vec3&, const vec3&, float) const { unreachable(); }
bool RayRenderer::sampleAreaLightForNEE(const vec3&, const vec3&, vec3&, float&, color3&) const { unreachable(); }
bool RayRenderer::sampleEnvmapForNEE(const vec3&, const vec3&, vec3&, float&, color3&) const { unreachable(); }
bool RayRenderer::sampleVolumeLightForNEE(const vec3&, const vec3&, vec3&, float&, float&, color3&) const {
  unreachable();
}
float RayRenderer::envmapDirectionPdf(const vec3&) const { unreachable(); }
}  // namespace raygen

using namespace raygen;

namespace {

struct RefScene {
  SceneObject object;
  Mesh mesh;
  std::vector<RenderMeshTriangle> tris;  // DFS order, never reallocated after build
  TriangleBVH bvh;
};

inline vec3 V(const float* p) { return vec3(p[0], p[1], p[2]); }
inline void put(float* o, const vec3& v) {
  o[0] = v.x;
  o[1] = v.y;
  o[2] = v.z;
}

}  // namespace

extern "C" {

// n view-space triangles (positions n x 9, vertex normals n x 9) -> a scene
// with the reference's BVH built over them.
void* ref_scene_create(const float* pos, const float* nrm, int32_t n) {
  RefScene* s = new RefScene();
  s->tris.reserve((size_t)n);
  const vec2 z2 = vec2(0.0f, 0.0f);
  for (int32_t i = 0; i < n; ++i) {
    const float* p = pos + (size_t)i * 9;
    const float* q = nrm + (size_t)i * 9;
    s->tris.emplace_back(V(p), V(p + 3), V(p + 6), V(q), V(q + 3), V(q + 6), z2, z2, z2, z2, z2, z2, s->object,
                         s->mesh);
  }
  std::vector<const RenderMeshTriangle*> prims;
  prims.reserve(s->tris.size());
  for (const RenderMeshTriangle& t : s->tris) prims.push_back(&t);
  s->bvh.build(prims);
  return s;
}

void ref_scene_destroy(void* h) { delete static_cast<RefScene*>(h); }

int32_t ref_bvh_nodes(void* h) { return (int32_t) static_cast<RefScene*>(h)->bvh.nodeCount(); }

// Closest hit of rays n x 6 (origin, direction): t/u/v n x 3 and the DFS
// triangle index (-1: miss), with the renderer's initial t (MAX_RAY_DISTANCE).
void ref_closest(void* h, const float* rays, int32_t n, float* out_tuv, int32_t* out_prim) {
  const RefScene& s = *static_cast<RefScene*>(h);
  for (int32_t i = 0; i < n; ++i) {
    const float* r = rays + (size_t)i * 6;
    const Ray ray = Ray(V(r), V(r + 3));
    RayTriangleIntersectionInfo info;
    const bool hit = s.bvh.intersectClosest(ray, info);
    out_prim[i] = hit ? (int32_t)(info.triangle - s.tris.data()) : -1;
    out_tuv[i * 3] = info.t;
    out_tuv[i * 3 + 1] = info.u;
    out_tuv[i * 3 + 2] = info.v;
  }
}

// Any hit in (1e-6, tmax) with every triangle an occluder.
void ref_any(void* h, const float* rays, const float* tmax, int32_t n, uint8_t* out) {
  const RefScene& s = *static_cast<RefScene*>(h);
  for (int32_t i = 0; i < n; ++i) {
    const float* r = rays + (size_t)i * 6;
    out[i] = s.bvh.intersectAny(Ray(V(r), V(r + 3)), tmax[i], [](const RenderMeshTriangle*) { return true; }) ? 1 : 0;
  }
}

// The Halton / Cranley-Patterson value of dimension `dim` (< 16) of a pixel
// sample: ldsBeginPixelSample(x, y, sample), then dim + 1 draws.
float ref_lds(int32_t x, int32_t y, int32_t sample, int32_t dim) {
  ldsBeginPixelSample(x, y, sample);
  float v = 0.0f;
  for (int32_t k = 0; k <= dim; ++k) v = ldsNext1D();
  return v;
}

// cosineWeightedDirection(normal) drawing dimensions dim, dim + 1.
void ref_cosine_direction(int32_t x, int32_t y, int32_t sample, int32_t dim, const float* normal, float* out3) {
  ldsBeginPixelSample(x, y, sample);
  for (int32_t k = 0; k < dim; ++k) ldsNext1D();
  put(out3, cosineWeightedDirection(V(normal)));
}

// ldsPointInTriangle(tri) drawing dimensions dim, dim + 1.
void ref_point_in_triangle(int32_t x, int32_t y, int32_t sample, int32_t dim, const float* tri9, float* out3) {
  ldsBeginPixelSample(x, y, sample);
  for (int32_t k = 0; k < dim; ++k) ldsNext1D();
  Triangle t;
  t.v1 = V(tri9);
  t.v2 = V(tri9 + 3);
  t.v3 = V(tri9 + 6);
  put(out3, ldsPointInTriangle(t));
}

// GGX helpers of bsdf.cpp, one row per input.
//   which 0 sampleGGXVNDF : in (Ve xyz, ax, ay, u1, u2) -> H xyz
//   which 1 smithG1       : in (w xyz, ax, ay)          -> G1
//   which 2 fresnelSchlick: in (cosTheta, ior)          -> F
//   which 3 refract       : in (d xyz, n xyz, ior)      -> dir xyz
//   which 4 buildTangentFrame: in (n xyz)               -> t xyz, b xyz
void ref_bsdf_probe(int32_t which, const float* in, int32_t n, float* out) {
  for (int32_t i = 0; i < n; ++i) {
    switch (which) {
      case 0: {
        const float* a = in + (size_t)i * 7;
        put(out + (size_t)i * 3, sampleGGXVNDF(V(a), a[3], a[4], a[5], a[6]));
        break;
      }
      case 1: {
        const float* a = in + (size_t)i * 5;
        out[i] = smithG1(V(a), a[3], a[4]);
        break;
      }
      case 2: {
        const float* a = in + (size_t)i * 2;
        out[i] = fresnelSchlick(a[0], a[1]);
        break;
      }
      case 3: {
        const float* a = in + (size_t)i * 7;
        put(out + (size_t)i * 3, raygen::refract(V(a), V(a + 3), a[6]));
        break;
      }
      case 4: {
        vec3 t, b;
        buildTangentFrame(V(in + (size_t)i * 3), t, b);
        put(out + (size_t)i * 6, t);
        put(out + (size_t)i * 6 + 3, b);
        break;
      }
      default:
        break;
    }
  }
}

// A homogeneous medium built the way the scene loader does (fields, then
// prepare()), with its render-space copies taken at the identity view.
//   p: sigma_a rgb, sigma_s rgb, g, density, densityField (0/1), noise
//      frequency, octaves, gain, lacunarity, amplitude, bias, offset xyz,
//      emission mode (0/1/2), sigma_e rgb, cone origin xyz, cone axis xyz,
//      cone length, radius, inner rgb, outer rgb, intensity, peak axial,
//      peak sharpness, heat haze (0/1), ior amplitude, frequency, octaves,
//      gain, lacunarity, march steps, ior offset xyz, ior falloff
//   (50 floats); path points are not set.
void* ref_medium_create(const float* p) {
  HomogeneousMedium* m = new HomogeneousMedium();
  int k = 0;
  auto c3 = [&]() {
    const color3 c = color3(p[k], p[k + 1], p[k + 2]);
    k += 3;
    return c;
  };
  auto v3 = [&]() {
    const vec3 c = vec3(p[k], p[k + 1], p[k + 2]);
    k += 3;
    return c;
  };
  m->sigma_a = c3();
  m->sigma_s = c3();
  m->g = p[k++];
  m->density = p[k++];
  m->densityField = p[k++] > 0.5f ? HomogeneousMedium::DensityField_FBmNoise : HomogeneousMedium::DensityField_None;
  m->noiseFrequency = p[k++];
  m->noiseOctaves = (int)p[k++];
  m->noiseGain = p[k++];
  m->noiseLacunarity = p[k++];
  m->noiseAmplitude = p[k++];
  m->noiseBias = p[k++];
  m->noiseOffset = v3();
  m->emissionMode = (HomogeneousMedium::EmissionMode)(int)p[k++];
  m->sigma_e = c3();
  m->coneOrigin = v3();
  m->coneAxis = v3();
  m->coneLength = p[k++];
  m->coneRadius = p[k++];
  m->coneInner = c3();
  m->coneOuter = c3();
  m->coneIntensity = p[k++];
  m->conePeakAxial = p[k++];
  m->conePeakSharpness = p[k++];
  m->heatHaze = p[k++] > 0.5f;
  m->iorAmplitude = p[k++];
  m->iorFrequency = p[k++];
  m->iorOctaves = (int)p[k++];
  m->iorGain = p[k++];
  m->iorLacunarity = p[k++];
  m->iorMarchSteps = (int)p[k++];
  m->iorOffset = v3();
  m->iorFalloff = p[k++];
  m->prepare();
  m->bake(Matrix4(), Matrix4());
  return m;
}

void ref_medium_destroy(void* m) { delete static_cast<HomogeneousMedium*>(m); }

// Medium probes, one row per input.
//   which 0 transmittance   : in (d)                 -> rgb
//   which 1 sampleFreeFlight: in (u)                 -> t
//   which 2 samplePhase     : in (wo xyz, u1, u2)    -> wi xyz
//   which 3 phasePdf        : in (wo xyz, wi xyz)    -> pdf
//   which 4 fields          : in (p xyz)             -> density, emission rgb, ior
//   which 5 bendRay         : in (o xyz, d xyz, len) -> o xyz, d xyz
//   which 6 sampleDeltaTracking: in (o xyz, d xyz, maxT, 16 uniforms) -> hit, t, density
void ref_medium_probe(void* mp, int32_t which, const float* in, int32_t n, float* out) {
  const HomogeneousMedium& m = *static_cast<HomogeneousMedium*>(mp);
  for (int32_t i = 0; i < n; ++i) {
    switch (which) {
      case 0: {
        const color3 c = m.transmittance(in[i]);
        out[i * 3] = c.r;
        out[i * 3 + 1] = c.g;
        out[i * 3 + 2] = c.b;
        break;
      }
      case 1:
        out[i] = m.sampleFreeFlight(in[i]);
        break;
      case 2: {
        const float* a = in + (size_t)i * 5;
        put(out + (size_t)i * 3, m.samplePhase(V(a), a[3], a[4]));
        break;
      }
      case 3: {
        const float* a = in + (size_t)i * 6;
        out[i] = m.phasePdf(V(a), V(a + 3));
        break;
      }
      case 4: {
        const vec3 p = V(in + (size_t)i * 3);
        const color3 e = m.emissionAt(p);
        float* o = out + (size_t)i * 5;
        o[0] = m.densityAt(p);
        o[1] = e.r;
        o[2] = e.g;
        o[3] = e.b;
        o[4] = m.iorAt(p);
        break;
      }
      case 5: {
        const float* a = in + (size_t)i * 7;
        const Ray b = m.bendRay(Ray(V(a), V(a + 3)), a[6]);
        put(out + (size_t)i * 6, b.origin);
        put(out + (size_t)i * 6 + 3, b.dir);
        break;
      }
      case 6: {
        const float* a = in + (size_t)i * 23;
        g_stream = a + 7;
        g_streamLen = 16;
        g_streamPos = 0;
        float t = 0.0f, dens = 0.0f;
        const bool hit = m.sampleDeltaTracking(Ray(V(a), V(a + 3)), a[6], t, dens);
        g_stream = nullptr;
        out[i * 3] = hit ? 1.0f : 0.0f;
        out[i * 3 + 1] = t;
        out[i * 3 + 2] = dens;
        break;
      }
      default:
        break;
    }
  }
}

}  // extern "C"
