// rg_api.cu - host runtime behind the C ABI (include/raygen_b200.h).
//
// Mirrors the RayRenderer lifecycle (rayrenderer.cpp:53-596): settings are
// copied at creation, the scene is flattened to view space and its BVH built
// on the device when it is set, and render() runs the wavefront tracer
// (optionally in adaptive passes), the A-Trous denoiser and the tonemap, all
// on the device.  Waves of paths are replayed through one captured CUDA
// graph; the wave descriptors live on the device and a one-thread kernel at
// the end of the graph advances to the next one.
#include <cuda_fp16.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <climits>
#include <cstdlib>
#include <unordered_map>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "rg_device.cuh"
#include "rg_host.h"
#include "rg_trace.cuh"

namespace rg {

static thread_local std::string g_lastError;
void setLastError(const std::string& msg) { g_lastError = msg; }

#define RG_CUDA_CHECK(call)                                                     \
  do {                                                                          \
    cudaError_t e__ = (call);                                                   \
    if (e__ != cudaSuccess) {                                                   \
      setLastError(std::string(#call) + ": " + cudaGetErrorString(e__));        \
      return RG_ERR_CUDA;                                                       \
    }                                                                           \
  } while (0)

__global__ void k_nextWave(int* cur) { *cur += 1; }

// The render's sample total: the sum of the per-pixel sample counts, added to *out.
__global__ void k_sumCounts(int n, const int* __restrict__ cnt, unsigned long long* out) {
  __shared__ unsigned long long part[8];
  unsigned long long v = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v += (unsigned)cnt[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += part[w];
    atomicAdd(out, t);
  }
}

void keepPoolMemory() {
  static std::mutex mu;
  static std::vector<char> done;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  std::lock_guard<std::mutex> lk(mu);
  if ((int)done.size() <= dev) done.resize(dev + 1, 0);
  if (done[dev]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done[dev] = 1;
}

void trimPoolMemory() {
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    cudaStreamSynchronize(cudaStreamPerThread);
    cudaMemPoolTrimTo(pool, 0);
  }
  cudaGetLastError();
}

// Camera view matrix, row-vector convention p_view = [p 1] * M.
// Camera orientation R = Ry(angle.y) * Rx(angle.x) * Rz(angle.z) (degrees);
// p_view = R^T (p - location).  With zero angles this is exactly p - location.
Mat4 viewMatrix(const rg_camera& c) {
  const float d2r = 3.14159265358979323846f / 180.0f;
  const float ax = c.angle[0] * d2r, ay = c.angle[1] * d2r, az = c.angle[2] * d2r;
  const double cx = std::cos(ax), sx = std::sin(ax), cy = std::cos(ay), sy = std::sin(ay), cz = std::cos(az), sz = std::sin(az);
  double Rx[3][3] = {{1, 0, 0}, {0, cx, -sx}, {0, sx, cx}};
  double Ry[3][3] = {{cy, 0, sy}, {0, 1, 0}, {-sy, 0, cy}};
  double Rz[3][3] = {{cz, -sz, 0}, {sz, cz, 0}, {0, 0, 1}};
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
  Mat4 M;
  std::memset(M.m, 0, sizeof(M.m));
  // p_view_j = sum_i (p_i - loc_i) R[i][j]
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) M.m[i * 4 + j] = (float)R[i][j];
  for (int j = 0; j < 3; j++) {
    const float t = c.location[0] * M.m[0 * 4 + j] + c.location[1] * M.m[1 * 4 + j] + c.location[2] * M.m[2 * 4 + j];
    M.m[12 + j] = -t;
  }
  M.m[15] = 1.0f;
  return M;
}

namespace {

inline void xformPoint(const Mat4& M, const float* p, float* o) {
  for (int j = 0; j < 3; j++) o[j] = ((p[0] * M.m[j] + p[1] * M.m[4 + j]) + p[2] * M.m[8 + j]) + M.m[12 + j];
}
inline void xformDir(const Mat4& M, const float* p, float* o) {
  for (int j = 0; j < 3; j++) o[j] = (p[0] * M.m[j] + p[1] * M.m[4 + j]) + p[2] * M.m[8 + j];
  const float l = std::sqrt((o[0] * o[0] + o[1] * o[1]) + o[2] * o[2]);
  if (l > 0) { o[0] /= l; o[1] /= l; o[2] /= l; }
}

struct F3h {
  float x, y, z;
};
inline F3h sub(F3h a, F3h b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline F3h crs(F3h a, F3h b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline float len(F3h a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }

DevMaterial toDev(const rg_material& m) {
  DevMaterial d;
  d.cr = m.color[0]; d.cg = m.color[1]; d.cb = m.color[2];
  d.glossy = m.glossy; d.roughness = m.roughness; d.transparency = m.transparency; d.refraction = m.refraction;
  d.ior = m.refraction_ratio; d.chroma = m.chroma_dispersion; d.metallic = m.metallic; d.aniso = m.anisotropy;
  d.anisoRot = m.aniso_rotation; d.emission = m.emission; d.spotRange = m.spot_range; d.texture = m.texture;
  d.tileU = m.tex_tiling[0]; d.tileV = m.tex_tiling[1]; d.pad = 0;
  return d;
}

// HomogeneousMedium::prepare (medium.cpp:18-57), constant mode.
inline int capCount(int n) { return n > kMaxMediumCount ? kMaxMediumCount : n; }

// One medium after HomogeneousMedium::prepare() and bake() (medium.cpp:18-101),
// in camera space: cone origin / axis transformed for cone-mode media only,
// path points for path-mode media only (the reference bakes nothing else),
// and isActive() (medium.h:226-234).
DevMedium toDev(const rg_medium& m, const Mat4& view, std::vector<DevPathPoint>& pts) {
  DevMedium d;
  std::memset(&d, 0, sizeof(d));
  const float dn = std::fmax(0.0f, m.density);
  d.ssr = m.sigma_s[0] * dn; d.ssg = m.sigma_s[1] * dn; d.ssb = m.sigma_s[2] * dn;
  d.ser = m.sigma_e[0] * dn; d.seg = m.sigma_e[1] * dn; d.seb = m.sigma_e[2] * dn;
  d.str = m.sigma_a[0] * dn + d.ssr; d.stg = m.sigma_a[1] * dn + d.ssg; d.stb = m.sigma_a[2] * dn + d.ssb;
  d.hero = (d.str + d.stg + d.stb) * (1.0f / 3.0f);
  d.g = m.g;
  d.densityScale = dn;
  d.mode = (m.emission_mode == RG_EMISSION_CONE || m.emission_mode == RG_EMISSION_PATH) ? m.emission_mode : 0;
  d.field = m.density_field == RG_DENSITY_FBM ? 1 : 0;
  d.tMaxHero = d.field ? d.hero * std::fmax(0.0f, m.noise_amplitude * 1.0f + m.noise_bias) : d.hero;
  // cone frame
  const float al2 = m.cone_axis[0] * m.cone_axis[0] + m.cone_axis[1] * m.cone_axis[1] + m.cone_axis[2] * m.cone_axis[2];
  float axN[3] = {0.0f, 0.0f, -1.0f};
  if (al2 > 1e-12f) {
    const float inv = 1.0f / std::sqrt(al2);
    for (int k = 0; k < 3; k++) axN[k] = m.cone_axis[k] * inv;
  }
  float org[3] = {m.cone_origin[0], m.cone_origin[1], m.cone_origin[2]}, ax[3] = {axN[0], axN[1], axN[2]};
  if (d.mode == RG_EMISSION_CONE) {
    xformPoint(view, m.cone_origin, org);
    float av[3];
    for (int j = 0; j < 3; j++) av[j] = (axN[0] * view.m[j] + axN[1] * view.m[4 + j]) + axN[2] * view.m[8 + j];
    const float vl2 = av[0] * av[0] + av[1] * av[1] + av[2] * av[2];
    if (vl2 > 1e-12f) {
      const float inv = 1.0f / std::sqrt(vl2);
      for (int k = 0; k < 3; k++) ax[k] = av[k] * inv;
    }
  }
  d.cox = org[0]; d.coy = org[1]; d.coz = org[2];
  d.cax = ax[0]; d.cay = ax[1]; d.caz = ax[2];
  d.coneLength = m.cone_length; d.coneRadius = m.cone_radius;
  d.cir = m.cone_inner[0]; d.cig = m.cone_inner[1]; d.cib = m.cone_inner[2];
  d.cor = m.cone_outer[0]; d.cog = m.cone_outer[1]; d.cob = m.cone_outer[2];
  d.coneIntensity = m.cone_intensity; d.conePeakAxial = m.cone_peak_axial; d.conePeakSharpness = m.cone_peak_sharpness;
  d.coneSamples = capCount(m.cone_emission_samples);
  // path tube
  d.pathCount = std::max(0, m.num_path_points);
  d.pathFirst = (int)pts.size();
  if (d.mode == RG_EMISSION_PATH)
    for (int i = 0; i < d.pathCount; i++) {
      const rg_medium_path_point& q = m.path_points[i];
      float pv[3];
      xformPoint(view, q.p, pv);
      pts.push_back(DevPathPoint{make_float4(pv[0], pv[1], pv[2], q.radius), make_float4(q.t, 0.0f, 0.0f, 0.0f)});
    }
  d.pir = m.path_inner[0]; d.pig = m.path_inner[1]; d.pib = m.path_inner[2];
  d.por = m.path_outer[0]; d.pog = m.path_outer[1]; d.pob = m.path_outer[2];
  d.pathIntensity = m.path_intensity; d.pathFalloff = m.path_falloff_power;
  d.pathSamples = capCount(m.path_emission_samples);
  // fBm density
  d.nFreq = m.noise_frequency; d.nOct = capCount(m.noise_octaves); d.nGain = m.noise_gain; d.nLac = m.noise_lacunarity;
  d.nAmp = m.noise_amplitude; d.nBias = m.noise_bias;
  d.nox = m.noise_offset[0]; d.noy = m.noise_offset[1]; d.noz = m.noise_offset[2];
  // heat haze
  d.hazeOn = m.heat_haze != 0;
  d.iAmp = m.ior_amplitude; d.iFreq = m.ior_frequency; d.iOct = capCount(m.ior_octaves); d.iGain = m.ior_gain;
  d.iLac = m.ior_lacunarity; d.iSteps = capCount(m.ior_march_steps);
  d.iox = m.ior_offset[0]; d.ioy = m.ior_offset[1]; d.ioz = m.ior_offset[2];
  d.iFalloff = m.ior_falloff;
  d.haze = d.hazeOn && d.iAmp > 0.0f && d.iSteps > 0;
  const bool glow = d.ser != 0.0f || d.seg != 0.0f || d.seb != 0.0f;
  d.active = d.hero > 0.0f || (d.mode == RG_EMISSION_CONE && d.coneIntensity > 0.0f) ||
             (d.mode == RG_EMISSION_PATH && d.pathIntensity > 0.0f && d.pathCount >= 2) || (d.hazeOn && d.iAmp > 0.0f) ||
             glow;
  return d;
}

// Camera-space media, the objects' interior media and the global medium with
// inactive media removed (readMedium drops them, sceneloader.cpp:325-333),
// the emissive volumes sampled by volume-light NEE in object order
// (rayrenderer.cpp:180-206), and the shade-kernel variant the scene needs.
struct MediaTables {
  std::vector<DevMedium> media;
  std::vector<DevPathPoint> pts;
  std::vector<DevVolLight> vols;
  std::vector<int> objMed;
  int globalMedium = -1;
  int level = 0;
  bool hasHaze = false;
};

void buildMedia(const rg_scene_desc* d, const Mat4& view, MediaTables& T) {
  T.media.resize(d->num_media);
  for (int i = 0; i < d->num_media; i++) T.media[i] = toDev(d->media[i], view, T.pts);
  auto live = [&](int m) { return m >= 0 && m < d->num_media && T.media[m].active ? m : -1; };
  T.globalMedium = live(d->global_medium);
  T.objMed.resize(d->num_objects);
  std::vector<char> used(d->num_media, 0);
  if (T.globalMedium >= 0) used[T.globalMedium] = 1;
  for (int o = 0; o < d->num_objects; o++) {
    const int m = live(d->objects[o].interior_medium);
    T.objMed[o] = m;
    if (m < 0) continue;
    used[m] = 1;
    const DevMedium& M = T.media[m];
    const bool cone = M.mode == RG_EMISSION_CONE && M.coneIntensity > 0.0f;
    const bool glow = M.mode == 0 && (M.ser != 0.0f || M.seg != 0.0f || M.seb != 0.0f);
    if (cone || glow) {
      float a[3];
      xformPoint(view, d->objects[o].location, a);
      T.vols.push_back(DevVolLight{m, a[0], a[1], a[2]});
    }
  }
  bool any = false, procedural = !T.vols.empty();
  for (int i = 0; i < d->num_media; i++) {
    if (!used[i]) continue;
    const DevMedium& M = T.media[i];
    any = true;
    if (M.mode != 0 || M.field != 0 || M.haze) procedural = true;
    if (M.haze) T.hasHaze = true;
  }
  T.level = procedural ? 2 : (any ? 1 : 0);
}


}  // namespace

}  // namespace rg

using namespace rg;

struct rg_handle {
  rg_settings st;
  std::mutex mu;
  cudaStream_t stream = nullptr;
  int device = 0;
  int numSMs = 148;
  std::unique_ptr<DeviceScene> scene;
  DevScene dscene{};
  rg_camera camera{};
  Mat4 view{};
  bool hasScene = false;
  // render buffers
  DevBuf<float4> sum, sumSq, hdr, ldr, bufA, bufB;
  DevBuf<float4> preBloom, bloomA, bloomB;  // HDR before bloom (reapply), glow buffers
  rg_denoiser* denoiser = nullptr;           // learned denoiser (NULL: A-Trous)
  DevBuf<float> bloomW;                     // Gaussian taps
  DevBuf<int> cnt, pixelList, listCount;
  DevBuf<__half> aovNormal, aovAlbedo, aovAlbedoA, aovDepth;
  int W = 0, H = 0;
  bool haveResult = false;
  // wavefront
  DevBuf<float4> rayO0, rayO1, rayD0, rayD1, hits, pathT0, pathT1, pathR0, pathR1, pathL, shO0, shO1, shO2, shD0, shD1, shD2, shC0, shC1, shC2;
  DevBuf<float4> shO3, shD3, shC3;  // volume-light shadow queue, allocated for scenes with volume lights
  DevBuf<int2> pathPS0, pathPS1;
  DevBuf<DevJob> jobsDev;
  DevBuf<DevSegment> segs;
  DevBuf<int> counters, error, curWave;
  DevBuf<unsigned long long> stats;
  DevBuf<DevWave> waves, waveSlot;
  int capacity = 0;
  int maxIter = 0;
  // graph
  cudaGraphExec_t graph = nullptr;
  std::string graphKey;
  // progress / cancel
  rg_progress_fn progress = nullptr;
  void* progressUser = nullptr;
  std::atomic<bool> cancel{false};
  std::atomic<float> progressValue{0.0f};  // completed waves / waves planned, for rg_poll
  std::atomic<bool> asyncBusy{false};      // an rg_render_async job is in flight
  double firstWaveHostMs = 0.0;            // host clock when the render's first wave was launched
  cudaEvent_t waveDone[2] = {nullptr, nullptr};
  // second stream of the wave graph: a bounce's shadow rays beside the next bounce's closest hits
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  rg_stats lastStats{};
  ~rg_handle() {
    for (auto e : waveDone)
      if (e) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    if (graph) cudaGraphExecDestroy(graph);
    scene.reset();
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace rg {

namespace {
double hostMs() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

// every device buffer of a DeviceScene but the texture texels
#define RG_SCENE_BUFFERS(X)                                                                                    \
  X(inPos) X(inNrm) X(inUV) X(inTriMesh) X(view) X(meshObj) X(meshTriCount) X(objMat) X(objMedium) X(mats)      \
  X(media) X(pathPts) X(volLights) X(areaLightObj) X(lightMeshList) X(lightObjMeshes) X(lightMeshTris)           \
  X(lightTris) X(points) X(textures) X(envMarg) X(envCond) X(cubeMargFace) X(cubeMargY) X(cubeCond) X(nodes)     \
  X(nodes8) X(triVerts) X(triShade) X(triUV) X(triOrig) X(triMat)

size_t DeviceScene::deviceBytes() const {
  size_t b = 0;
#define RG_ADD_BYTES(m) b += m.bytes();
  RG_SCENE_BUFFERS(RG_ADD_BYTES)
#undef RG_ADD_BYTES
  for (const auto* t : texels) b += t ? t->bytes() : 0;
  return b;
}

void DeviceScene::adoptBuffers(DeviceScene& old) {
#define RG_TAKE(m) m.swap(old.m);
  RG_SCENE_BUFFERS(RG_TAKE)
#undef RG_TAKE
  texels.swap(old.texels);
  std::swap(scratch, old.scratch);
}

namespace {

rg_status ensureQueues(rg_handle* h, int capacity, int maxIter, bool volQueue) {
  if (volQueue) {
    const size_t c = (size_t)std::max(capacity, h->capacity);
    if (!h->shO3.alloc(c) || !h->shD3.alloc(c) || !h->shC3.alloc(c)) {
      setLastError("out of device memory (wavefront queues)");
      return RG_ERR_OUT_OF_MEMORY;
    }
  }
  if (capacity <= h->capacity && maxIter <= h->maxIter) return RG_OK;
  const size_t c = (size_t)std::max(capacity, h->capacity);
  const int mi = std::max(maxIter, h->maxIter);
  bool ok = h->rayO0.alloc(c) && h->rayO1.alloc(c) && h->rayD0.alloc(c) && h->rayD1.alloc(c) && h->hits.alloc(c) &&
            h->pathT0.alloc(c) && h->pathT1.alloc(c) && h->pathR0.alloc(c) && h->pathR1.alloc(c) &&
            h->pathL.alloc(c) && h->shO0.alloc(c) && h->shO1.alloc(c) &&
            h->shD0.alloc(c) && h->shD1.alloc(c) && h->shC0.alloc(c) && h->shC1.alloc(c) && h->pathPS0.alloc(c) && h->pathPS1.alloc(c) &&
            h->shO2.alloc(c) && h->shD2.alloc(c) && h->shC2.alloc(c) &&
            h->counters.alloc((size_t)(mi + 1) * kCountersPerIter) && h->error.alloc(1) && h->stats.alloc(8) &&
            h->curWave.alloc(1);
  if (!ok) {
    setLastError("out of device memory (wavefront queues)");
    return RG_ERR_OUT_OF_MEMORY;
  }
  h->capacity = (int)c;
  h->maxIter = mi;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
    h->graphKey.clear();
  }
  return RG_OK;
}

DevQueues makeQueues(rg_handle* h, int maxIter) {
  DevQueues Q;
  Q.rayO[0] = h->rayO0.p; Q.rayO[1] = h->rayO1.p;
  Q.rayD[0] = h->rayD0.p; Q.rayD[1] = h->rayD1.p;
  Q.hits = h->hits.p;
  Q.pathT[0] = h->pathT0.p; Q.pathT[1] = h->pathT1.p;
  Q.pathR[0] = h->pathR0.p; Q.pathR[1] = h->pathR1.p;
  Q.pathL = h->pathL.p;
  Q.pathPS[0] = h->pathPS0.p; Q.pathPS[1] = h->pathPS1.p;
  Q.shO[0] = h->shO0.p; Q.shO[1] = h->shO1.p; Q.shO[2] = h->shO2.p;
  Q.shD[0] = h->shD0.p; Q.shD[1] = h->shD1.p; Q.shD[2] = h->shD2.p;
  Q.shC[0] = h->shC0.p; Q.shC[1] = h->shC1.p; Q.shC[2] = h->shC2.p;
  Q.shO[3] = h->shO3.p; Q.shD[3] = h->shD3.p; Q.shC[3] = h->shC3.p;
  Q.counters = h->counters.p;
  Q.stats = h->stats.p;
  Q.error = h->error.p;
  Q.capacity = h->capacity;
  Q.maxIter = maxIter;
  return Q;
}

}  // namespace

DevRender makeRenderParams(const rg_settings& s, const rg_camera& c) {
  DevRender R;
  R.width = s.resolution_width;
  R.height = s.resolution_height;
  const float fov = std::fmin(std::fmax(c.field_of_view, 1.0f), 179.0f);
  R.viewScale = (2.0f * std::tan(fov * (3.14159265358979323846f / 180.0f) * 0.5f)) / (float)R.height;
  R.halfW = (float)R.width * 0.5f;
  R.halfH = (float)R.height * 0.5f;
  R.dof = c.depth_of_field;
  R.aperture = c.aperture > 0.0f ? 1.0f / c.aperture : 0.0f;
  R.blades = c.aperture_blades;
  R.apertureRot = c.aperture_rotation * (3.14159265358979323846f / 180.0f);
  R.exposure = c.exposure;
  R.viewFar = c.view_far;
  R.aa = s.enable_antialias;
  R.colorSampling = s.enable_color_sampling;
  R.shader = s.shader_provider;
  R.maxDepth = s.max_depth;
  R.rrDepth = s.rr_depth;
  R.lightFix = s.light_pick_fix;
  R.seed = s.seed;
  R.clampMax = s.firefly_clamp;
  R.backR = s.back_color[0]; R.backG = s.back_color[1]; R.backB = s.back_color[2];
  R.worldR = s.world_color[0]; R.worldG = s.world_color[1]; R.worldB = s.world_color[2];
  R.aoSamples = std::max(1, s.samples);
  return R;
}

namespace {

DevRender makeRender(const rg_handle* h) { return makeRenderParams(h->st, h->camera); }

// Shade / accumulate blocks per SM of grid (two of 256 threads are resident at 119
// registers; the rest follow in grid-stride windows); build-time overridable (-D).
#ifndef RG_SHADE_BLOCKS_PER_SM
#define RG_SHADE_BLOCKS_PER_SM 4
#endif
struct Grids {
  int gen, ext, shade, conn, acc, simple;
};

Grids grids(rg_handle* h) {
  Grids g;
  g.gen = h->numSMs * 8;
  g.ext = h->numSMs * residentBlocks(0, h->dscene.bvhWidth);
  g.shade = h->numSMs * RG_SHADE_BLOCKS_PER_SM;
  g.conn = h->numSMs * residentBlocks(1, h->dscene.bvhWidth);
  g.acc = h->numSMs * 4;
  g.simple = h->numSMs * 8;
  return g;
}

// Launch one wave's kernel sequence on the stream (captured or direct).
void enqueueWave(rg_handle* h, const DevRender& R, const DevQueues& Q, const DevJob* jobs, const DevWave* W, bool profile,
                 std::vector<cudaEvent_t>* ev) {
  const int shader = R.shader;
  const Grids g = grids(h);
  const cudaStream_t st = h->stream;
  const int width = h->dscene.bvhWidth;
  if (shader != 5) {
    launchSimple(jobs, W, Q, g.simple, st);
  } else {
    auto connects = [&](int it, cudaStream_t cs) {
      launchConnect(&h->dscene, jobs, width, Q, it, 0, g.conn, cs);
      if (h->dscene.numPointLights > 0) launchConnect(&h->dscene, jobs, width, Q, it, 1, g.conn, cs);
      if (h->dscene.envOn) launchConnect(&h->dscene, jobs, width, Q, it, 2, g.conn, cs);
      if (h->dscene.numVolLights > 0) launchConnect(&h->dscene, jobs, width, Q, it, 3, g.conn, cs);
    };
    launchGenerate(jobs, W, Q, g.gen, st);
    for (int it = 0; it < Q.maxIter; it++) {
      if (profile) {  // serial, one event between kernels
        cudaEventRecord((*ev)[it * 4 + 0], st);
        launchExtend(&h->dscene, jobs, width, Q, it, g.ext, st);
        cudaEventRecord((*ev)[it * 4 + 1], st);
        launchShade(&h->dscene, &R, jobs, Q, it, g.shade, st);
        cudaEventRecord((*ev)[it * 4 + 2], st);
        connects(it, st);
        cudaEventRecord((*ev)[it * 4 + 3], st);
        continue;
      }
      // the previous bounce's shadow rays (they only add into the path radiance)
      // run beside this bounce's closest hits; the shade kernel, which rewrites the
      // shadow queues and the radiance, waits for both
      if (it > 0) {
        cudaEventRecord(h->fork, st);
        cudaStreamWaitEvent(h->side, h->fork, 0);
        connects(it - 1, h->side);
        cudaEventRecord(h->join, h->side);
      }
      launchExtend(&h->dscene, jobs, width, Q, it, g.ext, st);
      if (it > 0) cudaStreamWaitEvent(st, h->join, 0);
      launchShade(&h->dscene, &R, jobs, Q, it, g.shade, st);
    }
    if (!profile && Q.maxIter > 0) connects(Q.maxIter - 1, st);
  }
  launchAccumulate(jobs, W, Q, g.acc, st);
  k_nextWave<<<1, 1, 0, st>>>(h->curWave.p);
}

}  // namespace
}  // namespace rg

// The wave descriptor array is indexed through *curWave by every kernel; the
// kernels take a pointer to the current element computed on the device.
namespace rg {
namespace {
__global__ void k_selectWave(const DevWave* waves, const int* cur, DevWave* slot) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *slot = waves[*cur];
}
}  // namespace
}  // namespace rg

extern "C" {

void rg_settings_default(rg_settings* s) {
  if (!s) return;
  std::memset(s, 0, sizeof(*s));
  s->resolution_width = 800;  // DEFAULT_RENDER_WIDTH / HEIGHT, rayrenderer.h:25-26
  s->resolution_height = 600;
  s->threads = 1;             // RENDER_THREADS (linux), rayrenderer.h:42-44
  s->samples = 100;           // TRACE_PATH_SAMPLES (linux)
  s->shader_provider = 5;
  s->enable_antialias = 1;
  s->enable_point_light_antialias = 1;
  s->enable_color_sampling = 1;
  s->enable_rendering_postprocess = 0;
  s->enable_denoise = 0;
  s->cull_back_face = 0;
  s->denoise_levels = 5;
  s->denoise_sigma_color = 0.4f;
  s->denoise_sigma_normal = 128.0f;
  s->denoise_sigma_depth = 0.1f;
  s->denoise_intensity = 1.0f;
  s->firefly_clamp = 10.0f;
  s->enable_adaptive_sampling = 0;
  s->adaptive_base_samples = 4;
  s->adaptive_threshold = 0.02f;
  s->adaptive_mode = RG_ADAPTIVE_TILE;
  s->bloom_threshold = 1.0f;
  s->bloom_strength = 1.0f;
  s->bloom_radius = 0.03f;
  s->bloom_size_aspect = 0.15f;
  s->bloom_curve = 1.0f;
  s->world_color[0] = 0.1f; s->world_color[1] = 0.095f; s->world_color[2] = 0.09f;
  s->back_color[0] = 0.2f; s->back_color[1] = 0.19f; s->back_color[2] = 0.18f; s->back_color[3] = 0.0f;
  s->seed = 1;
  s->max_depth = 32;          // MAX_TRACE_DEPTH, rayrenderer.cpp:38
  s->rr_depth = 3;            // MIN_RR_DEPTH, rayrenderer.cpp:41
  s->light_pick_fix = 0;
  s->paths_per_wave = 0;
  s->bvh_bins = 32;
  s->bvh_width = 8;
}

const char* rg_last_error(void) { return g_lastError.c_str(); }
const char* rg_version(void) { return "raygen-b200 0.1 (sm_100a wavefront tracer)"; }

rg_status rg_create(const rg_settings* s, rg_handle** out) {
  if (!out) return RG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    setLastError("no CUDA device");
    return RG_ERR_NO_DEVICE;
  }
  if (s && (s->denoise_levels < 1 || s->denoise_levels > kMaxDenoiseLevels)) {
    setLastError("rg_create: denoise_levels must be in [1, " + std::to_string(kMaxDenoiseLevels) + "]");
    return RG_ERR_INVALID_ARGUMENT;
  }
  rg_handle* h = new (std::nothrow) rg_handle();
  if (!h) return RG_ERR_OUT_OF_MEMORY;
  if (s) h->st = *s;
  else rg_settings_default(&h->st);
  cudaGetDevice(&h->device);
  cudaDeviceGetAttribute(&h->numSMs, cudaDevAttrMultiProcessorCount, h->device);
  keepPoolMemory();
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->join, cudaEventDisableTiming) != cudaSuccess) {
    setLastError("cudaStreamCreate failed");
    delete h;
    return RG_ERR_CUDA;
  }
  *out = h;
  return RG_OK;
}

rg_status rg_destroy(rg_handle* h) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(h->mu);
    if (h->stream) cudaStreamSynchronize(h->stream);
  }
  delete h;
  trimPoolMemory();
  return RG_OK;
}

rg_status rg_update_settings(rg_handle* h, const rg_settings* s) {
  if (!h || !s) return RG_ERR_INVALID_ARGUMENT;
  if (h->asyncBusy.load()) {
    setLastError("rg_update_settings: an rg_render_async job of this handle is in flight");
    return RG_ERR_BUSY;
  }
  if (s->denoise_levels < 1 || s->denoise_levels > kMaxDenoiseLevels) {
    setLastError("rg_update_settings: denoise_levels must be in [1, " + std::to_string(kMaxDenoiseLevels) + "]");
    return RG_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lk(h->mu);
  h->st = *s;
  return RG_OK;
}

rg_status rg_set_denoiser(rg_handle* h, rg_denoiser* d) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  h->denoiser = d;
  return RG_OK;
}

rg_status rg_set_progress_cb(rg_handle* h, rg_progress_fn fn, void* user) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  h->progress = fn;
  h->progressUser = user;
  return RG_OK;
}

rg_status rg_cancel(rg_handle* h) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  h->cancel.store(true);
  return RG_OK;
}

}  // extern "C"

namespace rg {

// Importance-sampling CDFs of an equirectangular map, Scene::buildEnvmapCDF
// (scene.cpp:414-463): per row, running sums of luminance x sin(theta) over
// the raw texels, normalised to a conditional CDF; a marginal CDF over the
// row sums.  Sequential float sums in texel order, as the reference.  A
// W x H map is a few hundred microseconds of host work at scene set-up.
// Returns false (no sampling) for an empty image.
bool buildEnvmapCdf(const rg_texture& T, std::vector<float>& marg, std::vector<float>& cond, float& total) {
  const int W = T.width, H = T.height;
  total = 0.0f;
  if (W <= 0 || H <= 0) return false;
  std::vector<float> rowWeight(H, 0.0f);
  cond.assign((size_t)H * (W + 1), 0.0f);
  for (int y = 0; y < H; y++) {
    const float v = (y + 0.5f) / (float)H;
    const float sinTheta = sinf((float)M_PI * v);
    float rowSum = 0.0f;
    for (int x = 0; x < W; x++) {
      const float* c = T.rgba + ((size_t)y * W + x) * 4;
      const float lum = fmaxf(0.0f, 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]);
      rowSum += lum * sinTheta;
      cond[(size_t)y * (W + 1) + (x + 1)] = rowSum;
    }
    rowWeight[y] = rowSum;
  }
  for (int y = 0; y < H; y++)
    if (rowWeight[y] > 0.0f) {
      const float inv = 1.0f / rowWeight[y];
      for (int x = 1; x <= W; x++) cond[(size_t)y * (W + 1) + x] *= inv;
    }
  marg.assign(H + 1, 0.0f);
  for (int y = 0; y < H; y++) marg[y + 1] = marg[y] + rowWeight[y];
  total = marg[H];
  if (total > 0.0f) {
    const float inv = 1.0f / total;
    for (int y = 0; y <= H; y++) marg[y] *= inv;
  }
  return true;
}

// Scene::buildEnvmapCDF, cubemap part (scene.cpp:343-410): per face, running
// row sums of luminance x the texel's solid angle 1/(s^2+t^2+1)^1.5, rows
// normalised to conditional CDFs, a per-face marginal over rows and a CDF over
// the face totals; raw texels, sequential float sums.
void buildCubeCdf(const rg_texture* faces[6], std::vector<float>& margFace, std::vector<float>& margY,
                  std::vector<float>& cond, float& total) {
  const int W = faces[0]->width, H = faces[0]->height;
  margFace.assign(7, 0.0f);
  margY.assign((size_t)6 * (H + 1), 0.0f);
  cond.assign((size_t)6 * H * (W + 1), 0.0f);
  float faceWeights[6] = {0, 0, 0, 0, 0, 0};
  for (int f = 0; f < 6; f++) {
    std::vector<float> rowWeight(H, 0.0f);
    for (int y = 0; y < H; y++) {
      float* c = &cond[((size_t)f * H + y) * (W + 1)];
      float rowSum = 0.0f;
      const float t = 1.0f - (y + 0.5f) * (2.0f / (float)H);
      for (int x = 0; x < W; x++) {
        const float sx = (x + 0.5f) * (2.0f / (float)W) - 1.0f;
        const float denom = sx * sx + t * t + 1.0f;
        const float jac = 1.0f / (denom * sqrtf(denom));
        const float* px = faces[f]->rgba + ((size_t)y * W + x) * 4;
        const float lum = fmaxf(0.0f, 0.2126f * px[0] + 0.7152f * px[1] + 0.0722f * px[2]);
        rowSum += lum * jac;
        c[x + 1] = rowSum;
      }
      if (rowSum > 0.0f) {
        const float inv = 1.0f / rowSum;
        for (int x = 1; x <= W; x++) c[x] *= inv;
      }
      rowWeight[y] = rowSum;
    }
    float* my = &margY[(size_t)f * (H + 1)];
    for (int y = 0; y < H; y++) my[y + 1] = my[y] + rowWeight[y];
    faceWeights[f] = my[H];
    if (faceWeights[f] > 0.0f) {
      const float inv = 1.0f / faceWeights[f];
      for (int y = 0; y <= H; y++) my[y] *= inv;
    }
  }
  total = 0.0f;
  for (int f = 0; f < 6; f++) total += faceWeights[f];
  if (total > 0.0f) {
    const float inv = 1.0f / total;
    float acc = 0.0f;
    for (int f = 0; f < 6; f++) {
      acc += faceWeights[f];
      margFace[f + 1] = acc * inv;
    }
  }
}

// Host-side phase timing printed to stderr when RG_TRACE_HOST is set.
struct HostTrace {
  bool on = std::getenv("RG_TRACE_HOST") != nullptr;
  double t0 = hostMs(), last = t0;
  void mark(const char* what) {
    if (!on) return;
    const double t = hostMs();
    std::fprintf(stderr, "[rg] %-32s +%8.3f ms (%8.3f ms)\n", what, t - last, t - t0);
    last = t;
  }
};

// Validates a scene description, uploads it, builds its BVH and fills the
// device-side table of pointers.  Used by rg_set_scene and the job server.
rg_status prepareScene(const rg_scene_desc* d, int bins, bool wide, cudaStream_t st, int* errWord,
                       std::unique_ptr<DeviceScene>& out, DevScene& S, Mat4& view, float* buildMs, bool keep) {
  HostTrace trace;
  const int nt = d->num_triangles;
  if (nt < 0 || d->num_meshes < 0 || d->num_objects < 0 || d->num_materials < 0 || d->num_media < 0 ||
      d->num_point_lights < 0 || d->num_textures < 0) {
    setLastError("negative count in scene description");
    return RG_ERR_INVALID_ARGUMENT;
  }
  if (nt > 0 && (!d->positions || !d->normals || !d->tri_mesh)) {
    setLastError("scene description without triangle arrays");
    return RG_ERR_INVALID_ARGUMENT;
  }
  if (nt >= (1 << 28)) {
    setLastError("more than 2^28 triangles");
    return RG_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < d->num_meshes; i++)
    if (d->mesh_object[i] < 0 || d->mesh_object[i] >= d->num_objects) {
      setLastError("mesh_object index out of range");
      return RG_ERR_INVALID_ARGUMENT;
    }
  for (int i = 0; i < d->num_objects; i++)
    if (d->objects[i].material < 0 || d->objects[i].material >= d->num_materials ||
        d->objects[i].interior_medium >= d->num_media) {
      setLastError("object material / medium index out of range");
      return RG_ERR_INVALID_ARGUMENT;
    }
  for (int i = 0; i < d->num_materials; i++)
    if (d->materials[i].texture >= d->num_textures) {
      setLastError("material texture index out of range");
      return RG_ERR_INVALID_ARGUMENT;
    }
  if (d->global_medium >= d->num_media || d->num_media > 1000) {
    setLastError("global medium index out of range");
    return RG_ERR_INVALID_ARGUMENT;
  }
  for (int i = 0; i < d->num_media; i++)
    if (d->media[i].num_path_points < 0 || d->media[i].num_path_points > 1024 ||
        (d->media[i].num_path_points > 0 && !d->media[i].path_points)) {
      setLastError("medium path points: count outside [0, 1024] or no array");
      return RG_ERR_INVALID_ARGUMENT;
    }
  for (int i = 0; i < d->num_textures; i++)
    if (d->textures[i].width < 0 || d->textures[i].height < 0 ||
        (d->textures[i].width > 0 && d->textures[i].height > 0 && !d->textures[i].rgba)) {
      setLastError("texture without texels");
      return RG_ERR_INVALID_ARGUMENT;
    }
  if (d->has_envmap && (d->envmap_texture < 0 || d->envmap_texture >= d->num_textures)) {
    setLastError("envmap texture index out of range");
    return RG_ERR_INVALID_ARGUMENT;
  }
  if (d->envmap_cube) {
    for (int f = 0; f < 6; f++) {
      const int t = d->envmap_cube_faces[f];
      if (t < 0 || t >= d->num_textures) {
        setLastError("cubemap face texture index out of range");
        return RG_ERR_INVALID_ARGUMENT;
      }
      const rg_texture& T = d->textures[t];
      const rg_texture& T0 = d->textures[d->envmap_cube_faces[0]];
      if (T.width <= 0 || T.width != T.height || T.width != T0.width) {
        setLastError("cubemap faces must be square and of one size");
        return RG_ERR_INVALID_ARGUMENT;
      }
    }
  }
  // one pass over the triangles: mesh index check, triangles per mesh, and the
  // triangles of emissive meshes (area lights, rayrenderer.cpp:333-353: emissive
  // objects with meshes, object order)
  std::vector<int> objMat(d->num_objects);
  for (int i = 0; i < d->num_objects; i++) objMat[i] = d->objects[i].material;
  std::vector<std::vector<int>> objMeshes(d->num_objects);
  for (int i = 0; i < d->num_meshes; i++) objMeshes[d->mesh_object[i]].push_back(i);
  std::vector<char> isLightMesh(d->num_meshes, 0);
  for (int o = 0; o < d->num_objects; o++)
    if (d->materials[objMat[o]].emission > 0.0f)
      for (int m : objMeshes[o]) isLightMesh[m] = 1;
  trace.mark("scene: checks");
  // the previous scene's memory is reused (keep, unless the new scene has less
  // than half its triangles) or goes back to the pool; the triangle arrays start
  // copying now and the host pass below runs while they are in flight
  {
    std::unique_ptr<DeviceScene> next(new DeviceScene());
    if (keep && out && 2 * (int64_t)nt >= (int64_t)out->numTris) next->adoptBuffers(*out);
    next->keepBuffers = keep;
    out = std::move(next);
  }
  trace.mark("scene: previous scene replaced");
  DeviceScene& ds = *out;
  ds.numTris = nt;
  ds.hasUV = d->uvs != nullptr && d->num_textures > 0;
  bool ok = ds.inPos.upload(d->positions, (size_t)nt * 9, st) && ds.inNrm.upload(d->normals, (size_t)nt * 9, st) &&
            ds.inTriMesh.upload(d->tri_mesh, nt, st);
  if (ok && ds.hasUV) ok = ds.inUV.upload(d->uvs, (size_t)nt * 6, st);
  if (!ok) {
    cudaStreamSynchronize(st);
    setLastError("scene upload failed (device memory)");
    out.reset();
    return RG_ERR_OUT_OF_MEMORY;
  }
  trace.mark("scene: triangle copies issued");
  std::vector<int> meshTriCount(d->num_meshes, 0);
  std::vector<std::vector<int>> meshTris(d->num_meshes);
  // runs of equal mesh ids (a mesh's triangles are usually consecutive) are counted
  // in a register and checked once
  int runMesh = -1, run = 0;
  bool runLight = false;
  for (int i = 0; i < nt; i++) {
    const int m = d->tri_mesh[i];
    if (m != runMesh) {
      if (m < 0 || m >= d->num_meshes) {
        cudaStreamSynchronize(st);  // no copy into the buffers freed below is in flight
        setLastError("tri_mesh index out of range");
        out.reset();
        return RG_ERR_INVALID_ARGUMENT;
      }
      if (runMesh >= 0) meshTriCount[runMesh] += run;
      runMesh = m;
      run = 0;
      runLight = isLightMesh[m] != 0;
    }
    run++;
    if (runLight) meshTris[m].push_back(i);
  }
  if (runMesh >= 0) meshTriCount[runMesh] += run;
  trace.mark("scene: triangle pass");
  view = viewMatrix(d->camera);
  std::vector<DevMaterial> mats(d->num_materials);
  for (int i = 0; i < d->num_materials; i++) mats[i] = toDev(d->materials[i]);
  MediaTables MT;
  buildMedia(d, view, MT);
  std::vector<int>& objMed = MT.objMed;
  std::vector<DevMedium>& media = MT.media;
  ds.globalMedium = MT.globalMedium;
  ds.hasHaze = MT.hasHaze;
  // area lights (rayrenderer.cpp:333-353): emissive objects with meshes, object order
  std::vector<int> areaLightObj, lightMeshList;
  std::vector<int2> lightObjMeshes(std::max(1, d->num_objects), make_int2(0, 0));
  std::vector<int2> lightMeshTris(std::max(1, d->num_meshes), make_int2(0, 0));
  std::vector<float4> lightTris;
  {
    for (int o = 0; o < d->num_objects; o++) {
      if (!(d->materials[objMat[o]].emission > 0.0f) || objMeshes[o].empty()) continue;
      areaLightObj.push_back(o);
      lightObjMeshes[o] = make_int2((int)lightMeshList.size(), (int)objMeshes[o].size());
      for (int m : objMeshes[o]) lightMeshList.push_back(m);
    }
    for (int m = 0; m < d->num_meshes; m++) {
      if (!isLightMesh[m]) continue;
      lightMeshTris[m] = make_int2((int)(lightTris.size() / 6), (int)meshTris[m].size());
      for (int i : meshTris[m]) {
        float v[3][3], n[3][3];
        for (int k = 0; k < 3; k++) {
          xformPoint(view, &d->positions[(size_t)i * 9 + k * 3], v[k]);
          xformDir(view, &d->normals[(size_t)i * 9 + k * 3], n[k]);
        }
        const F3h v1{v[0][0], v[0][1], v[0][2]}, v2{v[1][0], v[1][1], v[1][2]}, v3_{v[2][0], v[2][1], v[2][2]};
        const float tia = 1.0f / len(crs(sub(v1, v2), sub(v1, v3_)));
        const float area = 0.5f * len(crs(sub(v2, v1), sub(v3_, v1)));
        lightTris.push_back(make_float4(v1.x, v1.y, v1.z, tia));
        lightTris.push_back(make_float4(v2.x, v2.y, v2.z, area));
        lightTris.push_back(make_float4(v3_.x, v3_.y, v3_.z, 0.0f));
        for (int k = 0; k < 3; k++) lightTris.push_back(make_float4(n[k][0], n[k][1], n[k][2], 0.0f));
      }
    }
  }
  std::vector<DevPointLight> pts(d->num_point_lights);
  for (int i = 0; i < d->num_point_lights; i++) {
    float p[3], n[3];
    xformPoint(view, d->point_lights[i].position, p);
    xformDir(view, d->point_lights[i].normal, n);
    pts[i] = DevPointLight{p[0], p[1], p[2], n[0], n[1], n[2], d->point_lights[i].material, 0};
  }
  trace.mark("scene: tables");
  ok = ds.meshTriCount.upload(meshTriCount.data(), meshTriCount.size(), st) &&
            ds.meshObj.upload(d->mesh_object, d->num_meshes, st) && ds.objMat.upload(objMat.data(), objMat.size(), st) &&
            ds.objMedium.upload(objMed.data(), objMed.size(), st) && ds.mats.upload(mats.data(), mats.size(), st) &&
            ds.media.upload(media.data(), media.size(), st) && ds.pathPts.upload(MT.pts.data(), MT.pts.size(), st) &&
            ds.volLights.upload(MT.vols.data(), MT.vols.size(), st) &&
            ds.areaLightObj.upload(areaLightObj.data(), areaLightObj.size(), st) &&
            ds.lightMeshList.upload(lightMeshList.data(), lightMeshList.size(), st) &&
            ds.lightObjMeshes.upload(lightObjMeshes.data(), lightObjMeshes.size(), st) &&
            ds.lightMeshTris.upload(lightMeshTris.data(), lightMeshTris.size(), st) &&
            ds.lightTris.upload(lightTris.data(), lightTris.size(), st) && ds.points.upload(pts.data(), pts.size(), st) &&
            ds.view.upload(view.m, 16, st);
  // textures
  std::vector<DevTexture> texs(d->num_textures);
  for (int i = 0; ok && i < d->num_textures; i++) {
    const rg_texture& t = d->textures[i];
    if ((size_t)i >= ds.texels.size()) ds.texels.push_back(new DevBuf<float4>());
    DevBuf<float4>* buf = ds.texels[i];
    const size_t cnt = (size_t)std::max(0, t.width) * std::max(0, t.height);
    ok = buf->upload(reinterpret_cast<const float4*>(t.rgba), cnt, st);
    texs[i] = DevTexture{buf->p, t.width, t.height, t.is_hdr, 0};
  }
  // texels adopted from a scene with more textures
  while (ok && ds.texels.size() > (size_t)d->num_textures) {
    delete ds.texels.back();
    ds.texels.pop_back();
  }
  if (ok) ok = ds.textures.upload(texs.data(), texs.size(), st);
  if (ok && (d->has_envmap || d->envmap_cube)) {
    ds.envIntensity = d->envmap_intensity;
    const float yaw = d->envmap_rotation * (float)(M_PI / 180.0);
    ds.envCosY = cosf(yaw);
    ds.envSinY = sinf(yaw);
  }
  if (ok && d->envmap_cube) {
    const rg_texture* faces[6];
    for (int f = 0; f < 6; f++) {
      faces[f] = &d->textures[d->envmap_cube_faces[f]];
      ds.envFace[f] = d->envmap_cube_faces[f];
    }
    ds.envCube = 1;
    std::vector<float> mf, my, mc;
    buildCubeCdf(faces, mf, my, mc, ds.envCubeTotal);
    ds.envCubeW = faces[0]->width;
    ok = ds.cubeMargFace.upload(mf.data(), mf.size(), st) && ds.cubeMargY.upload(my.data(), my.size(), st) &&
         ds.cubeCond.upload(mc.data(), mc.size(), st);
    if (ok) ok = cudaStreamSynchronize(st) == cudaSuccess;
  }
  if (ok && d->has_envmap) {
    const rg_texture& T = d->textures[d->envmap_texture];
    std::vector<float> marg, cond;
    ds.envTex = d->envmap_texture;
    if (buildEnvmapCdf(T, marg, cond, ds.envTotal)) {
      ds.envW = T.width;
      ds.envH = T.height;
      ok = ds.envMarg.upload(marg.data(), marg.size(), st) && ds.envCond.upload(cond.data(), cond.size(), st);
      // the host vectors go out of scope: finish the copies first
      if (ok) ok = cudaStreamSynchronize(st) == cudaSuccess;
    }
  }
  if (!ok) {
    cudaStreamSynchronize(st);  // no copy into the buffers freed below is in flight
    setLastError("scene upload failed (device memory)");
    out.reset();
    return RG_ERR_OUT_OF_MEMORY;
  }
  trace.mark("scene: uploads issued");
  ds.numAreaLights = (int)areaLightObj.size();
  ds.numPointLights = (int)pts.size();
  ds.numTextures = d->num_textures;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  std::string err;
  const rg_status rs = buildDeviceBvh(ds, bins > 1 ? bins : 32, wide, st, err);
  trace.mark("scene: build launched");
  cudaEventRecord(e1, st);
  cudaStreamSynchronize(st);
  trace.mark("scene: build done");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rs != RG_OK) {
    setLastError(err);
    out.reset();
    return rs;
  }
  if (buildMs) *buildMs = ms;
  if (!keep) {
    ds.inPos.release();
    ds.inNrm.release();
    ds.inUV.release();
    ds.inTriMesh.release();
    freeBvhScratch(ds.scratch);
    ds.scratch = nullptr;
  }
  std::memset(&S, 0, sizeof(S));
  S.nodes = ds.nodes.p;
  S.numNodes = ds.numNodes;
  S.rootIsLeaf = ds.rootIsLeaf;
  S.rootLeafRef = ds.rootLeafRef;
  S.triVerts = ds.triVerts.p;
  S.triShade = ds.triShade.p;
  S.triUV = ds.hasUV ? ds.triUV.p : nullptr;
  S.triOrig = ds.triOrig.p;
  S.numTris = nt;
  S.meshObj = ds.meshObj.p;
  S.meshTriCount = ds.meshTriCount.p;
  S.objMat = ds.objMat.p;
  S.objMedium = ds.objMedium.p;
  S.mats = ds.mats.p;
  S.media = ds.media.p;
  S.numMedia = d->num_media;
  S.globalMedium = ds.globalMedium;
  S.pathPts = ds.pathPts.p;
  S.volLights = ds.volLights.p;
  S.numVolLights = (int)MT.vols.size();
  S.mediaLevel = MT.level;
  S.numAreaLights = ds.numAreaLights;
  S.areaLightObj = ds.areaLightObj.p;
  S.lightObjMeshes = ds.lightObjMeshes.p;
  S.lightMeshList = ds.lightMeshList.p;
  S.lightMeshTris = ds.lightMeshTris.p;
  S.lightTris = ds.lightTris.p;
  S.numPointLights = ds.numPointLights;
  S.points = ds.points.p;
  S.textures = ds.textures.p;
  S.numTextures = ds.numTextures;
  S.error = errWord;
  S.nodes8 = ds.nodes8.p;
  S.numNodes8 = ds.numNodes8;
  S.bvhWidth = ds.bvhWidth;
  S.envTex = ds.envTex;
  S.envW = ds.envW;
  S.envH = ds.envH;
  S.envIntensity = ds.envIntensity;
  S.envCosY = ds.envCosY;
  S.envSinY = ds.envSinY;
  S.envTotal = ds.envTotal;
  S.envMarg = ds.envMarg.p;
  S.envCond = ds.envCond.p;
  S.envOn = (ds.envTex >= 0 || ds.envCube) ? 1 : 0;
  S.envCube = ds.envCube;
  for (int f = 0; f < 6; f++) S.envFace[f] = ds.envFace[f];
  S.envCubeW = ds.envCubeW;
  S.envCubeTotal = ds.envCubeTotal;
  S.cubeMargFace = ds.cubeMargFace.p;
  S.cubeMargY = ds.cubeMargY.p;
  S.cubeCond = ds.cubeCond.p;
  // per-triangle shading class and material (the shade kernel's sort key)
  if (!ds.triMat.alloc((size_t)std::max(1, nt))) {
    setLastError("scene upload failed (device memory)");
    out.reset();
    return RG_ERR_OUT_OF_MEMORY;
  }
  S.triMat = ds.triMat.p;
  if (nt > 0) launchTriMaterial(S, nt, ds.triMat.p, st);
  return RG_OK;
}

}  // namespace rg

extern "C" {

rg_status rg_set_scene(rg_handle* h, const rg_scene_desc* d) {
  if (!h || !d) return RG_ERR_INVALID_ARGUMENT;
  if (h->asyncBusy.load()) {
    setLastError("rg_set_scene: an rg_render_async job of this handle is in flight");
    return RG_ERR_BUSY;
  }
  std::lock_guard<std::mutex> lk(h->mu);
  h->hasScene = false;
  h->haveResult = false;
  if (!h->error.alloc(1)) return RG_ERR_OUT_OF_MEMORY;
  cudaMemsetAsync(h->error.p, 0, sizeof(int), h->stream);
  float ms = 0.0f;
  const rg_status rs = prepareScene(d, h->st.bvh_bins, h->st.bvh_width != 2, h->stream, h->error.p, h->scene,
                                    h->dscene, h->view, &ms, /*keep=*/true);
  if (rs != RG_OK) return rs;
  h->camera = d->camera;
  h->lastStats.build_ms = ms;
  h->lastStats.bvh_nodes = h->scene->bvhWidth == 8 ? h->scene->numNodes8 : h->scene->numNodes;
  h->hasScene = true;
  h->graphKey.clear();  // the wave graph carries the scene in its kernel parameters: recapture, then update
  return RG_OK;
}

// Keeps the denoised, not yet bloomed HDR (RayRenderer::preBloomHdrImage) and
// applies the bloom when post-processing is on (rayrenderer.cpp:584-592).
static rg_status postProcess(rg_handle* h, bool restore) {
  const rg_settings& s = h->st;
  const int W = h->W, H = h->H;
  const size_t N = (size_t)W * H;
  cudaStream_t st = h->stream;
  if (restore) {
    RG_CUDA_CHECK(cudaMemcpyAsync(h->hdr.p, h->preBloom.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
  } else {
    if (!h->preBloom.alloc(N)) {
      setLastError("out of device memory (pre-bloom copy)");
      return RG_ERR_OUT_OF_MEMORY;
    }
    RG_CUDA_CHECK(cudaMemcpyAsync(h->preBloom.p, h->hdr.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
  }
  if (s.enable_rendering_postprocess) {
    const BloomPlan p = planBloom(W, H, s.bloom_radius, s.bloom_size_aspect);
    const size_t n = (size_t)p.gw * p.gh;
    if (!h->bloomA.alloc(n) || !h->bloomB.alloc(n) || !h->bloomW.alloc(std::max<size_t>(1, p.weights.size()))) {
      setLastError("out of device memory (bloom buffers)");
      return RG_ERR_OUT_OF_MEMORY;
    }
    if (!p.weights.empty())  // pageable source: staged before the call returns
      RG_CUDA_CHECK(cudaMemcpyAsync(h->bloomW.p, p.weights.data(), sizeof(float) * p.weights.size(),
                                    cudaMemcpyHostToDevice, st));
    launchBloom(W, H, h->hdr.p, p, h->bloomW.p, s.bloom_threshold, s.bloom_strength, s.bloom_curve, h->bloomA.p,
                h->bloomB.p, st);
  }
  return RG_OK;
}

// Automatic wave size: large waves amortise the few-ray tail of the last
// bounces (measured on the 1080p 4M-triangle job: 8 Mi paths 239, 16 Mi 255,
// 32 Mi 264, 64 Mi 269 Msamples/s); bounded by a fifth of the free memory.
static long long wavePaths(const rg_settings& s) {
  if (s.paths_per_wave > 0) return s.paths_per_wave;
  constexpr long long kBytesPerPath = 370;  // rays / hits / path state (double-buffered) and four shadow queues
  long long cap = 64ll << 20;
  size_t freeB = 0, totalB = 0;
  if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess) {
    const long long fit = (long long)(freeB / 5) / kBytesPerPath;
    while (cap > (1ll << 20) && cap > fit) cap >>= 1;
  }
  cudaGetLastError();
  return cap;
}

// `start` is recorded on the stream right before the render's first wave (once
// per render, `started`), after this pass's host-side set-up: the render's
// device time then covers the device work and the waits between passes, not
// the host's preparation of the first one.
static rg_status runPass(rg_handle* h, const DevRender& R, int numPixels, const int* pixelList, int spp,
                         int& wavesDone, int totalWavesHint, bool profile, double* kernelMs, cudaEvent_t start,
                         bool& started) {
  if (numPixels <= 0 || spp <= 0) return RG_OK;
  HostTrace trace;
  const long long cap = wavePaths(h->st);
  trace.mark("pass: wave size");
  std::vector<DevSegment> sg;
  const int spw = numPixels >= cap ? 1 : (int)std::min<long long>(spp, std::max<long long>(1, cap / numPixels));
  const int pixChunk = (int)std::min<long long>(numPixels, cap);
  for (int s = 0; s < spp; s += spw)
    for (int p = 0; p < numPixels; p += pixChunk) {
      DevSegment e;
      e.slot = 0;
      e.numPixels = std::min(pixChunk, numPixels - p);
      e.samples = std::min(spw, spp - s);
      e.pathBase = 0;
      e.pixelOffset = p;
      e.pixBase = 0;
      e.pixelList = pixelList;
      sg.push_back(e);
    }
  if (!h->segs.alloc(sg.size())) {
    setLastError("out of device memory (segments)");
    return RG_ERR_OUT_OF_MEMORY;
  }
  std::vector<DevWave> ws(sg.size());
  for (size_t k = 0; k < sg.size(); k++) {
    ws[k].numSegments = 1;
    ws[k].numPaths = sg[k].numPixels * sg[k].samples;
    ws[k].numPixelsTotal = sg[k].numPixels;
    ws[k].pad = 0;
    ws[k].segs = h->segs.p + k;
  }
  RG_CUDA_CHECK(cudaMemcpyAsync(h->segs.p, sg.data(), sg.size() * sizeof(DevSegment), cudaMemcpyHostToDevice, h->stream));
  const int capacity = std::min<long long>(cap, (long long)pixChunk * spw);
  // one segment per vertex plus the eye ray; a heat-haze crossing adds a
  // segment without a vertex, at most one per medium entry
  const int maxIter = h->scene->hasHaze ? 2 * R.maxDepth + 3 : R.maxDepth + 2;
  rg_status rs = ensureQueues(h, capacity, maxIter, h->dscene.numVolLights > 0);
  if (rs != RG_OK) return rs;
  trace.mark("pass: queues");
  if (!h->waves.alloc(ws.size() + 1)) {
    setLastError("out of device memory (waves)");
    return RG_ERR_OUT_OF_MEMORY;
  }
  RG_CUDA_CHECK(cudaMemcpyAsync(h->waves.p, ws.data(), ws.size() * sizeof(DevWave), cudaMemcpyHostToDevice, h->stream));
  RG_CUDA_CHECK(cudaMemsetAsync(h->curWave.p, 0, sizeof(int), h->stream));
  const DevQueues Q = makeQueues(h, maxIter);
  // the single job of this handle
  if (!h->jobsDev.alloc(1)) return RG_ERR_OUT_OF_MEMORY;
  {
    DevJob J;
    std::memset(&J, 0, sizeof(J));
    J.S = h->dscene;
    J.R = R;
    J.sum = h->sum.p;
    J.sumSq = h->sumSq.p;
    J.cnt = h->cnt.p;
    RG_CUDA_CHECK(cudaMemcpyAsync(h->jobsDev.p, &J, sizeof(J), cudaMemcpyHostToDevice, h->stream));
    RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  }
  trace.mark("pass: job copied");
  // the kernels read the current wave from a fixed one-element slot
  if (!h->waveSlot.alloc(1)) return RG_ERR_OUT_OF_MEMORY;
  DevWave* slot = h->waveSlot.p;
  std::vector<cudaEvent_t> ev;
  if (profile) {
    ev.resize((size_t)maxIter * 4);
    for (auto& e : ev) cudaEventCreate(&e);
  }
  // graph of one wave: select the wave descriptor, then the kernel sequence
  const std::string key = std::to_string((uintptr_t)h->waves.p) + ":" + std::to_string((uintptr_t)slot) + ":" +
                          std::to_string(maxIter) + ":" + std::to_string(R.shader) + ":" + std::to_string(h->capacity) +
                          ":" + std::to_string((uintptr_t)pixelList) + ":" + std::to_string((uintptr_t)h->jobsDev.p) + ":" +
                          std::to_string((uintptr_t)h->shO3.p) + ":" + std::string((const char*)&R, sizeof(R));
  if (!profile && (h->graph == nullptr || h->graphKey != key)) {
    cudaGraph_t g;
    RG_CUDA_CHECK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    k_selectWave<<<1, 1, 0, h->stream>>>(h->waves.p, h->curWave.p, slot);
    enqueueWave(h, R, Q, h->jobsDev.p, slot, false, nullptr);
    RG_CUDA_CHECK(cudaStreamEndCapture(h->stream, &g));
    // same kernel sequence with new parameters (a new scene, new settings):
    // update the instantiated graph in place; otherwise instantiate anew
    bool updated = false;
    if (h->graph) {
      cudaGraphExecUpdateResultInfo info;
      updated = cudaGraphExecUpdate(h->graph, g, &info) == cudaSuccess;
      if (!updated) {
        cudaGetLastError();
        cudaGraphExecDestroy(h->graph);
        h->graph = nullptr;
      }
    }
    const cudaError_t ie = updated ? cudaSuccess : cudaGraphInstantiate(&h->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      setLastError(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
      h->graph = nullptr;
      return RG_ERR_CUDA;
    }
    h->graphKey = key;
    trace.mark("pass: wave graph captured");
  }
  // Waves are paced: wave k is launched, then the host waits for wave k-1.  One
  // wave stays queued behind the running one (the device never idles), while
  // progress is reported for completed waves and a cancel stops the render
  // within one wave.
  for (int e = 0; e < 2; e++)
    if (!h->waveDone[e]) RG_CUDA_CHECK(cudaEventCreateWithFlags(&h->waveDone[e], cudaEventDisableTiming));
  auto reportProgress = [&](int completed) {
    const float pr = totalWavesHint > 0 ? std::min(1.0f, (float)completed / (float)totalWavesHint) : 0.0f;
    if (pr > h->progressValue.load()) h->progressValue.store(pr);
    if (h->progress) h->progress(h->progressValue.load(), h->progressUser);
  };
  for (size_t k = 0; k < ws.size(); k++) {
    if (h->cancel.load()) return RG_ERR_CANCELLED;
    if (!started) {
      cudaEventRecord(start, h->stream);
      started = true;
      h->firstWaveHostMs = hostMs();
    }
    if (profile) {
      k_selectWave<<<1, 1, 0, h->stream>>>(h->waves.p, h->curWave.p, slot);
      enqueueWave(h, R, Q, h->jobsDev.p, slot, true, &ev);
      RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
      if (R.shader == 5) {
        for (int it = 0; it < maxIter; it++) {
          float a = 0, b = 0, c = 0;
          cudaEventElapsedTime(&a, ev[it * 4 + 0], ev[it * 4 + 1]);
          cudaEventElapsedTime(&b, ev[it * 4 + 1], ev[it * 4 + 2]);
          cudaEventElapsedTime(&c, ev[it * 4 + 2], ev[it * 4 + 3]);
          kernelMs[0] += a;
          kernelMs[1] += b;
          kernelMs[2] += c;
        }
      }
    } else {
      RG_CUDA_CHECK(cudaGraphLaunch(h->graph, h->stream));
    }
    RG_CUDA_CHECK(cudaEventRecord(h->waveDone[wavesDone & 1], h->stream));
    wavesDone++;
    if (wavesDone >= 2) {
      RG_CUDA_CHECK(cudaEventSynchronize(h->waveDone[wavesDone & 1]));  // wave wavesDone-2 of the render
      reportProgress(wavesDone - 1);
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  return RG_OK;
}

namespace {

// Host-side phase marks of a render, printed to stderr when RG_TRACE_HOST is
// set (for finding host stalls between the call and the first wave).

// The render itself; the caller holds h->mu.
rg_status renderLocked(rg_handle* h) {
  const double tEntry = hostMs();
  h->firstWaveHostMs = 0.0;
  HostTrace trace;
  const rg_settings& s = h->st;
  if (s.shader_provider == 4) {
    setLastError("shader 4 is reserved (no provider in the reference)");
    return RG_ERR_UNSUPPORTED;
  }
  if (s.shader_provider < 0 || s.shader_provider > 5) {
    setLastError("unknown shader id");
    return RG_ERR_INVALID_ARGUMENT;
  }
  if (!h->hasScene) {
    setLastError("no scene set");
    return RG_ERR_NO_SCENE;
  }
  if (s.resolution_width <= 0 || s.resolution_height <= 0 ||
      (long long)s.resolution_width * s.resolution_height > (1ll << 28) || s.max_depth < 1 || s.max_depth > 250 ||
      s.samples < 0) {
    setLastError("invalid resolution / depth / samples");
    return RG_ERR_INVALID_ARGUMENT;
  }
  h->cancel.store(false);
  h->haveResult = false;
  h->progressValue.store(0.0f);
  const int W = s.resolution_width, H = s.resolution_height, N = W * H;
  const bool profile = std::getenv("RG_PROFILE_KERNELS") != nullptr;
  if (!h->sum.alloc(N) || !h->sumSq.alloc(N) || !h->cnt.alloc(N) || !h->hdr.alloc(N) || !h->ldr.alloc(N) ||
      !h->pixelList.alloc(N) || !h->listCount.alloc(1)) {
    setLastError("out of device memory (image buffers)");
    return RG_ERR_OUT_OF_MEMORY;
  }
  h->W = W;
  h->H = H;
  cudaStream_t st = h->stream;
  RG_CUDA_CHECK(cudaMemsetAsync(h->sum.p, 0, sizeof(float4) * N, st));
  RG_CUDA_CHECK(cudaMemsetAsync(h->sumSq.p, 0, sizeof(float4) * N, st));
  RG_CUDA_CHECK(cudaMemsetAsync(h->cnt.p, 0, sizeof(int) * N, st));
  trace.mark("image buffers");
  DevRender R = makeRender(h);
  // stats reset
  if (!h->stats.alloc(8) || !h->error.alloc(1)) return RG_ERR_OUT_OF_MEMORY;
  RG_CUDA_CHECK(cudaMemsetAsync(h->stats.p, 0, sizeof(unsigned long long) * 8, st));
  RG_CUDA_CHECK(cudaMemsetAsync(h->error.p, 0, sizeof(int), st));
  if (s.enable_denoise) {
    if (!h->aovNormal.alloc((size_t)N * 3) || !h->aovAlbedo.alloc((size_t)N * 3) || !h->aovAlbedoA.alloc(N) ||
        !h->aovDepth.alloc(N) || !h->bufA.alloc(N) || !h->bufB.alloc(N)) {
      setLastError("out of device memory (denoise buffers)");
      return RG_ERR_OUT_OF_MEMORY;
    }
    launchAov(h->dscene, R, h->aovNormal.p, h->aovAlbedo.p, h->aovAlbedoA.p, h->aovDepth.p, st);
  }
  cudaEvent_t t0, t1, t2;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  cudaEventCreate(&t2);
  bool started = false;  // t0 is recorded by runPass right before the first wave
  int wavesDone = 0;
  double kms[3] = {0, 0, 0};
  rg_status rs = RG_OK;
  const int target = std::max(0, s.samples);
  if (!s.enable_adaptive_sampling) {
    const long long cap = wavePaths(s);
    const int spw = N >= cap ? 1 : (int)std::min<long long>(std::max(1, target), std::max<long long>(1, cap / N));
    const int hint = (int)(((target + spw - 1) / std::max(1, spw)) * ((N + cap - 1) / cap));
    rs = runPass(h, R, N, nullptr, target, wavesDone, hint, profile, kms, t0, started);
  } else {
    // renderAdaptive (rayrenderer.cpp:1162-1252): base pass, then refinement passes
    const int base = std::max(1, s.adaptive_base_samples);
    int spent = std::min(base, target);
    rs = runPass(h, R, N, nullptr, spent, wavesDone, 0, profile, kms, t0, started);
    while (rs == RG_OK && spent < target) {
      RG_CUDA_CHECK(cudaMemsetAsync(h->listCount.p, 0, sizeof(int), st));
      if (s.adaptive_mode == RG_ADAPTIVE_TILE)
        launchAdaptiveTiles(W, H, h->sum.p, h->sumSq.p, h->cnt.p, target, s.adaptive_threshold, h->pixelList.p,
                            h->listCount.p, st);
      else
        launchAdaptivePixels(N, h->sum.p, h->sumSq.p, h->cnt.p, target, s.adaptive_threshold, h->pixelList.p,
                             h->listCount.p, st);
      int active = 0;
      RG_CUDA_CHECK(cudaMemcpyAsync(&active, h->listCount.p, sizeof(int), cudaMemcpyDeviceToHost, st));
      RG_CUDA_CHECK(cudaStreamSynchronize(st));
      if (active == 0) break;
      const int passCount = std::min(base, target - spent);
      rs = runPass(h, R, active, h->pixelList.p, passCount, wavesDone, 0, profile, kms, t0, started);
      spent += passCount;
    }
  }
  trace.mark("waves launched");
  if (!started) cudaEventRecord(t0, st);  // no wave ran (0 samples)
  cudaEventRecord(t1, st);
  if (rs != RG_OK) {
    cudaStreamSynchronize(st);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaEventDestroy(t2);
    return rs;
  }
  launchResolve(N, h->sum.p, h->cnt.p, h->camera.exposure, h->hdr.p, st);
  if (s.enable_denoise && h->denoiser) {
    const rg_status ds = kpcnDenoiseDevice(*kpcnOf(h->denoiser), W, H, h->hdr.p, h->aovNormal.p, h->aovAlbedo.p,
                                           h->aovDepth.p, h->cnt.p, s.denoise_intensity, h->ldr.p, st);
    if (ds != RG_OK) {
      cudaStreamSynchronize(st);
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      cudaEventDestroy(t2);
      return ds;
    }
    RG_CUDA_CHECK(cudaMemcpyAsync(h->hdr.p, h->ldr.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
  } else if (s.enable_denoise) {
    launchDenoise(W, H, h->hdr.p, h->aovNormal.p, h->aovDepth.p, h->aovAlbedo.p, h->aovAlbedoA.p, s.denoise_levels,
                  s.denoise_sigma_color, s.denoise_sigma_normal, s.denoise_sigma_depth, s.denoise_intensity, h->bufA.p,
                  h->bufB.p, h->ldr.p, st);
    RG_CUDA_CHECK(cudaMemcpyAsync(h->hdr.p, h->ldr.p, sizeof(float4) * N, cudaMemcpyDeviceToDevice, st));
  }
  {
    const rg_status ps = postProcess(h, false);
    if (ps != RG_OK) {
      cudaStreamSynchronize(st);
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
      cudaEventDestroy(t2);
      return ps;
    }
  }
  launchTonemap(N, h->hdr.p, h->ldr.p, st);
  cudaEventRecord(t2, st);
  k_sumCounts<<<std::min((N + 255) / 256, 4 * 148), 256, 0, st>>>(N, h->cnt.p, h->stats.p + 6);
  trace.mark("post launched");
  const cudaError_t se = cudaStreamSynchronize(st);
  trace.mark("stream synchronised");
  float traceMs = 0, postMs = 0;
  cudaEventElapsedTime(&traceMs, t0, t1);
  cudaEventElapsedTime(&postMs, t1, t2);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(t2);
  if (se != cudaSuccess) {
    setLastError(std::string("render failed: ") + cudaGetErrorString(se));
    return RG_ERR_CUDA;
  }
  unsigned long long stv[8] = {0};
  int derr = 0;
  cudaMemcpy(stv, h->stats.p, sizeof(stv), cudaMemcpyDeviceToHost);
  cudaMemcpy(&derr, h->error.p, sizeof(int), cudaMemcpyDeviceToHost);
  rg_stats& S = h->lastStats;
  S.trace_ms = traceMs;
  S.post_ms = postMs;
  S.nodes_visited = stv[0];
  S.tris_tested = stv[1];
  S.shadow_nodes_visited = stv[2];
  S.shadow_tris_tested = stv[3];
  S.closest_rays = stv[4];
  S.shadow_rays = stv[5];
  S.extend_ms = kms[0];
  S.shade_ms = kms[1];
  S.connect_ms = kms[2];
  S.waves = wavesDone;
  S.device_error = derr;
  S.samples = stv[6];
  const int perIter = 3 + (h->dscene.numPointLights > 0) + (h->dscene.envOn != 0) + (h->dscene.numVolLights > 0);
  const int perWave = s.shader_provider == 5 ? (3 + h->maxIter * perIter) : 4;
  S.kernel_launches = wavesDone * perWave + 1;  // + the sample total
  if (derr != 0) {
    setLastError("device error flag raised: " + std::to_string(derr));
    return RG_ERR_DEVICE_STATUS;
  }
  h->haveResult = true;
  S.host_setup_ms = h->firstWaveHostMs > 0.0 ? h->firstWaveHostMs - tEntry : 0.0;
  S.host_total_ms = hostMs() - tEntry;
  trace.mark("stats read back");
  h->progressValue.store(1.0f);
  if (h->progress) h->progress(1.0f, h->progressUser);
  return RG_OK;
}

}  // namespace

rg_status rg_render(rg_handle* h) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  if (h->asyncBusy.load()) {
    setLastError("rg_render: an rg_render_async job of this handle is in flight");
    return RG_ERR_BUSY;
  }
  std::lock_guard<std::mutex> lk(h->mu);
  return renderLocked(h);
}

// One asynchronous render: a host thread runs the render of its handle.
struct rg_job {
  rg_handle* h = nullptr;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv;
  bool done = false;
  rg_status status = RG_OK;
  float finalProgress = 0.0f;  // the handle's progress when the render ended
};

rg_status rg_render_async(rg_handle* h, rg_job** out) {
  if (!h || !out) return RG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  bool expected = false;
  if (!h->asyncBusy.compare_exchange_strong(expected, true)) {
    setLastError("rg_render_async: a render of this handle is already in flight");
    return RG_ERR_BUSY;
  }
  rg_job* j = new (std::nothrow) rg_job();
  if (!j) {
    h->asyncBusy.store(false);
    return RG_ERR_OUT_OF_MEMORY;
  }
  j->h = h;
  h->progressValue.store(0.0f);
  try {
    j->worker = std::thread([j]() {
      rg_status rs;
      float pr;
      {
        // the handle is released (and may be destroyed) once this lock is
        // dropped: nothing below touches it
        std::lock_guard<std::mutex> lk(j->h->mu);
        rs = renderLocked(j->h);
        pr = j->h->progressValue.load();
        j->h->asyncBusy.store(false);
      }
      std::lock_guard<std::mutex> lk(j->mu);
      j->status = rs;
      j->finalProgress = pr;
      j->done = true;
      j->cv.notify_all();
    });
  } catch (...) {
    h->asyncBusy.store(false);
    delete j;
    setLastError("rg_render_async: could not start the render thread");
    return RG_ERR_OUT_OF_MEMORY;
  }
  *out = j;
  return RG_OK;
}

rg_status rg_poll(rg_job* j, int32_t* done, float* progress) {
  if (!j) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(j->mu);
  if (done) *done = j->done ? 1 : 0;
  if (progress) *progress = j->done ? j->finalProgress : j->h->progressValue.load();
  return RG_OK;
}

rg_status rg_wait(rg_job* j, double timeout_ms) {
  if (!j) return RG_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(j->mu);
  if (timeout_ms < 0) {
    j->cv.wait(lk, [j]() { return j->done; });
  } else if (!j->cv.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), [j]() { return j->done; })) {
    return RG_ERR_BUSY;
  }
  return j->status;
}

rg_status rg_job_free(rg_job* j) {
  if (!j) return RG_ERR_INVALID_ARGUMENT;
  if (j->worker.joinable()) j->worker.join();
  delete j;
  return RG_OK;
}

rg_status rg_reapply_postprocess(rg_handle* h) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->haveResult) return RG_ERR_NO_SCENE;
  const rg_status rs = postProcess(h, true);
  if (rs != RG_OK) return rs;
  launchTonemap(h->W * h->H, h->hdr.p, h->ldr.p, h->stream);
  RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  return RG_OK;
}

rg_status rg_get_hdr(rg_handle* h, float* rgba, size_t count) {
  if (!h || !rgba) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->haveResult) return RG_ERR_NO_SCENE;
  if (count < (size_t)h->W * h->H * 4) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA_CHECK(cudaMemcpy(rgba, h->hdr.p, sizeof(float4) * h->W * h->H, cudaMemcpyDeviceToHost));
  return RG_OK;
}

rg_status rg_get_ldr(rg_handle* h, float* rgba, size_t count) {
  if (!h || !rgba) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->haveResult) return RG_ERR_NO_SCENE;
  if (count < (size_t)h->W * h->H * 4) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA_CHECK(cudaMemcpy(rgba, h->ldr.p, sizeof(float4) * h->W * h->H, cudaMemcpyDeviceToHost));
  return RG_OK;
}

rg_status rg_get_aovs(rg_handle* h, float* normal, float* albedo, float* depth, size_t count) {
  if (!h) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->haveResult || !h->st.enable_denoise) return RG_ERR_NO_SCENE;
  const int N = h->W * h->H;
  if (count < (size_t)N * 3) return RG_ERR_INVALID_ARGUMENT;
  DevBuf<float> tmp;
  if (!tmp.alloc((size_t)N * 3)) return RG_ERR_OUT_OF_MEMORY;
  if (normal) {
    launchHalfToFloat(N * 3, h->aovNormal.p, tmp.p, h->stream);
    RG_CUDA_CHECK(cudaMemcpyAsync(normal, tmp.p, sizeof(float) * N * 3, cudaMemcpyDeviceToHost, h->stream));
    RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  }
  if (albedo) {
    launchHalfToFloat(N * 3, h->aovAlbedo.p, tmp.p, h->stream);
    RG_CUDA_CHECK(cudaMemcpyAsync(albedo, tmp.p, sizeof(float) * N * 3, cudaMemcpyDeviceToHost, h->stream));
    RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  }
  if (depth) {
    launchHalfToFloat(N, h->aovDepth.p, tmp.p, h->stream);
    RG_CUDA_CHECK(cudaMemcpyAsync(depth, tmp.p, sizeof(float) * N, cudaMemcpyDeviceToHost, h->stream));
    RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  }
  return RG_OK;
}

rg_status rg_get_sample_counts(rg_handle* h, int32_t* counts, size_t count) {
  if (!h || !counts) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->haveResult) return RG_ERR_NO_SCENE;
  if (count < (size_t)h->W * h->H) return RG_ERR_INVALID_ARGUMENT;
  RG_CUDA_CHECK(cudaMemcpy(counts, h->cnt.p, sizeof(int) * h->W * h->H, cudaMemcpyDeviceToHost));
  return RG_OK;
}

rg_status rg_get_stats(rg_handle* h, rg_stats* out) {
  if (!h || !out) return RG_ERR_INVALID_ARGUMENT;
  *out = h->lastStats;
  return RG_OK;
}

namespace {
rg_status mediumQuery(rg_handle* h, int32_t medium, bool bend, const float* in, int32_t n, float* out) {
  if (!h || n < 0 || (n > 0 && (!in || !out))) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->hasScene) return RG_ERR_NO_SCENE;
  if (medium < 0 || medium >= h->dscene.numMedia) return RG_ERR_INVALID_ARGUMENT;
  if (n == 0) return RG_OK;
  const int inW = bend ? 7 : 3, outW = bend ? 6 : 5;
  DevBuf<float> di, dout;
  DevBuf<DevJob> job;
  DevJob J;
  std::memset(&J, 0, sizeof(J));
  J.S = h->dscene;
  if (!di.upload(in, (size_t)n * inW, h->stream) || !dout.alloc((size_t)n * outW) || !job.upload(&J, 1, h->stream))
    return RG_ERR_OUT_OF_MEMORY;
  launchMediumQuery(job.p, medium, bend, di.p, n, dout.p, h->stream);
  RG_CUDA_CHECK(cudaGetLastError());
  RG_CUDA_CHECK(cudaMemcpyAsync(out, dout.p, sizeof(float) * (size_t)n * outW, cudaMemcpyDeviceToHost, h->stream));
  RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  return RG_OK;
}
}  // namespace

rg_status rg_medium_eval(rg_handle* h, int32_t medium, const float* points, int32_t n, float* out) {
  return mediumQuery(h, medium, false, points, n, out);
}

rg_status rg_medium_bend(rg_handle* h, int32_t medium, const float* rays, int32_t n, float* out) {
  return mediumQuery(h, medium, true, rays, n, out);
}

rg_status rg_debug_set_traversal_step_cap(int32_t cap) {
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  if (!setTraversalStepCap(cap)) {
    cudaGetLastError();
    setLastError("rg_debug_set_traversal_step_cap: cudaMemcpyToSymbol failed");
    return RG_ERR_CUDA;
  }
  return RG_OK;
}

rg_status rg_probe_sampling(int32_t which, const float* in, int32_t n, float* out) {
  static const int kInW[11] = {7, 5, 2, 7, 3, 7, 13, 4, 6, 7, 2};
  static const int kOutW[11] = {3, 1, 1, 3, 6, 3, 3, 1, 3, 1, 1};
  if (which < 0 || which > 10 || n < 0 || (n > 0 && (!in || !out))) return RG_ERR_INVALID_ARGUMENT;
  if (n == 0) return RG_OK;
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  DevBuf<float> din, dout;
  if (!din.upload(in, (size_t)n * kInW[which], 0) || !dout.alloc((size_t)n * kOutW[which])) return RG_ERR_OUT_OF_MEMORY;
  launchProbeSampling(which, din.p, n, dout.p, 0);
  RG_CUDA_CHECK(cudaGetLastError());
  RG_CUDA_CHECK(cudaMemcpy(out, dout.p, sizeof(float) * (size_t)n * kOutW[which], cudaMemcpyDeviceToHost));
  return RG_OK;
}

rg_status rg_get_view_matrix(rg_handle* h, float* m16) {
  if (!h || !m16) return RG_ERR_INVALID_ARGUMENT;
  std::memcpy(m16, h->view.m, sizeof(float) * 16);
  return RG_OK;
}

rg_status rg_trace_closest(rg_handle* h, const float* rays, int32_t n, float* out_tuv, int32_t* out_prim) {
  if (!h || n < 0 || (n > 0 && (!rays || !out_tuv || !out_prim))) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->hasScene) return RG_ERR_NO_SCENE;
  if (n == 0) return RG_OK;
  DevBuf<float> r, t;
  DevBuf<int> p;
  if (!r.upload(rays, (size_t)n * 6, h->stream) || !t.alloc((size_t)n * 3) || !p.alloc(n)) return RG_ERR_OUT_OF_MEMORY;
  RG_CUDA_CHECK(cudaMemsetAsync(h->error.p, 0, sizeof(int), h->stream));  // this query's flag only
  launchQueryClosest(h->dscene, r.p, n, t.p, p.p, h->stream);
  RG_CUDA_CHECK(cudaMemcpyAsync(out_tuv, t.p, sizeof(float) * n * 3, cudaMemcpyDeviceToHost, h->stream));
  RG_CUDA_CHECK(cudaMemcpyAsync(out_prim, p.p, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  int derr = 0;
  RG_CUDA_CHECK(cudaMemcpyAsync(&derr, h->error.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  if (derr) {
    setLastError("device error flag raised: " + std::to_string(derr));
    return RG_ERR_DEVICE_STATUS;
  }
  return RG_OK;
}

rg_status rg_trace_any(rg_handle* h, const float* rays, const float* tmax, int32_t n, int32_t predicate, uint8_t* out) {
  if (!h || n < 0 || predicate < 0 || predicate > 4 || (n > 0 && (!rays || !tmax || !out))) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!h->hasScene) return RG_ERR_NO_SCENE;
  if (n == 0) return RG_OK;
  DevBuf<float> r, tm;
  DevBuf<uint8_t> o;
  if (!r.upload(rays, (size_t)n * 6, h->stream) || !tm.upload(tmax, n, h->stream) || !o.alloc(n)) return RG_ERR_OUT_OF_MEMORY;
  const uint32_t occs[5] = {kOccArea, kOccPoint, kOccAO, kOccAll, kOccVol};
  const uint32_t occ = occs[predicate];
  RG_CUDA_CHECK(cudaMemsetAsync(h->error.p, 0, sizeof(int), h->stream));  // this query's flag only
  launchQueryAny(h->dscene, r.p, tm.p, n, occ, o.p, h->stream);
  RG_CUDA_CHECK(cudaMemcpyAsync(out, o.p, n, cudaMemcpyDeviceToHost, h->stream));
  int derr = 0;
  RG_CUDA_CHECK(cudaMemcpyAsync(&derr, h->error.p, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  RG_CUDA_CHECK(cudaStreamSynchronize(h->stream));
  if (derr) {
    setLastError("device error flag raised: " + std::to_string(derr));
    return RG_ERR_DEVICE_STATUS;
  }
  return RG_OK;
}

rg_status rg_denoise_atrous(int32_t w, int32_t h, const float* color, const float* normal, const float* depth,
                            const float* albedo, const float* albedo_alpha, int32_t levels, float sigma_color,
                            float sigma_normal, float sigma_depth, float intensity, float* out) {
  if (w <= 0 || h <= 0 || !color || !normal || !depth || !albedo || !albedo_alpha || !out) return RG_ERR_INVALID_ARGUMENT;
  if (levels < 1 || levels > kMaxDenoiseLevels) {
    setLastError("rg_denoise_atrous: levels must be in [1, " + std::to_string(kMaxDenoiseLevels) + "]");
    return RG_ERR_INVALID_ARGUMENT;
  }
  const size_t nPix = (size_t)w * (size_t)h;
  if (nPix * 3 > (size_t)INT_MAX) {
    setLastError("rg_denoise_atrous: image of " + std::to_string(nPix) + " pixels is too large");
    return RG_ERR_INVALID_ARGUMENT;
  }
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  const int N = (int)nPix;
  std::vector<float4> c4(N);
  for (int i = 0; i < N; i++) c4[i] = make_float4(color[i * 3], color[i * 3 + 1], color[i * 3 + 2], 1.0f);
  DevBuf<float4> c, a, b, o;
  DevBuf<float> fn, fa, fd, faa;
  DevBuf<__half> hn, ha, hd, haa;
  cudaStream_t st = 0;
  if (!c.upload(c4.data(), N, st) || !a.alloc(N) || !b.alloc(N) || !o.alloc(N) || !fn.upload(normal, (size_t)N * 3, st) ||
      !fa.upload(albedo, (size_t)N * 3, st) || !fd.upload(depth, N, st) || !faa.upload(albedo_alpha, N, st) ||
      !hn.alloc((size_t)N * 3) || !ha.alloc((size_t)N * 3) || !hd.alloc(N) || !haa.alloc(N))
    return RG_ERR_OUT_OF_MEMORY;
  launchFloatToHalf(N * 3, fn.p, hn.p, st);
  launchFloatToHalf(N * 3, fa.p, ha.p, st);
  launchFloatToHalf(N, fd.p, hd.p, st);
  launchFloatToHalf(N, faa.p, haa.p, st);
  launchDenoise(w, h, c.p, hn.p, hd.p, ha.p, haa.p, levels, sigma_color, sigma_normal, sigma_depth, intensity, a.p, b.p,
                o.p, st);
  RG_CUDA_CHECK(cudaMemcpy(c4.data(), o.p, sizeof(float4) * N, cudaMemcpyDeviceToHost));
  for (int i = 0; i < N; i++) { out[i * 3] = c4[i].x; out[i * 3 + 1] = c4[i].y; out[i * 3 + 2] = c4[i].z; }
  return RG_OK;
}

rg_status rg_tonemap(int32_t w, int32_t h, const float* hdr_rgba, float* ldr_rgba) {
  if (w <= 0 || h <= 0 || !hdr_rgba || !ldr_rgba) return RG_ERR_INVALID_ARGUMENT;
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  const int N = w * h;
  DevBuf<float4> a, b;
  if (!a.upload(reinterpret_cast<const float4*>(hdr_rgba), N, 0) || !b.alloc(N)) return RG_ERR_OUT_OF_MEMORY;
  launchTonemap(N, a.p, b.p, 0);
  RG_CUDA_CHECK(cudaMemcpy(ldr_rgba, b.p, sizeof(float4) * N, cudaMemcpyDeviceToHost));
  return RG_OK;
}

rg_status rg_bloom(int32_t w, int32_t h, const float* hdr_rgba, float threshold, float strength, float radius,
                   float size_aspect, float curve, float* out_rgba) {
  if (w <= 0 || h <= 0 || !hdr_rgba || !out_rgba) return RG_ERR_INVALID_ARGUMENT;
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  const int N = w * h;
  const BloomPlan p = planBloom(w, h, radius, size_aspect);
  const size_t n = (size_t)p.gw * p.gh;
  DevBuf<float4> a, sa, sb;
  DevBuf<float> wt;
  if (!a.upload(reinterpret_cast<const float4*>(hdr_rgba), N, 0) || !sa.alloc(n) || !sb.alloc(n) ||
      !wt.upload(p.weights.data(), p.weights.size(), 0))
    return RG_ERR_OUT_OF_MEMORY;
  launchBloom(w, h, a.p, p, wt.p, threshold, strength, curve, sa.p, sb.p, 0);
  RG_CUDA_CHECK(cudaMemcpy(out_rgba, a.p, sizeof(float4) * N, cudaMemcpyDeviceToHost));
  return RG_OK;
}

static std::mutex g_storeMu;
static std::unordered_map<const rg_scene_desc*, SceneStore*> g_stores;

static rg_scene_desc* registerStore(SceneStore* st) {
  std::lock_guard<std::mutex> lk(g_storeMu);
  g_stores[&st->desc] = st;
  return &st->desc;
}

rg_status rg_scene_builtin(int32_t kind, uint32_t seed, const int32_t* iparams, int32_t n_iparams, rg_scene_desc** out) {
  if (!out) return RG_ERR_INVALID_ARGUMENT;
  SceneStore* st = nullptr;
  const rg_status rs = buildBuiltinScene(kind, seed, iparams, n_iparams, &st);
  if (rs != RG_OK) return rs;
  *out = registerStore(st);
  return RG_OK;
}

rg_status rg_scene_free(rg_scene_desc* scene) {
  if (!scene) return RG_ERR_INVALID_ARGUMENT;
  SceneStore* st = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_storeMu);
    auto it = g_stores.find(scene);
    if (it == g_stores.end()) return RG_ERR_INVALID_ARGUMENT;
    st = it->second;
    g_stores.erase(it);
  }
  delete st;
  return RG_OK;
}

rg_status rg_save_image(const char* path, int32_t width, int32_t height, const float* rgba) {
  if (!path || !rgba || width <= 0 || height <= 0) return RG_ERR_INVALID_ARGUMENT;
  std::string err;
  if (!writeImageFile(path, width, height, rgba, err)) {
    setLastError(err);
    return err.rfind("unsupported", 0) == 0 ? RG_ERR_UNSUPPORTED : RG_ERR_IO;
  }
  return RG_OK;
}

rg_status rg_load_image(const char* path, int32_t* width, int32_t* height, int32_t* is_hdr, float* rgba,
                        size_t count) {
  if (!path || !width || !height) return RG_ERR_INVALID_ARGUMENT;
  TextureStore t;
  std::string err;
  if (!readImageFile(path, t, err)) {
    setLastError(err);
    return err.find("cannot open") != std::string::npos ? RG_ERR_IO : RG_ERR_PARSE;
  }
  *width = t.width;
  *height = t.height;
  if (is_hdr) *is_hdr = t.isHdr;
  if (!rgba) return RG_OK;
  if (count < t.rgba.size()) return RG_ERR_INVALID_ARGUMENT;
  std::memcpy(rgba, t.rgba.data(), t.rgba.size() * sizeof(float));
  return RG_OK;
}

rg_status rg_load_scene_json(const char* path, rg_scene_desc** out) {
  if (!path || !out) return RG_ERR_INVALID_ARGUMENT;
  SceneStore* st = nullptr;
  std::string err;
  const rg_status rs = loadSceneJson(path, &st, err);
  if (rs != RG_OK) {
    setLastError(err);
    return rs;
  }
  *out = registerStore(st);
  return RG_OK;
}

}  // extern "C"
