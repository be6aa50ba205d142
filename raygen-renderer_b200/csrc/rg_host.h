// rg_host.h - host-side internals of the B200 tracer (not part of the C ABI).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <memory>
#include <cstdint>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/raygen_b200.h"

namespace rg {

struct DevMaterial;
struct DevMedium;
struct DevPathPoint;
struct DevVolLight;
struct DevScene;
struct DevRender;

// 4x4 row-major matrix, row-vector convention p' = [p 1] * M.
struct Mat4 {
  float m[16];
};
Mat4 viewMatrix(const rg_camera& c);
DevRender makeRenderParams(const rg_settings& s, const rg_camera& c);
struct DevPointLight;
struct DevTexture;

// Device buffers come from the device's default stream-ordered pool.  With
// its default release threshold (0) every synchronisation hands freed memory
// back to the driver, so re-uploading a large scene re-maps hundreds of MB;
// keepPoolMemory() raises the threshold for the current device (once), and
// trimPoolMemory() returns unused memory when a handle goes away.
void keepPoolMemory();
void trimPoolMemory();

// Owning device allocation from the stream-ordered pool.  Allocation and free
// are ordered on the calling thread's per-thread stream, so releasing a buffer
// does not synchronise the device; callers release a buffer only after the
// streams that used it have been synchronised.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void swap(DevBuf& o) {
    std::swap(p, o.p);
    std::swap(n, o.n);
  }
  bool alloc(size_t count) {
    if (count <= n && p) return true;
    release();
    if (count == 0) count = 1;
    if (cudaMallocAsync((void**)&p, count * sizeof(T), cudaStreamPerThread) != cudaSuccess ||
        cudaStreamSynchronize(cudaStreamPerThread) != cudaSuccess) {
      p = nullptr;
      n = 0;
      cudaGetLastError();
      return false;
    }
    n = count;
    return true;
  }
  size_t bytes() const { return p ? n * sizeof(T) : 0; }
  void release() {
    if (p) cudaFreeAsync(p, cudaStreamPerThread);
    p = nullptr;
    n = 0;
  }
  bool upload(const T* src, size_t count, cudaStream_t st) {
    if (!alloc(count)) return false;
    if (count && src) return cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, st) == cudaSuccess;
    return true;
  }
};

// Procedural / loaded scene description owned by the library.
struct TextureStore {
  int width = 0, height = 0, isHdr = 0;
  std::vector<float> rgba;
};

struct SceneStore {
  std::vector<float> positions, normals, uvs;
  std::vector<int32_t> triMesh, meshObject;
  std::vector<rg_object> objects;
  std::vector<rg_material> materials;
  std::vector<rg_medium> media;
  std::vector<std::vector<rg_medium_path_point>> mediumPaths;  // per medium; finalize() points media at them
  int32_t globalMedium = -1;
  std::vector<rg_point_light> pointLights;
  std::vector<TextureStore> textures;
  std::vector<rg_texture> textureDescs;
  rg_camera camera{};
  int32_t envmapTexture = -1;  // index into textures, -1 none
  int32_t envCube = 0;         // cubemap faces present (px nx py ny pz nz)
  int32_t envCubeFaces[6] = {-1, -1, -1, -1, -1, -1};
  float envmapIntensity = 1.0f, envmapRotation = 0.0f;
  rg_scene_desc desc{};
  void finalize();
};

rg_status buildBuiltinScene(int kind, uint32_t seed, const int32_t* ip, int nip, SceneStore** out);
rg_status loadSceneJson(const char* path, SceneStore** out, std::string& err);

// Image files (rg_image.cpp): RGBA float, row 0 at the top.
bool readRadianceHdr(const std::string& path, TextureStore& out, std::string& err);
bool readPfm(const std::string& path, TextureStore& out, std::string& err);
bool readImageFile(const std::string& path, TextureStore& out, std::string& err);
// JPEG (baseline / extended sequential) and PNG decoders (rg_decode.cpp): LDR RGBA in [0, 1].
bool decodeJpeg(const std::vector<unsigned char>& bytes, TextureStore& out, std::string& err);
bool decodePng(const std::vector<unsigned char>& bytes, TextureStore& out, std::string& err);
bool writeImageFile(const std::string& path, int W, int H, const float* rgba, std::string& err);

// Working memory of the BVH build (rg_bvh.cu).
struct BvhScratch;
void freeBvhScratch(BvhScratch* s);

// Device-resident scene (BVH + triangle and light tables).
struct DeviceScene {
  int numTris = 0;
  bool hasUV = false;
  // keepBuffers: the scene is rebuilt in place (a render handle): the inputs and
  // the build's working memory stay allocated for the next scene, otherwise
  // they are freed after the build
  bool keepBuffers = false;
  BvhScratch* scratch = nullptr;
  // world-space inputs
  DevBuf<float> inPos, inNrm, inUV;
  DevBuf<int> inTriMesh;
  DevBuf<float> view;
  // tables
  DevBuf<int> meshObj, meshTriCount, objMat, objMedium;
  DevBuf<DevMaterial> mats;
  DevBuf<DevMedium> media;
  DevBuf<DevPathPoint> pathPts;
  DevBuf<DevVolLight> volLights;
  int globalMedium = -1;
  bool hasHaze = false;       // a heat-haze medium is in use: paths take extra segments
  DevBuf<int> areaLightObj, lightMeshList;
  DevBuf<int2> lightObjMeshes, lightMeshTris;
  DevBuf<float4> lightTris;
  int numAreaLights = 0;
  DevBuf<DevPointLight> points;
  int numPointLights = 0;
  DevBuf<DevTexture> textures;
  std::vector<DevBuf<float4>*> texels;
  int numTextures = 0;
  // equirectangular environment map: texture index and importance-sampling CDFs
  int envTex = -1, envW = 0, envH = 0;
  float envIntensity = 1.0f, envCosY = 1.0f, envSinY = 0.0f, envTotal = 0.0f;
  DevBuf<float> envMarg, envCond;
  // cubemap environment: face textures and the per-face sampling CDFs
  int envCube = 0, envFace[6] = {-1, -1, -1, -1, -1, -1}, envCubeW = 0;
  float envCubeTotal = 0.0f;
  DevBuf<float> cubeMargFace, cubeMargY, cubeCond;
  // BVH + leaf-order triangles
  DevBuf<float4> nodes, nodes8, triVerts, triShade;
  int numNodes8 = 0;
  int bvhWidth = 2;
  DevBuf<float2> triUV;
  DevBuf<int> triOrig, triMat;
  int numNodes = 0;
  int rootIsLeaf = 0, rootLeafRef = 0;
  int buildLevels = 0;
  // device bytes held by the scene after its build
  size_t deviceBytes() const;
  // takes over the device buffers of the scene it replaces: DevBuf::alloc only
  // grows, so a scene no larger than the last one allocates no device memory
  void adoptBuffers(DeviceScene& old);
  ~DeviceScene() {
    for (auto* t : texels) delete t;
    freeBvhScratch(scratch);
  }
};

rg_status buildDeviceBvh(DeviceScene& ds, int nbins, bool wide, cudaStream_t st, std::string& err);

// Learned denoiser (rg_kpcn.cu): inference on device buffers (noisy HDR and the
// renderer's half guides), blended with the noisy image by `intensity`.
struct KpcnNet;
KpcnNet* kpcnOf(rg_denoiser* d);
rg_status kpcnDenoiseDevice(KpcnNet& n, int W, int H, const float4* noisy, const __half* normal, const __half* albedo,
                            const __half* depth, const int* cnt, float intensity, float4* out, cudaStream_t st);
// keep: reuse `out`'s buffers for the new scene and keep them afterwards
// (DeviceScene::keepBuffers); otherwise `out` is replaced by a fresh scene.
rg_status prepareScene(const rg_scene_desc* d, int bins, bool wide, cudaStream_t st, int* errWord,
                       std::unique_ptr<DeviceScene>& out, DevScene& S, Mat4& view, float* buildMs, bool keep = false);

void setLastError(const std::string& msg);

}  // namespace rg
