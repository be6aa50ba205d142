// rg_trace.cuh - launchers of the trace and post kernels (host-callable).
#pragma once

#include <vector>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "rg_device.cuh"

namespace rg {

int residentBlocks(int kernel, int width);
void launchGenerate(const DevJob* jobs, const DevWave* W, const DevQueues& Q, int grid, cudaStream_t st);
// `single` (and `singleR`) non-null: one job with its constants as kernel parameters;
// null: per-ray job slots into `jobs`.
void launchExtend(const DevScene* single, const DevJob* jobs, int width, const DevQueues& Q, int iter, int grid,
                  cudaStream_t st);
// single == nullptr: the multi-job kernel; multiMediaLevel 2 includes the
// procedural-media code, 1 homogeneous media only (no volume-light queue)
void launchShade(const DevScene* single, const DevRender* singleR, const DevJob* jobs, const DevQueues& Q, int iter,
                 int grid, cudaStream_t st, int multiMediaLevel = 2);
void launchConnect(const DevScene* single, const DevJob* jobs, int width, const DevQueues& Q, int iter, int which,
                   int grid, cudaStream_t st);
void launchSimple(const DevJob* jobs, const DevWave* W, const DevQueues& Q, int grid, cudaStream_t st);
void launchAccumulate(const DevJob* jobs, const DevWave* W, const DevQueues& Q, int grid, cudaStream_t st);
void launchAov(const DevScene& S, const DevRender& R, __half* normal, __half* albedo, __half* albedoA, __half* depth,
               cudaStream_t st);
void launchQueryClosest(const DevScene& S, const float* rays, int n, float* tuv, int* prim, cudaStream_t st);
void launchQueryAny(const DevScene& S, const float* rays, const float* tmax, int n, uint32_t occ, uint8_t* out,
                    cudaStream_t st);
// node-step bound of every traversal loop (cap <= 0: the built-in bound); a test hook
bool setTraversalStepCap(int cap);
// sampling-helper probes (rg_probe_sampling)
void launchProbeSampling(int which, const float* in, int n, float* out, cudaStream_t st);
// triMat[i] = shading class << 28 | material index of leaf-order triangle i
void launchTriMaterial(const DevScene& S, int n, int* triMat, cudaStream_t st);
// jobs[0].S is the scene; eval: n x 3 points -> n x 5, bend: n x 7 rays -> n x 6
void launchMediumQuery(const DevJob* jobs, int medium, bool bend, const float* in, int n, float* out, cudaStream_t st);

// post (rg_post.cu)
// A-Trous levels accepted by the entry points (step 2^l stays far inside int)
constexpr int kMaxDenoiseLevels = 16;
void launchResolve(int n, const float4* sum, const int* cnt, float exposure, float4* hdr, cudaStream_t st);
void launchDenoise(int w, int h, const float4* noisy, const __half* normal, const __half* depth, const __half* albedo,
                   const __half* albedoA, int levels, float sigC, float sigN, float sigD, float intensity,
                   float4* bufA, float4* bufB, float4* out, cudaStream_t st);
void launchTonemap(int n, const float4* hdr, float4* ldr, cudaStream_t st);
// HDR bloom: glow buffer size and the normalised Gaussian taps (host), then
// extract + area downsample, 2 x (horizontal, vertical) blur, upsample + add.
struct BloomPlan {
  int gw = 1, gh = 1, r = 0;    // glow buffer size, blur radius (0: no blur)
  std::vector<float> weights;   // 2r+1 taps
};
BloomPlan planBloom(int W, int H, float radius, float sizeAspect);
void launchBloom(int W, int H, float4* hdr, const BloomPlan& p, const float* weightsDev, float threshold,
                 float strength, float curve, float4* smallA, float4* smallB, cudaStream_t st);
// adaptive: per-pixel relative SEM -> compacted active pixel list; returns count via *outCount (device)
void launchAdaptivePixels(int n, const float4* sum, const float4* sumSq, const int* cnt, int target, float threshold,
                          int* list, int* outCount, cudaStream_t st);
void launchAdaptiveTiles(int w, int h, const float4* sum, const float4* sumSq, const int* cnt, int target,
                         float threshold, int* list, int* outCount, cudaStream_t st);
void launchHalfToFloat(int n, const __half* in, float* out, cudaStream_t st);
void launchFloatToHalf(int n, const float* in, __half* out, cudaStream_t st);

}  // namespace rg
