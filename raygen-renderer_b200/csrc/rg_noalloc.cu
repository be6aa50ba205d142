// rg_noalloc.cu - A-Trous denoise on caller device buffers, without allocating.
//
// rg_denoise_atrous takes host buffers and allocates its own device copies
// and working buffers on every call.  Some callers cannot have the library
// allocate: an interactive preview loop that denoises every progressive
// snapshot cannot absorb the device-wide synchronisation that cudaFree
// implies, and a host application that owns all device memory through its
// own pool (a framework's caching allocator, a fixed memory budget per
// process) does not want a second allocator touching the device at all.
// rg_denoise_atrous_noalloc serves them: inputs and output stay in the
// caller's device memory and the filter's working buffers live in one
// statically sized __device__ array of this module, so a call makes no
// cudaMalloc / cudaFree / allocating-library call of any kind.
//
// It runs exactly the kernels of rg_denoise_atrous (float -> half guide
// conversion, firefly pre-clamp + albedo demodulation, the A-Trous levels,
// remodulation), so the two agree bit for bit on the same inputs.
//
// Limits and rules (also stated in the C header):
//  * w * h <= kMaxPixels (1,048,576, e.g. 1024 x 1024); larger images are
//    rejected with RG_ERR_INVALID_ARGUMENT before any device work.
//  * The working buffers are shared by all calls on a device: calls whose
//    device work overlaps (different streams, or different host threads
//    without ordering) race on them and corrupt each other's results.
//    Serialise them on one stream, or wait for one call's stream work before
//    the next call is issued.
//  * Nothing in the working buffers has to start at zero: every pass writes
//    each pixel of its destination before any later pass reads it, so no
//    clearing is done between calls.
//  * The first call in a CUDA context (per device, and again after a device
//    reset) resolves the array's device address (cudaGetSymbolAddress, which
//    may load this module); make that first call before any stream capture
//    begins.
//  * levels in [1, 16]; out_rgba may not overlap any input.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <climits>
#include <mutex>
#include <string>

#include "rg_host.h"
#include "rg_trace.cuh"

namespace rg {

namespace {

constexpr size_t kMaxPixels = size_t(1) << 20;
// Layout of the working array, each part 256-byte aligned:
//   two float4 ping-pong colour buffers, then the half guides
//   (normal x3, albedo x3, depth, albedo alpha).
constexpr size_t kColourBytes = kMaxPixels * sizeof(float4);
constexpr size_t kOffA = 0;
constexpr size_t kOffB = kOffA + kColourBytes;
constexpr size_t kOffNormal = kOffB + kColourBytes;
constexpr size_t kOffAlbedo = kOffNormal + kMaxPixels * 3 * sizeof(__half);
constexpr size_t kOffDepth = kOffAlbedo + kMaxPixels * 3 * sizeof(__half);
constexpr size_t kOffAlbedoA = kOffDepth + kMaxPixels * sizeof(__half);
constexpr size_t kScratchBytes = kOffAlbedoA + kMaxPixels * sizeof(__half);  // 48 MiB
static_assert(kOffB % 256 == 0 && kOffNormal % 256 == 0 && kOffAlbedo % 256 == 0 && kOffDepth % 256 == 0 &&
                  kOffAlbedoA % 256 == 0,
              "working buffer parts must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_atrousScratch[kScratchBytes];

// Working-array addresses by CUDA context id.  Bounded: when full, the oldest
// entry (most likely a context that no longer exists) is dropped.
class ScratchCache {
 public:
  static constexpr int kEntries = 64;
  unsigned char* find(unsigned long long id) const {
    for (int i = 0; i < n_; ++i)
      if (ids_[i] == id) return ptrs_[i];
    return nullptr;
  }
  void insert(unsigned long long id, unsigned char* p) {
    int slot;
    if (n_ < kEntries) {
      slot = n_++;
    } else {
      slot = next_;
      next_ = (next_ + 1) % kEntries;
    }
    ids_[slot] = id;
    ptrs_[slot] = p;
  }

 private:
  unsigned long long ids_[kEntries] = {};
  unsigned char* ptrs_[kEntries] = {};
  int n_ = 0;
  int next_ = 0;
};

// The array's device address belongs to the CUDA context the module was
// loaded into: a device reset, or a second (non-primary) context on the same
// device, loads the module again at another address.  So the cache is keyed
// by the context's process-unique id (cuCtxGetId), not by device ordinal; an
// id is never reused, so an entry of a destroyed context can never match.
// The driver functions come through cudaGetDriverEntryPoint, so the library
// needs no link against libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

std::mutex g_setupMu;
ScratchCache g_cache;

rg_status currentContextId(unsigned long long* id) {
  static CtxGetCurrentFn getCurrent = nullptr;
  static CtxGetIdFn getId = nullptr;
  if (!getCurrent || !getId) {
    void* a = nullptr;
    void* b = nullptr;
    cudaDriverEntryPointQueryResult qa, qb;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) != cudaSuccess ||
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) != cudaSuccess ||
        qa != cudaDriverEntryPointSuccess || qb != cudaDriverEntryPointSuccess || !a || !b) {
      cudaGetLastError();
      setLastError("rg_denoise_atrous_noalloc: the driver does not provide cuCtxGetCurrent / cuCtxGetId");
      return RG_ERR_CUDA;
    }
    getCurrent = reinterpret_cast<CtxGetCurrentFn>(a);
    getId = reinterpret_cast<CtxGetIdFn>(b);
  }
  CUcontext ctx = nullptr;
  if (getCurrent(&ctx) != CUDA_SUCCESS || !ctx) return RG_ERR_NO_DEVICE;
  if (getId(ctx, id) != CUDA_SUCCESS) {
    setLastError("rg_denoise_atrous_noalloc: cuCtxGetId failed");
    return RG_ERR_CUDA;
  }
  return RG_OK;
}

rg_status resolveScratch(unsigned char** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_atrousScratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    setLastError(std::string("rg_denoise_atrous_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    return RG_ERR_CUDA;
  }
  *out = static_cast<unsigned char*>(p);
  return RG_OK;
}

// Device address of the working array in the current context, resolved once
// per context (with that context current).
rg_status scratchForCurrentContext(unsigned char** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    cudaGetLastError();
    setLastError(std::string("rg_denoise_atrous_noalloc: no current CUDA device: ") + cudaGetErrorString(e));
    return RG_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lk(g_setupMu);
  unsigned long long id = 0;
  rg_status rs = currentContextId(&id);
  if (rs == RG_ERR_NO_DEVICE) {
    // No context is current yet on this thread: the runtime makes the
    // device's primary context current on its first call that needs one, and
    // resolving the symbol is such a call.
    unsigned char* p = nullptr;
    rs = resolveScratch(&p);
    if (rs != RG_OK) return rs;
    rs = currentContextId(&id);
    if (rs == RG_ERR_NO_DEVICE) setLastError("rg_denoise_atrous_noalloc: no CUDA context is current");
  }
  if (rs != RG_OK) return rs;
  if (unsigned char* hit = g_cache.find(id)) {
    *out = hit;
    return RG_OK;
  }
  unsigned char* p = nullptr;
  rs = resolveScratch(&p);
  if (rs != RG_OK) return rs;
  g_cache.insert(id, p);
  *out = p;
  return RG_OK;
}

bool overlaps(const void* a, size_t an, const void* b, size_t bn) {
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + bn && y < x + an;
}

// A caller pointer must be device (or managed) memory visible on the current
// device and aligned for its element type; host pointers are refused here
// rather than faulting in a kernel.
bool deviceBuffer(const void* p, size_t align, int dev, const char* name) {
  if (!p || (reinterpret_cast<uintptr_t>(p) % align) != 0) {
    setLastError(std::string("rg_denoise_atrous_noalloc: ") + name + " is null or misaligned");
    return false;
  }
  cudaPointerAttributes a;
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    setLastError(std::string("rg_denoise_atrous_noalloc: ") + name + ": " + cudaGetErrorString(e));
    return false;
  }
  const bool ok = a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
  if (!ok) setLastError(std::string("rg_denoise_atrous_noalloc: ") + name + " is not device memory of the current device");
  return ok;
}

}  // namespace

}  // namespace rg

extern "C" rg_status rg_denoise_atrous_noalloc(int32_t w, int32_t h, const float* color_rgba, const float* normal,
                                               const float* depth, const float* albedo, const float* albedo_alpha,
                                               int32_t levels, float sigma_color, float sigma_normal,
                                               float sigma_depth, float intensity, float* out_rgba, void* stream) {
  using namespace rg;
  if (w <= 0 || h <= 0) {
    setLastError("rg_denoise_atrous_noalloc: width and height must be positive");
    return RG_ERR_INVALID_ARGUMENT;
  }
  const size_t n = (size_t)w * (size_t)h;
  if (n > kMaxPixels) {
    setLastError("rg_denoise_atrous_noalloc: " + std::to_string(w) + " x " + std::to_string(h) + " = " +
                 std::to_string(n) + " pixels exceeds the working-buffer limit of " + std::to_string(kMaxPixels) +
                 " pixels; use rg_denoise_atrous");
    return RG_ERR_INVALID_ARGUMENT;
  }
  if (levels < 1 || levels > kMaxDenoiseLevels) {
    setLastError("rg_denoise_atrous_noalloc: levels must be in [1, " + std::to_string(kMaxDenoiseLevels) + "]");
    return RG_ERR_INVALID_ARGUMENT;
  }
  unsigned char* s = nullptr;
  const rg_status rs = scratchForCurrentContext(&s);
  if (rs != RG_OK) return rs;
  int dev = 0;
  cudaGetDevice(&dev);
  if (!deviceBuffer(color_rgba, 16, dev, "color_rgba") || !deviceBuffer(out_rgba, 16, dev, "out_rgba") ||
      !deviceBuffer(normal, 4, dev, "normal") || !deviceBuffer(depth, 4, dev, "depth") ||
      !deviceBuffer(albedo, 4, dev, "albedo") || !deviceBuffer(albedo_alpha, 4, dev, "albedo_alpha"))
    return RG_ERR_INVALID_ARGUMENT;
  // The output is written while the colour input is still read (the last pass
  // reads the noisy colour beside the filtered one), so it may not share
  // memory with any input.
  const size_t outBytes = n * sizeof(float4);
  if (overlaps(out_rgba, outBytes, color_rgba, n * sizeof(float4)) ||
      overlaps(out_rgba, outBytes, normal, n * 3 * sizeof(float)) ||
      overlaps(out_rgba, outBytes, albedo, n * 3 * sizeof(float)) ||
      overlaps(out_rgba, outBytes, depth, n * sizeof(float)) ||
      overlaps(out_rgba, outBytes, albedo_alpha, n * sizeof(float))) {
    setLastError("rg_denoise_atrous_noalloc: out_rgba overlaps an input buffer");
    return RG_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float4* bufA = reinterpret_cast<float4*>(s + kOffA);
  float4* bufB = reinterpret_cast<float4*>(s + kOffB);
  __half* hn = reinterpret_cast<__half*>(s + kOffNormal);
  __half* ha = reinterpret_cast<__half*>(s + kOffAlbedo);
  __half* hd = reinterpret_cast<__half*>(s + kOffDepth);
  __half* haa = reinterpret_cast<__half*>(s + kOffAlbedoA);
  const int N = (int)n;
  launchFloatToHalf(N * 3, normal, hn, st);
  launchFloatToHalf(N * 3, albedo, ha, st);
  launchFloatToHalf(N, depth, hd, st);
  launchFloatToHalf(N, albedo_alpha, haa, st);
  launchDenoise(w, h, reinterpret_cast<const float4*>(color_rgba), hn, hd, ha, haa, levels, sigma_color, sigma_normal,
                sigma_depth, intensity, bufA, bufB, reinterpret_cast<float4*>(out_rgba), st);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    setLastError(std::string("rg_denoise_atrous_noalloc: launch failed: ") + cudaGetErrorString(e));
    return RG_ERR_CUDA;
  }
  return RG_OK;
}

// Test hook for the context-keyed address cache (no CUDA call): feeds a
// sequence of context ids through a fresh cache whose resolver hands out a new
// address per resolve, and reports for each lookup whether it resolved
// (out_resolved[i] = 1) and which address it returned (out_slot[i], the
// resolve's ordinal).  No reference counterpart.
extern "C" rg_status rg_noalloc_cache_probe(const uint64_t* ids, int32_t n, int32_t* out_resolved, int32_t* out_slot) {
  using namespace rg;
  if (n < 0 || (n > 0 && (!ids || !out_resolved || !out_slot))) return RG_ERR_INVALID_ARGUMENT;
  ScratchCache cache;
  int32_t resolves = 0;
  for (int32_t i = 0; i < n; ++i) {
    unsigned char* hit = cache.find(ids[i]);
    out_resolved[i] = hit ? 0 : 1;
    if (!hit) {
      // stand-in addresses 1, 2, 3, ...: the ordinal of the resolve
      hit = reinterpret_cast<unsigned char*>(static_cast<uintptr_t>(++resolves));
      cache.insert(ids[i], hit);
    }
    out_slot[i] = (int32_t)reinterpret_cast<uintptr_t>(hit);
  }
  return RG_OK;
}
