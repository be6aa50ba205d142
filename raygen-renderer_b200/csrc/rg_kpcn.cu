// rg_kpcn.cu - learned denoiser: a kernel-predicting CNN on the 5th-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulation in tensor memory).
//
// Network (after Bako et al. 2017, kernel-predicting convolutional networks
// for Monte Carlo denoising): features [P x 16] = log1p(radiance), albedo,
// normal and depth guides (the A-Trous guides, rayrenderer.cpp:819-844), the
// noise level log2(1 + samples per pixel) / 12 and 5 zero channels; five 3x3 convolutions with ReLU (16 -> 32, then 32 -> 32);
// a 3x3 convolution to 25 logits; softmax -> a 5 x 5 kernel per pixel applied
// to the noisy radiance (clamp to edge).  Loss: relMSE (o - r)^2 / (r^2 + 0.01).
//
// Every convolution pass is an implicit GEMM on the tensor-core block of
// rg_tc.cuh (M = 128 rows, N = 32, K a multiple of 16):
//   forward        rows = 128 pixels of an image row, K = (tap, input
//                  channel); A is addressed straight in a ring of input rows
//                  loaded by TMA, by per-tap descriptors (k_convStrip, a
//                  producer thread and four epilogue warps); B = weights;
//   backward data  the same with the gradient, mirrored taps and transposed
//                  weights, the ReLU mask of the layer input in the epilogue;
//   backward wt.   rows = (tap, input channel), K = pixels (a chunk of 512
//                  per CTA, 128 at a time), B = the output gradient;
//                  per-chunk partials reduced in chunk order (deterministic).
// Activations and gradients are stored BF16 (NHWC, channels contiguous),
// master weights and Adam moments FP32.  Softmax, kernel application, loss,
// bias gradients and Adam run on the CUDA cores.
#include <atomic>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "raygen_b200.h"
#include "rg_host.h"
#include "rg_tc.cuh"

namespace rg {

namespace {

// D[M x N] = A[M x K] * B[N x K]^T, one CTA of 128 threads per 128 rows of A.
// A and B are row-major BF16 with K contiguous; M, N, K are checked by the host
// (K % 16 == 0, N % 16 == 0, N <= 128, K <= 256).
__global__ void __launch_bounds__(128) k_tcGemm(int M, int N, int K, const __nv_bfloat16* __restrict__ A,
                                                const __nv_bfloat16* __restrict__ B, float* __restrict__ D,
                                                int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  unsigned char* sA = sm;
  unsigned char* sB = sm + (size_t)128 * K * 2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int row0 = blockIdx.x * 128;
  const uint32_t cols = N <= 32 ? 32u : (N <= 64 ? 64u : 128u);
  if (warp == 0) tc::tmemAlloc(&tbase, cols);
  if (tid == 0) tc::mbarInit(&bar, 1);
  const int kc = K / 8;
  for (int c = tid; c < 128 * kc; c += 128) {
    const int r = c / kc, q = c % kc;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (row0 + r < M) v = *reinterpret_cast<const uint4*>(A + (size_t)(row0 + r) * K + q * 8);
    *reinterpret_cast<uint4*>(sA + tc::chunkOffset(r, q, K)) = v;
  }
  for (int c = tid; c < N * kc; c += 128) {
    const int r = c / kc, q = c % kc;
    *reinterpret_cast<uint4*>(sB + tc::chunkOffset(r, q, K)) =
        *reinterpret_cast<const uint4*>(B + (size_t)r * K + q * 8);
  }
  tc::fenceProxyAsync();  // generic-proxy smem writes -> visible to the tensor core
  __syncthreads();
  tc::fenceAfterSync();
  const uint32_t tmem = tbase;
  if (tid == 0) {
    const uint32_t idesc = tc::instrDescBf16(128, N);
    const uint32_t aBase = tc::smemAddr(sA), bBase = tc::smemAddr(sB);
    const uint32_t sbo = (uint32_t)(K / 8) * 128u;
    for (int s = 0; s < K / 16; ++s)
      tc::mmaBf16(tmem, tc::smemDesc(aBase + s * 256, 128, sbo), tc::smemDesc(bBase + s * 256, 128, sbo), idesc, s > 0);
    tc::commit(&bar);
  }
  const bool ok = __syncthreads_and(tc::mbarWait(&bar, 0)) != 0;
  tc::fenceAfterSync();
  if (ok) {
    for (int c0 = 0; c0 < N; c0 += 32) {
      float v[32];
      tc::tmemLoad32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      const int r = row0 + warp * 32 + lane;
      if (r < M)
        for (int j = 0; j < 32 && c0 + j < N; ++j) D[(size_t)r * N + c0 + j] = v[j];
    }
  } else {
    if (tid == 0) atomicCAS(err, 0, tc::kErrTcTimeout);
    tc::mbarWait(&bar, 0);  // give the MMAs a last bounded chance to drain before freeing TMEM
  }
  tc::fenceBeforeSync();
  __syncthreads();
  if (warp == 0) tc::tmemFree(tmem, cols);
}


// ---------------------------------------------------------------- network --
constexpr int kC = 32;          // hidden channels (and padded logits)
constexpr int kKP = 25;         // predicted kernel taps (5 x 5)
constexpr int kRealInputs = 11; // feature channels that carry data (of 16)
constexpr int kLayers = 6;
__host__ __device__ constexpr int cinOf(int l) { return l == 0 ? 16 : 32; }  // 16, 32, 32, 32, 32, 32
constexpr int kChunk = 512;     // pixels per backward-weight CTA
constexpr int kSub = 128;       // pixels per backward-weight staging step
constexpr float kLossEps = 0.01f;

__host__ __device__ constexpr int layerWeights(int l) { return kC * 9 * cinOf(l); }
__host__ __device__ constexpr int layerOffset(int l) {
  int o = 0;
  for (int i = 0; i < l; ++i) o += layerWeights(i) + kC;
  return o;
}
constexpr int kNumParams = layerOffset(kLayers);

// (b, y, x) of pixel p in a batch of H x W images, neighbour at (dy, dx) or -1
__device__ __forceinline__ int neighbor(int p, int dy, int dx, int H, int W) {
  const int x = p % W, t = p / W, y = t % H, b = t / H;
  const int yy = y + dy, xx = x + dx;
  if (yy < 0 || yy >= H || xx < 0 || xx >= W) return -1;
  return (b * H + yy) * W + xx;
}

__device__ __forceinline__ int clampNeighbor(int p, int dy, int dx, int H, int W) {
  const int x = p % W, t = p / W, y = t % H, b = t / H;
  const int yy = min(max(y + dy, 0), H - 1), xx = min(max(x + dx, 0), W - 1);
  return (b * H + yy) * W + xx;
}

// Softmax of the 25 logits w, in place: the 5 x 5 kernel weights.
__device__ __forceinline__ void softmax25(float (&w)[kKP]) {
  float mx = -3.0e38f;
#pragma unroll
  for (int j = 0; j < kKP; ++j) mx = fmaxf(mx, w[j]);
  float sum = 0.0f;
#pragma unroll
  for (int j = 0; j < kKP; ++j) {
    w[j] = expf(w[j] - mx);
    sum += w[j];
  }
  const float inv = 1.0f / sum;
#pragma unroll
  for (int j = 0; j < kKP; ++j) w[j] *= inv;
}

// Softmax of the 25 logits w (replaced by the kernel weights) and the 5 x 5
// kernel applied to the noisy radiance around pixel p (clamp to edge).
__device__ __forceinline__ void softmaxApply(float (&w)[kKP], int p, int H, int W, const float4* __restrict__ noisy,
                                             float& o0, float& o1, float& o2) {
  softmax25(w);
  o0 = o1 = o2 = 0.0f;
#pragma unroll
  for (int j = 0; j < kKP; ++j) {
    const float4 c = noisy[clampNeighbor(p, j / 5 - 2, j % 5 - 2, H, W)];
    o0 += w[j] * c.x;
    o1 += w[j] * c.y;
    o2 += w[j] * c.z;
  }
}

template <typename T>
__device__ __forceinline__ float loadf(const T* p, size_t i);
template <>
__device__ __forceinline__ float loadf<float>(const float* p, size_t i) { return p[i]; }
template <>
__device__ __forceinline__ float loadf<__half>(const __half* p, size_t i) { return __half2float(p[i]); }

// Features: X0[p] = (log1p(max(rgb, 0)), albedo, normal guide, depth guide,
// log2(1 + spp) / 12, 0 x 5), BF16.  spp: the pixel's sample count from `cnt`
// (the renderer's per-pixel counts, adaptive sampling included) or, without
// it, the image's uniform `spp`.
constexpr float kSppFeatureScale = 1.0f / 12.0f;

template <typename T>
__global__ void k_features(int P, const float4* __restrict__ noisy, const T* __restrict__ normal,
                           const T* __restrict__ albedo, const T* __restrict__ depth, const int* __restrict__ cnt,
                           float spp, __nv_bfloat16* __restrict__ X0) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const float4 c = noisy[p];
  float f[16];
  f[0] = log1pf(fmaxf(c.x, 0.0f));
  f[1] = log1pf(fmaxf(c.y, 0.0f));
  f[2] = log1pf(fmaxf(c.z, 0.0f));
  for (int k = 0; k < 3; ++k) {
    f[3 + k] = loadf(albedo, (size_t)p * 3 + k);
    f[6 + k] = loadf(normal, (size_t)p * 3 + k);
  }
  f[9] = loadf(depth, (size_t)p);
  f[10] = log2f(1.0f + fmaxf(cnt ? (float)cnt[p] : spp, 0.0f)) * kSppFeatureScale;
  for (int k = 11; k < 16; ++k) f[k] = 0.0f;
  __align__(16) __nv_bfloat16 o[16];
  for (int k = 0; k < 16; ++k) o[k] = __float2bfloat16_rn(f[k]);
  uint4* dst = reinterpret_cast<uint4*>(X0 + (size_t)p * 16);
  dst[0] = reinterpret_cast<const uint4*>(o)[0];
  dst[1] = reinterpret_cast<const uint4*>(o)[1];
}

// Strip-pipelined implicit GEMM for the forward and backward-data
// convolutions.  A CTA owns strips of S image rows x 128 columns; one output
// row of a strip (128 pixels) is one M = 128 tile.  Input rows live in a ring
// of kRing row slots in shared memory, each holding pixels x0 - 1 .. x0 + 128
// pixel-major (CIN x 2 bytes per pixel) in the 32- or 64-byte swizzled K-major
// layout: one TMA box of all channels x 130 pixels per row (rows and columns
// outside the image are zero-filled by the copy).  The A operand of tap
// (dy, dx) is a descriptor into the slot of input row y + dy, its start moved
// by 1 + dx pixels (and by 32 bytes for the second K step of 32 channels) --
// no im2col copy, and each input row is loaded once per strip (plus two halo
// rows).  One wide box per row matters: a box of 16-byte rows (one 8-channel
// chunk) costs the copy engine about as much per row as a box of 64-byte rows.
//
// Roles (160 threads):
//  * warp 4, one thread: the producer.  It loads input rows two ahead of the
//    tensor cores and issues the 9 taps x CIN / 16 MMAs of each output row
//    into one of two 32-column TMEM accumulators, committed to
//    tmemFull[row & 1];
//  * warps 0-3: the epilogue.  Each reads its 32 accumulator lanes, frees the
//    accumulator (tmemEmpty) and writes bias + ReLU in BF16, the FP32 logits
//    (LAST), the denoised pixel (LAST and APPLY: softmax of the logits and the
//    5 x 5 kernel applied to the noisy radiance, so the logits never reach
//    memory), or the ReLU-masked data gradient (TRANSPOSED).
// So row r + 1's loads and MMAs overlap row r's epilogue.  Every wait is
// bounded; a wait that runs out sets the error word and the CTA drains its
// outstanding copies and MMAs before it frees the tensor memory.
// Poll limit of the strip pipeline's waits (loads landed, accumulator full /
// empty).  The drain before the CTA exits always uses the full tc::kWaitLimit,
// so a pipeline wait that gives up still lets every issued copy and MMA
// complete before the tensor memory is freed.  A test lowers this limit
// (rg_debug_set_tc_wait_limit) to make the pipeline's waits run out.
__constant__ uint32_t c_pipeWaitLimit = tc::kWaitLimit;
// Only the kernel instantiations launched while a test has lowered the limit read
// it (LIMITED = true); the others keep the compile-time bound, which measured 23%
// faster for the 1080p inference than a bound read from constant memory.
std::atomic<bool> g_pipeLimited{false};

constexpr int kRing = 6;                // input row slots: 3 in use, 1 landing, 2 loading ahead
constexpr int kSlots = 130;             // pixels per slot: x0 - 1 .. x0 + 128
constexpr int kConvThreads = 160;

// Bytes per ring slot (1024-aligned: the swizzle follows the address).
template <int CIN>
__host__ __device__ constexpr int slotBytes() { return (kSlots * CIN * 2 + 1023) / 1024 * 1024; }
template <int CIN>
__host__ __device__ constexpr size_t ringBytes() { return (size_t)kRing * slotBytes<CIN>(); }
template <int CIN>
__host__ __device__ constexpr size_t rowSmem() { return ringBytes<CIN>() + (size_t)kC * 9 * CIN * 2; }

// Forward (TRANSPOSED = false): Y = bf16(relu(conv(X) + b)); LAST: Z = conv(X) + b,
// or with APPLY the denoised image out = kernel(softmax(conv(X) + b)) * noisy.
// Backward data (TRANSPOSED = true, CIN = 32): Y = bf16(mask(Xin) * convT(X = G, Wk = W^T)).
// `xmap` is the tensor map of X ({CIN, W, H, B}, box {8, 130, 1, 1}).
template <int CIN, bool LAST, bool TRANSPOSED, bool APPLY, bool LIMITED>
__global__ void __launch_bounds__(kConvThreads) k_convStrip(const __grid_constant__ CUtensorMap xmap, int B, int H,
                                                            int W, int S, const __nv_bfloat16* __restrict__ Wk,
                                                            const float* __restrict__ bias,
                                                            const __nv_bfloat16* __restrict__ Xin,
                                                            __nv_bfloat16* __restrict__ Y, float* __restrict__ Z,
                                                            const float4* __restrict__ noisy, float4* __restrict__ out,
                                                            int* __restrict__ err) {
  constexpr int CC = CIN / 8, K = 9 * CIN, KC = K / 8;
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t full[kRing], tmemFull[2], tmemEmpty[2];
  __shared__ uint32_t tbase;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ringBase = tc::smemAddr(sm), bBase = ringBase + (uint32_t)ringBytes<CIN>();
  const int tilesPerRow = (W + 127) / 128, stripsY = (H + S - 1) / S, strips = B * stripsY * tilesPerRow;
  if (warp == 0) tc::tmemAlloc(&tbase, 64);
  if (tid == 0) {
    for (int i = 0; i < kRing; ++i) tc::mbarInit(&full[i], 1);
    for (int i = 0; i < 2; ++i) {
      tc::mbarInit(&tmemFull[i], 1);
      tc::mbarInit(&tmemEmpty[i], 128);
    }
    failed = 0;
    tc::fenceBarrierInit();
  }
  for (int c = tid; c < kC * KC; c += kConvThreads) {
    const int r = c / KC, q = c % KC;
    tc::cpAsync16(bBase + tc::chunkOffset(r, q, K), Wk + (size_t)r * K + q * 8, true);
  }
  tc::cpAsyncCommit();
  tc::cpAsyncWait<0>();
  tc::fenceProxyAsync();
  __syncthreads();
  tc::fenceAfterSync();
  const uint32_t tmem = tbase;
  bool ok = true;

  if (warp == 4) {
    if (lane == 0) {
      // ------------------------------------------------------------ producer
      const uint32_t idesc = tc::instrDescBf16(128, kC);
      const uint64_t aDesc0 = CIN == 32 ? tc::smemDescSw64(0) : tc::smemDescSw32(0);
      const uint64_t bDesc0 = tc::smemDesc(bBase, 128, KC * 128);
      int r = 0;      // output rows issued
      int uNext = 0;  // next input row (CTA-local index) to load
      int uBase = 0;  // index of the current strip's first input row
      for (int strip = blockIdx.x; strip < strips && ok; strip += gridDim.x) {
        const int xt = strip % tilesPerRow, sy = (strip / tilesPerRow) % stripsY, b = strip / (tilesPerRow * stripsY);
        const int y0 = sy * S, n = min(S, H - y0), x0 = xt * 128;
        // Ring slots of earlier strips are reused below: their rows' MMAs must be done.
        if (r > 0) ok = tc::mbarWait(&tmemFull[(r - 1) & 1], ((r - 1) >> 1) & 1, LIMITED ? c_pipeWaitLimit : tc::kWaitLimit);
        for (int j = 0; j < n && ok; ++j, ++r) {
          const int t = uBase + j;  // input rows t, t + 1, t + 2 = image rows y0 + j - 1 .. y0 + j + 1
          // The accumulator r & 1 is free once row r - 2's epilogue has read it; that also
          // retires the MMAs of rows up to r - 2, whose ring slots the loads below reuse
          // (input row u goes where row u - kRing <= t - 2 was).
          if (r >= 2 && !(ok = tc::mbarWait(&tmemEmpty[r & 1], ((r - 2) >> 1) & 1, LIMITED ? c_pipeWaitLimit : tc::kWaitLimit))) break;
          for (const int last = min(t + kRing - 2, uBase + n + 1); uNext <= last; ++uNext) {
            const int slot = uNext % kRing, yy = y0 - 1 + (uNext - uBase);
            tc::mbarArriveExpectTx(&full[slot], (uint32_t)(kSlots * CIN * 2));
            tc::tmaLoad4d(ringBase + (uint32_t)(slot * slotBytes<CIN>()), &xmap, 0, x0 - 1, yy, b, &full[slot]);
          }
          for (int i = j == 0 ? 0 : 2; i < 3 && ok; ++i)  // rows t, t + 1 were waited for by row r - 1
            ok = tc::mbarWait(&full[(t + i) % kRing], ((t + i) / kRing) & 1, LIMITED ? c_pipeWaitLimit : tc::kWaitLimit);
          if (!ok) break;
          tc::fenceAfterSync();
          // The issue loop is this thread's whole per-row cost, so the descriptors are a
          // fixed template plus (address >> 4) in the start field, the tap and chunk
          // offsets folded at compile time.
          const uint32_t acc = tmem + (uint32_t)((r & 1) * 32);
          uint32_t rowStart[3];  // start field of input rows t, t + 1, t + 2
#pragma unroll
          for (int i = 0; i < 3; ++i) rowStart[i] = (ringBase + (uint32_t)(((t + i) % kRing) * slotBytes<CIN>())) >> 4;
#pragma unroll
          for (int tap = 0; tap < 9; ++tap) {
            // gradient gathered at p - offset for the data gradient
            const int dy = TRANSPOSED ? 1 - tap / 3 : tap / 3 - 1, dx = TRANSPOSED ? 1 - tap % 3 : tap % 3 - 1;
#pragma unroll
            for (int k = 0; k < CC / 2; ++k)
              tc::mmaBf16(acc, aDesc0 + rowStart[dy + 1] + (uint32_t)(((1 + dx) * CIN * 2 + k * 32) >> 4),
                          bDesc0 + (uint32_t)(((tap * CC + 2 * k) * 128) >> 4), idesc, tap > 0 || k > 0);
          }
          tc::commit(&tmemFull[r & 1]);
        }
        uBase += n + 2;
      }
      // Drain: every issued MMA and every TMA copy has completed before the CTA exits.
      if (r > 0 && !tc::mbarWait(&tmemFull[(r - 1) & 1], ((r - 1) >> 1) & 1)) ok = false;
      for (int u = max(0, uNext - kRing); u < uNext; ++u)
        if (!tc::mbarWait(&full[u % kRing], (u / kRing) & 1)) ok = false;
      if (!ok) failed = 1;
    }
  } else {
    // -------------------------------------------------------------- epilogue
    float bv[kC];
#pragma unroll
    for (int j = 0; j < kC; ++j) bv[j] = TRANSPOSED ? 0.0f : bias[j];
    int r = 0;
    for (int strip = blockIdx.x; strip < strips && ok; strip += gridDim.x) {
      const int xt = strip % tilesPerRow, sy = (strip / tilesPerRow) % stripsY, b = strip / (tilesPerRow * stripsY);
      const int y0 = sy * S, n = min(S, H - y0), x = xt * 128 + warp * 32 + lane;
      for (int j = 0; j < n; ++j, ++r) {
        if (!(ok = tc::mbarWait(&tmemFull[r & 1], (r >> 1) & 1, LIMITED ? c_pipeWaitLimit : tc::kWaitLimit))) break;
        tc::fenceAfterSync();
        float v[32];
        tc::tmemLoad32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)((r & 1) * 32), v);
        tc::fenceBeforeSync();
        tc::mbarArrive(&tmemEmpty[r & 1]);
        if (x < W) {
          const size_t p = ((size_t)(b * H + y0 + j)) * W + x;
          if (LAST && APPLY) {
            float w[kKP];
#pragma unroll
            for (int c = 0; c < kKP; ++c) w[c] = v[c] + bv[c];
            float o0, o1, o2;
            softmaxApply(w, (int)p, H, W, noisy, o0, o1, o2);
            out[p] = make_float4(o0, o1, o2, 1.0f);
          } else if (LAST) {
            float4* z = reinterpret_cast<float4*>(Z + p * kC);
#pragma unroll
            for (int c = 0; c < kC; c += 4)
              z[c / 4] = make_float4(v[c] + bv[c], v[c + 1] + bv[c + 1], v[c + 2] + bv[c + 2], v[c + 3] + bv[c + 3]);
          } else {
            __align__(16) __nv_bfloat16 o[kC];
            if (TRANSPOSED) {
              __align__(16) __nv_bfloat16 xin[kC];
              const uint4* xs = reinterpret_cast<const uint4*>(Xin + p * kC);
#pragma unroll
              for (int c = 0; c < 4; ++c) reinterpret_cast<uint4*>(xin)[c] = xs[c];
#pragma unroll
              for (int c = 0; c < kC; ++c) o[c] = __float2bfloat16_rn(__bfloat162float(xin[c]) > 0.0f ? v[c] : 0.0f);
            } else {
#pragma unroll
              for (int c = 0; c < kC; ++c) o[c] = __float2bfloat16_rn(fmaxf(v[c] + bv[c], 0.0f));
            }
            uint4* yo = reinterpret_cast<uint4*>(Y + p * kC);
#pragma unroll
            for (int c = 0; c < 4; ++c) yo[c] = reinterpret_cast<const uint4*>(o)[c];
          }
        }
      }
    }
    if (!ok) failed = 1;
  }
  tc::fenceBeforeSync();
  __syncthreads();
  if (tid == 0 && failed) atomicCAS(err, 0, tc::kErrTcTimeout);
  if (warp == 0) tc::tmemFree(tmem, 64);
}

// Backward weights: partial[chunk][m = (t, ci)][co] = sum over the chunk's
// pixels q of X[q + off(t)][ci] * G[q][co].  Grid: (M tiles of 128 rows,
// pixel chunks).  Rows beyond 9 * CIN are zero.
template <int CIN>
__global__ void __launch_bounds__(128) k_convBwdWeight(int B, int H, int W, const __nv_bfloat16* __restrict__ X,
                                                       const __nv_bfloat16* __restrict__ G, float* __restrict__ partial,
                                                       int* __restrict__ err) {
  constexpr int M = 9 * CIN;
  __shared__ __align__(1024) unsigned char sA[128 * kSub * 2];
  __shared__ __align__(1024) unsigned char sB[kC * kSub * 2];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int P = B * H * W;
  const int mt = blockIdx.x, chunk = blockIdx.y;
  const int m0 = mt * 128;
  if (warp == 0) tc::tmemAlloc(&tbase, 32);
  if (tid == 0) tc::mbarInit(&bar, 1);
  __syncthreads();
  const uint32_t tmem = tbase;
  const uint32_t idesc = tc::instrDescBf16(128, kC);
  uint32_t phase = 0;
  bool ok = true;
  for (int sub = 0; sub < kChunk / kSub; ++sub) {
    const int q0 = chunk * kChunk + sub * kSub;
    if (q0 >= P) break;
    // thread tid stages pixel q = q0 + tid: its column in A (all rows of this tile) and in B
    const int q = q0 + tid;
    const int kcol = tid;
    auto put = [&](unsigned char* base, int row, __nv_bfloat16 val) {
      *reinterpret_cast<__nv_bfloat16*>(base + tc::chunkOffset(row, kcol >> 3, kSub) + (kcol & 7) * 2) = val;
    };
    for (int r = 0; r < 128; r += CIN) {  // one tap (CIN rows) at a time
      const int m = m0 + r, t = m / CIN;
      __align__(16) __nv_bfloat16 xv[CIN];
#pragma unroll
      for (int j = 0; j < CIN; ++j) xv[j] = __float2bfloat16_rn(0.0f);
      if (m < M && q < P) {
        const int n = neighbor(q, t / 3 - 1, t % 3 - 1, H, W);
        if (n >= 0) {
          const uint4* src = reinterpret_cast<const uint4*>(X + (size_t)n * CIN);
#pragma unroll
          for (int j = 0; j < CIN / 8; ++j) reinterpret_cast<uint4*>(xv)[j] = src[j];
        }
      }
#pragma unroll
      for (int j = 0; j < CIN; ++j) put(sA, r + j, xv[j]);
    }
    {
      __align__(16) __nv_bfloat16 gv[kC];
#pragma unroll
      for (int j = 0; j < kC; ++j) gv[j] = __float2bfloat16_rn(0.0f);
      if (q < P) {
        const uint4* src = reinterpret_cast<const uint4*>(G + (size_t)q * kC);
#pragma unroll
        for (int j = 0; j < 4; ++j) reinterpret_cast<uint4*>(gv)[j] = src[j];
      }
#pragma unroll
      for (int j = 0; j < kC; ++j) put(sB, j, gv[j]);
    }
    tc::fenceProxyAsync();
    __syncthreads();
    tc::fenceAfterSync();
    if (tid == 0) {
      const uint32_t aBase = tc::smemAddr(sA), bBase = tc::smemAddr(sB);
      for (int s = 0; s < kSub / 16; ++s)
        tc::mmaBf16(tmem, tc::smemDesc(aBase + s * 256, 128, (kSub / 8) * 128),
                    tc::smemDesc(bBase + s * 256, 128, (kSub / 8) * 128), idesc, sub > 0 || s > 0);
      tc::commit(&bar);
    }
    ok = __syncthreads_and(tc::mbarWait(&bar, phase)) != 0;
    phase ^= 1u;
    tc::fenceAfterSync();
    if (!ok) break;
  }
  if (ok) {
    float v[32];
    tc::tmemLoad32(tmem + ((uint32_t)(warp * 32) << 16), v);
    const int m = m0 + warp * 32 + lane;
    // a chunk that starts past the end of the batch contributes zeros
    const bool any = chunk * kChunk < P;
    if (m < M) {
      float4* dst = reinterpret_cast<float4*>(partial + ((size_t)chunk * M + m) * kC);
#pragma unroll
      for (int j = 0; j < kC; j += 4)
        dst[j / 4] = any ? make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  } else {
    if (tid == 0) atomicCAS(err, 0, tc::kErrTcTimeout);
    tc::mbarWait(&bar, phase ^ 1u);
  }
  tc::fenceBeforeSync();
  __syncthreads();
  if (warp == 0) tc::tmemFree(tmem, 32);
}

// grad W[co][t][ci] = sum over chunks (in order) of partial[chunk][(t, ci)][co].
__global__ void k_reduceWeightGrad(int M, int chunks, const float* __restrict__ partial, float* __restrict__ gradW) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;  // over M * 32
  if (i >= M * kC) return;
  const int co = i / M, m = i % M;
  float s = 0.0f;
  for (int c = 0; c < chunks; ++c) s += partial[((size_t)c * M + m) * kC + co];
  gradW[(size_t)co * M + m] = s;
}

// grad b[co] = sum_q G[q][co]: per-chunk partials, then an in-order reduction.
__global__ void k_biasPartial(int P, const __nv_bfloat16* __restrict__ G, float* __restrict__ partial) {
  const int chunk = blockIdx.x, co = threadIdx.x & 31, lane4 = threadIdx.x >> 5;  // 128 threads: 4 pixel lanes
  __shared__ float acc[4][kC];
  float s = 0.0f;
  for (int q = chunk * kChunk + lane4; q < min(P, (chunk + 1) * kChunk); q += 4) s += __bfloat162float(G[(size_t)q * kC + co]);
  acc[lane4][co] = s;
  __syncthreads();
  if (lane4 == 0) partial[(size_t)chunk * kC + co] = ((acc[0][co] + acc[1][co]) + acc[2][co]) + acc[3][co];
}

__global__ void k_reduceBiasGrad(int chunks, const float* __restrict__ partial, float* __restrict__ gradB) {
  const int co = threadIdx.x;
  if (co >= kC) return;
  float s = 0.0f;
  for (int c = 0; c < chunks; ++c) s += partial[(size_t)c * kC + co];
  gradB[co] = s;
}

// Softmax + 5 x 5 kernel application.  TRAIN: also the relMSE loss and its
// gradient with respect to the logits, G[p][0..24] (BF16), zero for the pad.
template <bool TRAIN>
__global__ void k_head(int B, int H, int W, const float* __restrict__ Z, const float4* __restrict__ noisy,
                       const float4* __restrict__ ref, float4* __restrict__ out, __nv_bfloat16* __restrict__ G,
                       float* __restrict__ lossSum) {
  const int P = B * H * W;
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  float lp = 0.0f;
  if (p < P) {
    float w[kKP];
    const float* z = Z + (size_t)p * kC;
#pragma unroll
    for (int j = 0; j < kKP; ++j) w[j] = z[j];
    float o0, o1, o2;
    softmaxApply(w, p, H, W, noisy, o0, o1, o2);
    if (out) out[p] = make_float4(o0, o1, o2, 1.0f);
    if (TRAIN) {
      const float4 r = ref[p];
      const float d0 = 1.0f / (r.x * r.x + kLossEps), d1 = 1.0f / (r.y * r.y + kLossEps),
                  d2 = 1.0f / (r.z * r.z + kLossEps);
      lp = (o0 - r.x) * (o0 - r.x) * d0 + (o1 - r.y) * (o1 - r.y) * d1 + (o2 - r.z) * (o2 - r.z) * d2;
      const float sc = 2.0f / (3.0f * (float)P);
      const float g0 = sc * (o0 - r.x) * d0, g1 = sc * (o1 - r.y) * d1, g2 = sc * (o2 - r.z) * d2;
      float dw[kKP];
      float dot = 0.0f;
#pragma unroll
      for (int j = 0; j < kKP; ++j) {
        const float4 c = noisy[clampNeighbor(p, j / 5 - 2, j % 5 - 2, H, W)];
        dw[j] = g0 * c.x + g1 * c.y + g2 * c.z;
        dot += w[j] * dw[j];
      }
      __align__(16) __nv_bfloat16 gz[kC];
#pragma unroll
      for (int j = 0; j < kC; ++j) gz[j] = __float2bfloat16_rn(j < kKP ? w[j] * (dw[j] - dot) : 0.0f);
      uint4* dst = reinterpret_cast<uint4*>(G + (size_t)p * kC);
#pragma unroll
      for (int j = 0; j < 4; ++j) dst[j] = reinterpret_cast<const uint4*>(gz)[j];
    }
  }
  if (TRAIN) {
    __shared__ float red[256];
    red[threadIdx.x] = lp;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(lossSum, red[0] / (3.0f * (float)P));
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters.
// Adam; the step number t = state[1] + 1 is read on the device so that a
// captured training step can be replayed.
__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, const int* __restrict__ state, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = (float)(state[1] + 1);
  const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi, vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// One training example on the device: features, noisy radiance, reference.
struct ExampleRef {
  const __nv_bfloat16* x;
  const float4* noisy;
  const float4* ref;
};

// The batch of training step state[0]: example picks[step * B + b] into slot b.
__global__ void k_gatherBatch(int B, int Pi, const int* __restrict__ picks, const int* __restrict__ state,
                              const ExampleRef* __restrict__ ex, __nv_bfloat16* __restrict__ X0,
                              float4* __restrict__ noisy, float4* __restrict__ ref) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (size_t)B * Pi) return;
  const int b = (int)(i / Pi), p = (int)(i % Pi);
  const ExampleRef e = ex[picks[state[0] * B + b]];
  const uint4* xs = reinterpret_cast<const uint4*>(e.x + (size_t)p * 16);
  uint4* xd = reinterpret_cast<uint4*>(X0 + i * 16);
  xd[0] = xs[0];
  xd[1] = xs[1];
  noisy[i] = e.noisy[p];
  ref[i] = e.ref[p];
}

// End of a training step: its loss into the history, next step, one more Adam step.
__global__ void k_stepEnd(int* __restrict__ state, const float* __restrict__ loss, float* __restrict__ hist) {
  hist[state[0]] = *loss;
  state[0]++;
  state[1]++;
}

// Master FP32 weights -> BF16 forward layout [co][(t, ci)] and the transposed
// backward-data layout [ci][(t, co)] (32-channel inputs only).
__global__ void k_packWeights(const float* __restrict__ params, __nv_bfloat16* __restrict__ wf,
                              __nv_bfloat16* __restrict__ wt, int layer) {
  const int cin = layer == 0 ? 16 : 32;
  const int n = kC * 9 * cin;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* W = params + layerOffset(layer);
  const int co = i / (9 * cin), rem = i % (9 * cin), t = rem / cin, ci = rem % cin;
  const __nv_bfloat16 b = __float2bfloat16_rn(W[i]);
  wf[i] = b;
  if (wt) wt[(size_t)ci * (9 * kC) + t * kC + co] = b;
}

}  // namespace

}  // namespace rg

using namespace rg;

extern "C" rg_status rg_tc_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B,
                                     float* D) {
  if (M <= 0 || !A || !B || !D || N < 16 || N > 128 || N % 16 || K < 16 || K > 256 || K % 16) {
    setLastError("rg_tc_gemm_bf16: need M > 0, N in 16..128 and K in 16..256, both multiples of 16");
    return RG_ERR_INVALID_ARGUMENT;
  }
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  DevBuf<__nv_bfloat16> a, b;
  DevBuf<float> d;
  DevBuf<int> err;
  if (!a.upload(reinterpret_cast<const __nv_bfloat16*>(A), (size_t)M * K, 0) ||
      !b.upload(reinterpret_cast<const __nv_bfloat16*>(B), (size_t)N * K, 0) || !d.alloc((size_t)M * N) ||
      !err.alloc(1))
    return RG_ERR_OUT_OF_MEMORY;
  cudaMemsetAsync(err.p, 0, sizeof(int), 0);
  const size_t smem = (size_t)(128 + N) * K * 2;
  cudaFuncSetAttribute(k_tcGemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_tcGemm<<<(M + 127) / 128, 128, smem, 0>>>(M, N, K, a.p, b.p, d.p, err.p);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    setLastError(std::string("rg_tc_gemm_bf16: ") + cudaGetErrorString(e));
    return RG_ERR_CUDA;
  }
  int flag = 0;
  cudaMemcpy(&flag, err.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (flag) {
    setLastError("rg_tc_gemm_bf16: tensor-core completion wait timed out");
    return RG_ERR_DEVICE_STATUS;
  }
  cudaMemcpy(D, d.p, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost);
  return RG_OK;
}

// ------------------------------------------------------------------ host --
#define RG_CUDA_CHECK(call)                                              \
  do {                                                                   \
    cudaError_t e__ = (call);                                            \
    if (e__ != cudaSuccess) {                                            \
      setLastError(std::string(#call) + ": " + cudaGetErrorString(e__)); \
      return RG_ERR_CUDA;                                                \
    }                                                                    \
  } while (0)

namespace rg {

namespace {
// out = noisy * (1 - t) + denoised * t, t = clamp(intensity, 0, 1) (the blend of denoiseImage).
__global__ void k_blend(int n, const float4* __restrict__ noisy, const float4* __restrict__ den, float intensity,
                        float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = fminf(fmaxf(intensity, 0.0f), 1.0f), s = 1.0f - t;
  const float4 a = noisy[i], b = den[i];
  out[i] = make_float4(a.x * s + b.x * t, a.y * s + b.y * t, a.z * s + b.z * t, 1.0f);
}
}  // namespace

struct KpcnNet {
  std::mutex mu;  // one user of the work buffers at a time (renderers, servers, API calls)
  cudaStream_t st = nullptr;
  int numSMs = 148;
  bool mapFailed = false;                  // a convolution's tensor map could not be encoded
  DevBuf<float> params, grad, m, v;
  DevBuf<__nv_bfloat16> wf[kLayers], wt[kLayers];
  float lastApplyMs = 0.0f, lastStepMs = 0.0f;  // device time of the last apply / mean training step
  std::mt19937 rng;
  int perSm[5] = {1, 1, 1, 1, 1};  // resident strip-convolution CTAs per SM, by kernel variant (convVariant)
  // training examples (all W x H)
  int dsW = 0, dsH = 0, dsN = 0;
  std::vector<__nv_bfloat16*> exX;
  std::vector<float4*> exNoisy, exRef;
  // A training step is captured once and replayed as a CUDA graph; what changes
  // between steps lives on the device: state[0] = step of the current train()
  // call, state[1] = Adam steps taken; the example picks of every step and the
  // loss history of the call.
  DevBuf<int> state, picks;
  DevBuf<float> lossHist;
  DevBuf<ExampleRef> exRefs;
  bool exDirty = true;
  cudaGraphExec_t trainGraph = nullptr;
  std::string trainKey;
  // work buffers for P pixels
  size_t cap = 0;
  DevBuf<__nv_bfloat16> X0, act[kLayers - 1], gA, gB;
  DevBuf<float> Z, partial, bpartial, loss;
  DevBuf<float4> noisy, ref, out;
  DevBuf<int> err;
  ~KpcnNet() {
    if (trainGraph) cudaGraphExecDestroy(trainGraph);
    for (auto* p : exX) cudaFree(p);
    for (auto* p : exNoisy) cudaFree(p);
    for (auto* p : exRef) cudaFree(p);
    if (st) cudaStreamDestroy(st);
  }
};

namespace {

int chunksFor(size_t P) { return (int)((P + kChunk - 1) / kChunk); }

bool ensureWork(KpcnNet& n, size_t P) {
  if (P <= n.cap) return true;
  const int ch = chunksFor(P);
  bool ok = n.X0.alloc(P * 16) && n.gA.alloc(P * kC) && n.gB.alloc(P * kC) && n.Z.alloc(P * kC) &&
            n.partial.alloc((size_t)ch * 9 * kC * kC) && n.bpartial.alloc((size_t)ch * kC) && n.loss.alloc(1) &&
            n.noisy.alloc(P) && n.ref.alloc(P) && n.out.alloc(P) && n.err.alloc(1);
  for (int l = 0; l < kLayers - 1; ++l) ok = ok && n.act[l].alloc(P * kC);
  if (ok) {
    n.cap = P;
    ok = cudaMemsetAsync(n.err.p, 0, sizeof(int), n.st) == cudaSuccess;  // the error word starts clear
  }
  return ok;
}

// Dynamic shared memory above the default limit, and the largest shared-memory
// carveout, so that as many CTAs as the memory allows are resident per SM (the
// occupancy query below sees the same preference).
template <typename K>
void setSmem(K kernel, size_t bytes) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
}

void packWeights(KpcnNet& n) {
  for (int l = 0; l < kLayers; ++l) {
    const int cnt = layerWeights(l);
    k_packWeights<<<(cnt + 255) / 256, 256, 0, n.st>>>(n.params.p, n.wf[l].p, l > 0 ? n.wt[l].p : nullptr, l);
  }
}

// Resident CTAs per SM of a strip-convolution kernel, from its shared memory,
// registers, threads and tensor-memory columns (64 per CTA).  The runtime's
// occupancy query answers one CTA per SM for these tensor-memory kernels,
// while the SM runs as many as these resources allow.
template <typename K>
int stripResidency(K kernel, size_t dynSmem) {
  int dev = 0, smemSm = 0, reserved = 0, regsSm = 0, thrSm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&smemSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
  cudaDeviceGetAttribute(&regsSm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
  cudaDeviceGetAttribute(&thrSm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
    cudaGetLastError();
    return 1;
  }
  const int bySmem = smemSm / (int)(fa.sharedSizeBytes + dynSmem + (size_t)reserved);
  const int regsPerCta = (fa.numRegs + 7) / 8 * 8 * kConvThreads;  // registers are allocated 8 per thread at a time
  const int byRegs = regsPerCta > 0 ? regsSm / regsPerCta : 16;
  const int byTmem = 512 / 64;
  return std::max(1, std::min({bySmem, byRegs, thrSm / kConvThreads, byTmem}));
}

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
PFN_cuTensorMapEncodeTiled_v12000 tensorMapEncoder() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      f = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// Tensor map of a BF16 NHWC activation [B][H][W][C], C = 16 or 32: boxes of all
// channels x 130 pixels of one row (32- / 64-byte swizzle), zero fill outside
// the tensor.
bool rowMap(CUtensorMap& m, const __nv_bfloat16* X, int B, int H, int W, int C) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensorMapEncoder();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
  const cuuint64_t strides[3] = {(cuuint64_t)C * 2, (cuuint64_t)W * C * 2, (cuuint64_t)H * W * C * 2};
  // one box of all channels per row, with the swizzle the convolution's descriptors read
  if (C != 16 && C != 32) return false;
  const cuuint32_t box[4] = {(cuuint32_t)C, (cuuint32_t)kSlots, 1, 1};
  const cuuint32_t elemStrides[4] = {1, 1, 1, 1};
  return enc(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<__nv_bfloat16*>(X), dims, strides, box, elemStrides,
             CU_TENSOR_MAP_INTERLEAVE_NONE, C == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Strip height S and grid for B images of H rows x ceil(W / 128) column tiles
// on `slots` resident CTAs: the fewest rounds of strips, a strip of S rows
// costing S + 2 row loads (two halo rows) and about one row of pipeline fill.
void stripPlan(int B, int H, int W, int slots, int& grid, int& S) {
  const long tiles = (long)B * ((W + 127) / 128);
  long best = -1;
  S = 1;
  for (int s = 1; s <= H && s <= 256; ++s) {
    const long strips = tiles * ((H + s - 1) / s), rounds = (strips + slots - 1) / slots, cost = rounds * (s + 3);
    if (best < 0 || cost < best) {
      best = cost;
      S = s;
    }
  }
  grid = (int)std::min<long>(tiles * ((H + S - 1) / S), slots);
}

// Index of a strip-convolution variant in KpcnNet::perSm.
constexpr int convVariant(int cin, bool last, bool transposed, bool apply) {
  return cin == 16 ? 0 : transposed ? 4 : !last ? 1 : apply ? 3 : 2;
}

template <int CIN, bool LAST, bool TRANSPOSED, bool APPLY = false>
void launchConv(KpcnNet& n, int B, int H, int W, const __nv_bfloat16* X, const __nv_bfloat16* Wk, const float* bias,
                const __nv_bfloat16* Xin, __nv_bfloat16* Y, float* Z, const float4* noisy = nullptr,
                float4* out = nullptr) {
  CUtensorMap m;
  if (!rowMap(m, X, B, H, W, CIN)) {
    n.mapFailed = true;
    return;
  }
  int grid = 1, S = 1;
  stripPlan(B, H, W, n.numSMs * n.perSm[convVariant(CIN, LAST, TRANSPOSED, APPLY)], grid, S);
  if (g_pipeLimited.load())
    k_convStrip<CIN, LAST, TRANSPOSED, APPLY, true><<<grid, kConvThreads, rowSmem<CIN>(), n.st>>>(
        m, B, H, W, S, Wk, bias, Xin, Y, Z, noisy, out, n.err.p);
  else
    k_convStrip<CIN, LAST, TRANSPOSED, APPLY, false><<<grid, kConvThreads, rowSmem<CIN>(), n.st>>>(
        m, B, H, W, S, Wk, bias, Xin, Y, Z, noisy, out, n.err.p);
}

// X0 must be filled; writes act[0..4] and Z, or with `out` the denoised image
// (softmax and kernel application fused into the last convolution).
void forward(KpcnNet& n, int B, int H, int W, const float4* noisy = nullptr, float4* out = nullptr) {
  launchConv<16, false, false>(n, B, H, W, n.X0.p, n.wf[0].p, n.params.p + layerOffset(0) + layerWeights(0), nullptr,
                               n.act[0].p, nullptr);
  for (int l = 1; l < kLayers - 1; ++l)
    launchConv<32, false, false>(n, B, H, W, n.act[l - 1].p, n.wf[l].p, n.params.p + layerOffset(l) + layerWeights(l),
                                 nullptr, n.act[l].p, nullptr);
  const float* lastBias = n.params.p + layerOffset(kLayers - 1) + layerWeights(kLayers - 1);
  if (out)
    launchConv<32, true, false, true>(n, B, H, W, n.act[kLayers - 2].p, n.wf[kLayers - 1].p, lastBias, nullptr,
                                      nullptr, nullptr, noisy, out);
  else
    launchConv<32, true, false>(n, B, H, W, n.act[kLayers - 2].p, n.wf[kLayers - 1].p, lastBias, nullptr, nullptr,
                                n.Z.p);
}

// Head gradient must be in gA; fills n.grad.
void backward(KpcnNet& n, int B, int H, int W) {
  const size_t P = (size_t)B * H * W;
  const int ch = chunksFor(P);
  __nv_bfloat16* G = n.gA.p;
  __nv_bfloat16* Gn = n.gB.p;
  for (int l = kLayers - 1; l >= 0; --l) {
    const __nv_bfloat16* in = l == 0 ? n.X0.p : n.act[l - 1].p;
    const int M = 9 * cinOf(l);
    const dim3 g((M + 127) / 128, ch);
    if (l == 0) k_convBwdWeight<16><<<g, 128, 0, n.st>>>(B, H, W, in, G, n.partial.p, n.err.p);
    else k_convBwdWeight<32><<<g, 128, 0, n.st>>>(B, H, W, in, G, n.partial.p, n.err.p);
    k_reduceWeightGrad<<<(M * kC + 255) / 256, 256, 0, n.st>>>(M, ch, n.partial.p, n.grad.p + layerOffset(l));
    k_biasPartial<<<ch, 128, 0, n.st>>>((int)P, G, n.bpartial.p);
    k_reduceBiasGrad<<<1, 32, 0, n.st>>>(ch, n.bpartial.p, n.grad.p + layerOffset(l) + layerWeights(l));
    if (l > 0) {
      launchConv<32, false, true>(n, B, H, W, G, n.wt[l].p, nullptr, in, Gn, nullptr);
      std::swap(G, Gn);
    }
  }
}

rg_status setPipeWaitLimit(uint32_t polls) {
  const uint32_t v = polls ? polls : tc::kWaitLimit;
  const cudaError_t e = cudaMemcpyToSymbol(c_pipeWaitLimit, &v, sizeof(v));
  if (e == cudaSuccess) g_pipeLimited.store(polls != 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    setLastError(std::string("rg_debug_set_tc_wait_limit: ") + cudaGetErrorString(e));
    return RG_ERR_CUDA;
  }
  return RG_OK;
}

rg_status checkErr(KpcnNet& n, const char* what) {
  if (n.mapFailed) {
    n.mapFailed = false;
    cudaStreamSynchronize(n.st);
    setLastError(std::string(what) + ": the driver could not encode a TMA tensor map");
    return RG_ERR_CUDA;
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(n.st);
  if (e != cudaSuccess) {
    setLastError(std::string(what) + ": " + cudaGetErrorString(e));
    return RG_ERR_CUDA;
  }
  int flag = 0;
  cudaMemcpy(&flag, n.err.p, sizeof(int), cudaMemcpyDeviceToHost);
  if (flag) {
    cudaMemset(n.err.p, 0, sizeof(int));  // reported once
    setLastError(std::string(what) + ": tensor-core completion wait timed out");
    return RG_ERR_DEVICE_STATUS;
  }
  return RG_OK;
}

bool initNet(KpcnNet& n, uint32_t seed) {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n.numSMs, cudaDevAttrMultiProcessorCount, dev);
  if (cudaStreamCreateWithFlags(&n.st, cudaStreamNonBlocking) != cudaSuccess) return false;
  n.rng.seed(seed);
  bool ok = n.params.alloc(kNumParams) && n.grad.alloc(kNumParams) && n.m.alloc(kNumParams) && n.v.alloc(kNumParams);
  for (int l = 0; l < kLayers && ok; ++l) {
    ok = n.wf[l].alloc(layerWeights(l));
    if (l > 0) ok = ok && n.wt[l].alloc(layerWeights(l));
  }
  if (!ok) return false;
  // He-normal weights (fan-in 9 x input channels; 11 real inputs for layer 1),
  // zero biases, the last layer scaled by 0.1 and its 7 padding logits zero.
  std::vector<float> h(kNumParams, 0.0f);
  std::normal_distribution<float> nd(0.0f, 1.0f);
  for (int l = 0; l < kLayers; ++l) {
    const int cin = cinOf(l), fan = 9 * (l == 0 ? kRealInputs : cin);
    const float sd = std::sqrt(2.0f / fan) * (l == kLayers - 1 ? 0.1f : 1.0f);
    float* W = h.data() + layerOffset(l);
    for (int co = 0; co < kC; ++co)
      for (int t = 0; t < 9; ++t)
        for (int ci = 0; ci < cin; ++ci) {
          const bool pad = (l == 0 && ci >= kRealInputs) || (l == kLayers - 1 && co >= kKP);
          W[(co * 9 + t) * cin + ci] = pad ? 0.0f : nd(n.rng) * sd;
        }
  }
  cudaMemcpyAsync(n.params.p, h.data(), sizeof(float) * kNumParams, cudaMemcpyHostToDevice, n.st);
  cudaMemsetAsync(n.m.p, 0, sizeof(float) * kNumParams, n.st);
  cudaMemsetAsync(n.v.p, 0, sizeof(float) * kNumParams, n.st);
  setSmem(k_convStrip<16, false, false, false, false>, rowSmem<16>());
  setSmem(k_convStrip<16, false, false, false, true>, rowSmem<16>());
  setSmem(k_convStrip<32, false, false, false, false>, rowSmem<32>());
  setSmem(k_convStrip<32, false, false, false, true>, rowSmem<32>());
  setSmem(k_convStrip<32, true, false, false, false>, rowSmem<32>());
  setSmem(k_convStrip<32, true, false, false, true>, rowSmem<32>());
  setSmem(k_convStrip<32, true, false, true, false>, rowSmem<32>());
  setSmem(k_convStrip<32, true, false, true, true>, rowSmem<32>());
  setSmem(k_convStrip<32, false, true, false, false>, rowSmem<32>());
  setSmem(k_convStrip<32, false, true, false, true>, rowSmem<32>());
  n.perSm[convVariant(16, false, false, false)] = stripResidency(k_convStrip<16, false, false, false, false>, rowSmem<16>());
  n.perSm[convVariant(32, false, false, false)] = stripResidency(k_convStrip<32, false, false, false, false>, rowSmem<32>());
  n.perSm[convVariant(32, true, false, false)] = stripResidency(k_convStrip<32, true, false, false, false>, rowSmem<32>());
  n.perSm[convVariant(32, true, false, true)] = stripResidency(k_convStrip<32, true, false, true, false>, rowSmem<32>());
  n.perSm[convVariant(32, false, true, false)] = stripResidency(k_convStrip<32, false, true, false, false>, rowSmem<32>());
  if (!n.state.alloc(2) || cudaMemsetAsync(n.state.p, 0, 2 * sizeof(int), n.st) != cudaSuccess) return false;
  packWeights(n);
  return cudaStreamSynchronize(n.st) == cudaSuccess;
}

// Upload host images (n images of w x h) into the work buffers and build X0.
bool uploadInputs(KpcnNet& n, size_t P, const float* noisy, const float* normal, const float* albedo, const float* depth,
                  float spp, const float* ref) {
  DevBuf<float> nb, ab, db;
  if (!nb.upload(normal, P * 3, n.st) || !ab.upload(albedo, P * 3, n.st) || !db.upload(depth, P, n.st)) return false;
  if (cudaMemcpyAsync(n.noisy.p, noisy, sizeof(float4) * P, cudaMemcpyHostToDevice, n.st) != cudaSuccess) return false;
  if (ref && cudaMemcpyAsync(n.ref.p, ref, sizeof(float4) * P, cudaMemcpyHostToDevice, n.st) != cudaSuccess) return false;
  k_features<float><<<(unsigned)((P + 255) / 256), 256, 0, n.st>>>((int)P, n.noisy.p, nb.p, ab.p, db.p, nullptr, spp,
                                                                   n.X0.p);
  return cudaStreamSynchronize(n.st) == cudaSuccess;  // the temporaries die here
}

}  // namespace

// Denoise W x H on the device: noisy float4 HDR, half guides (the renderer's
// AOV buffers), result into out (may alias nothing else); intensity blends
// with the noisy image as denoiseImage does.
rg_status kpcnDenoiseDevice(KpcnNet& n, int W, int H, const float4* noisy, const __half* normal, const __half* albedo,
                            const __half* depth, const int* cnt, float intensity, float4* out, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(n.mu);
  const size_t P = (size_t)W * H;
  if (!ensureWork(n, P)) {
    setLastError("learned denoiser: out of device memory");
    return RG_ERR_OUT_OF_MEMORY;
  }
  cudaEvent_t ev;
  cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  cudaEventRecord(ev, st);
  cudaStreamWaitEvent(n.st, ev, 0);
  k_features<__half><<<(unsigned)((P + 255) / 256), 256, 0, n.st>>>((int)P, noisy, normal, albedo, depth, cnt, 0.0f,
                                                                    n.X0.p);
  forward(n, 1, H, W, noisy, n.out.p);
  const rg_status rs = checkErr(n, "learned denoiser");
  if (rs != RG_OK) {
    cudaEventDestroy(ev);
    return rs;
  }
  // the renderer's stream waits for the denoiser before blending
  cudaEventRecord(ev, n.st);
  cudaStreamWaitEvent(st, ev, 0);
  k_blend<<<(unsigned)((P + 255) / 256), 256, 0, st>>>((int)P, noisy, n.out.p, intensity, out);
  cudaEventDestroy(ev);
  return RG_OK;
}

}  // namespace rg

struct rg_denoiser {
  rg::KpcnNet net;
};

namespace rg {
KpcnNet* kpcnOf(rg_denoiser* d) { return d ? &d->net : nullptr; }
}  // namespace rg

extern "C" {

rg_status rg_debug_set_tc_wait_limit(uint32_t polls) { return rg::setPipeWaitLimit(polls); }

int32_t rg_denoiser_num_params(void) { return rg::kNumParams; }

rg_status rg_denoiser_create(uint32_t seed, rg_denoiser** out) {
  if (!out) return RG_ERR_INVALID_ARGUMENT;
  int dc = 0;
  if (cudaGetDeviceCount(&dc) != cudaSuccess || dc == 0) {
    cudaGetLastError();
    return RG_ERR_NO_DEVICE;
  }
  std::unique_ptr<rg_denoiser> d(new rg_denoiser());
  if (!rg::initNet(d->net, seed)) {
    setLastError("learned denoiser: device set-up failed");
    return RG_ERR_OUT_OF_MEMORY;
  }
  *out = d.release();
  return RG_OK;
}

rg_status rg_denoiser_destroy(rg_denoiser* d) {
  delete d;
  return RG_OK;
}

rg_status rg_denoiser_get_params(rg_denoiser* d, float* out, size_t n) {
  if (!d || !out || n < (size_t)rg::kNumParams) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(d->net.mu);
  RG_CUDA_CHECK(cudaMemcpyAsync(out, d->net.params.p, sizeof(float) * rg::kNumParams, cudaMemcpyDeviceToHost, d->net.st));
  RG_CUDA_CHECK(cudaStreamSynchronize(d->net.st));
  return RG_OK;
}

rg_status rg_denoiser_set_params(rg_denoiser* d, const float* in, size_t n) {
  if (!d || !in || n != (size_t)rg::kNumParams) return RG_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(d->net.mu);
  RG_CUDA_CHECK(cudaMemcpyAsync(d->net.params.p, in, sizeof(float) * rg::kNumParams, cudaMemcpyHostToDevice, d->net.st));
  RG_CUDA_CHECK(cudaMemsetAsync(d->net.m.p, 0, sizeof(float) * rg::kNumParams, d->net.st));
  RG_CUDA_CHECK(cudaMemsetAsync(d->net.v.p, 0, sizeof(float) * rg::kNumParams, d->net.st));
  RG_CUDA_CHECK(cudaMemsetAsync(d->net.state.p, 0, 2 * sizeof(int), d->net.st));  // Adam restarts
  rg::packWeights(d->net);
  RG_CUDA_CHECK(cudaStreamSynchronize(d->net.st));
  return RG_OK;
}

rg_status rg_denoiser_add_example(rg_denoiser* d, int32_t w, int32_t h, const float* noisy_rgba, const float* normal,
                                  const float* albedo, const float* depth, float spp, const float* ref_rgba) {
  if (!d || w <= 0 || h <= 0 || !noisy_rgba || !normal || !albedo || !depth || !ref_rgba || !(spp >= 0.0f))
    return RG_ERR_INVALID_ARGUMENT;
  rg::KpcnNet& n = d->net;
  std::lock_guard<std::mutex> lk(n.mu);
  if (n.dsN > 0 && (w != n.dsW || h != n.dsH)) {
    setLastError("learned denoiser: every training example must have the same size");
    return RG_ERR_INVALID_ARGUMENT;
  }
  const size_t P = (size_t)w * h;
  if (!rg::ensureWork(n, P) || !rg::uploadInputs(n, P, noisy_rgba, normal, albedo, depth, spp, ref_rgba))
    return RG_ERR_OUT_OF_MEMORY;
  __nv_bfloat16* x = nullptr;
  float4 *nz = nullptr, *rf = nullptr;
  if (cudaMalloc(&x, P * 16 * sizeof(__nv_bfloat16)) != cudaSuccess || cudaMalloc(&nz, P * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&rf, P * sizeof(float4)) != cudaSuccess) {
    cudaFree(x);
    cudaFree(nz);
    cudaFree(rf);
    setLastError("learned denoiser: out of device memory (examples)");
    return RG_ERR_OUT_OF_MEMORY;
  }
  cudaMemcpyAsync(x, n.X0.p, P * 16 * sizeof(__nv_bfloat16), cudaMemcpyDeviceToDevice, n.st);
  cudaMemcpyAsync(nz, n.noisy.p, P * sizeof(float4), cudaMemcpyDeviceToDevice, n.st);
  cudaMemcpyAsync(rf, n.ref.p, P * sizeof(float4), cudaMemcpyDeviceToDevice, n.st);
  RG_CUDA_CHECK(cudaStreamSynchronize(n.st));
  n.exX.push_back(x);
  n.exNoisy.push_back(nz);
  n.exRef.push_back(rf);
  n.exDirty = true;
  n.dsW = w;
  n.dsH = h;
  n.dsN++;
  return RG_OK;
}

rg_status rg_denoiser_clear_examples(rg_denoiser* d) {
  if (!d) return RG_ERR_INVALID_ARGUMENT;
  rg::KpcnNet& n = d->net;
  std::lock_guard<std::mutex> lk(n.mu);
  for (auto* p : n.exX) cudaFree(p);
  for (auto* p : n.exNoisy) cudaFree(p);
  for (auto* p : n.exRef) cudaFree(p);
  n.exX.clear();
  n.exNoisy.clear();
  n.exRef.clear();
  n.exDirty = true;
  n.dsN = 0;
  return RG_OK;
}

rg_status rg_denoiser_train(rg_denoiser* d, int32_t steps, int32_t batch, float lr, float* losses) {
  if (!d || steps < 0 || batch <= 0) return RG_ERR_INVALID_ARGUMENT;
  rg::KpcnNet& n = d->net;
  std::lock_guard<std::mutex> lk(n.mu);
  if (n.dsN == 0) {
    setLastError("learned denoiser: no training examples");
    return RG_ERR_INVALID_ARGUMENT;
  }
  const int B = batch, H = n.dsH, W = n.dsW;
  const size_t Pi = (size_t)H * W, P = Pi * B;
  if (!rg::ensureWork(n, P)) return RG_ERR_OUT_OF_MEMORY;
  if (steps == 0) return RG_OK;
  // the picks of every step, drawn in the order of the host generator
  std::uniform_int_distribution<int> pick(0, n.dsN - 1);
  std::vector<int> pk((size_t)steps * B);
  for (auto& e : pk) e = pick(n.rng);
  if (!n.picks.upload(pk.data(), pk.size(), n.st) || !n.lossHist.alloc((size_t)steps)) return RG_ERR_OUT_OF_MEMORY;
  if (n.exDirty) {
    std::vector<rg::ExampleRef> ex(n.dsN);
    for (int i = 0; i < n.dsN; ++i) ex[i] = {n.exX[i], n.exNoisy[i], n.exRef[i]};
    if (!n.exRefs.upload(ex.data(), ex.size(), n.st)) return RG_ERR_OUT_OF_MEMORY;
    n.exDirty = false;
  }
  RG_CUDA_CHECK(cudaMemsetAsync(n.state.p, 0, sizeof(int), n.st));  // step 0 of this call
  uint32_t lrBits;
  std::memcpy(&lrBits, &lr, sizeof(lrBits));
  const std::string key = std::to_string(B) + ":" + std::to_string(H) + ":" + std::to_string(W) + ":" +
                          std::to_string(lrBits) + ":" + std::to_string(n.cap) + ":" +
                          std::to_string((uintptr_t)n.X0.p) + ":" + std::to_string((uintptr_t)n.picks.p) + ":" +
                          std::to_string((uintptr_t)n.lossHist.p) + ":" + std::to_string((uintptr_t)n.exRefs.p) + ":" +
                          std::to_string((int)rg::g_pipeLimited.load());
  if (!n.trainGraph || n.trainKey != key) {
    if (n.trainGraph) {
      cudaGraphExecDestroy(n.trainGraph);
      n.trainGraph = nullptr;
    }
    cudaGraph_t g;
    RG_CUDA_CHECK(cudaStreamBeginCapture(n.st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(n.loss.p, 0, sizeof(float), n.st);
    rg::k_gatherBatch<<<(unsigned)((P + 255) / 256), 256, 0, n.st>>>(B, (int)Pi, n.picks.p, n.state.p, n.exRefs.p,
                                                                     n.X0.p, n.noisy.p, n.ref.p);
    rg::forward(n, B, H, W);
    rg::k_head<true><<<(unsigned)((P + 255) / 256), 256, 0, n.st>>>(B, H, W, n.Z.p, n.noisy.p, n.ref.p, nullptr, n.gA.p,
                                                                     n.loss.p);
    rg::backward(n, B, H, W);
    rg::k_adam<<<(rg::kNumParams + 255) / 256, 256, 0, n.st>>>(rg::kNumParams, n.params.p, n.grad.p, n.m.p, n.v.p, lr,
                                                               0.9f, 0.999f, n.state.p, 1e-8f);
    rg::packWeights(n);
    rg::k_stepEnd<<<1, 1, 0, n.st>>>(n.state.p, n.loss.p, n.lossHist.p);
    RG_CUDA_CHECK(cudaStreamEndCapture(n.st, &g));
    const cudaError_t ie = cudaGraphInstantiate(&n.trainGraph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess || n.mapFailed) {
      if (n.trainGraph) cudaGraphExecDestroy(n.trainGraph);
      n.trainGraph = nullptr;
      n.mapFailed = false;
      setLastError(std::string("learned denoiser: training graph: ") +
                   (ie != cudaSuccess ? cudaGetErrorString(ie) : "the driver could not encode a TMA tensor map"));
      return RG_ERR_CUDA;
    }
    n.trainKey = key;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, n.st);
  for (int s = 0; s < steps; ++s) RG_CUDA_CHECK(cudaGraphLaunch(n.trainGraph, n.st));
  cudaEventRecord(e1, n.st);
  const rg_status rs = rg::checkErr(n, "learned denoiser training");
  float ms = 0.0f;
  if (rs == RG_OK && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) n.lastStepMs = ms / steps;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rs == RG_OK && losses)
    RG_CUDA_CHECK(cudaMemcpy(losses, n.lossHist.p, sizeof(float) * steps, cudaMemcpyDeviceToHost));
  return rs;
}

rg_status rg_denoiser_timing(rg_denoiser* d, float* apply_ms, float* train_step_ms) {
  if (!d) return RG_ERR_INVALID_ARGUMENT;
  if (apply_ms) *apply_ms = d->net.lastApplyMs;
  if (train_step_ms) *train_step_ms = d->net.lastStepMs;
  return RG_OK;
}

rg_status rg_denoiser_gradients(rg_denoiser* d, int32_t count, int32_t w, int32_t h, const float* noisy_rgba,
                                const float* normal, const float* albedo, const float* depth, float spp,
                                const float* ref_rgba, float* loss, float* grad) {
  if (!d || count <= 0 || w <= 0 || h <= 0 || !noisy_rgba || !normal || !albedo || !depth || !ref_rgba || !grad ||
      !(spp >= 0.0f))
    return RG_ERR_INVALID_ARGUMENT;
  rg::KpcnNet& n = d->net;
  std::lock_guard<std::mutex> lk(n.mu);
  const size_t P = (size_t)count * w * h;
  if (!rg::ensureWork(n, P) || !rg::uploadInputs(n, P, noisy_rgba, normal, albedo, depth, spp, ref_rgba))
    return RG_ERR_OUT_OF_MEMORY;
  cudaMemsetAsync(n.loss.p, 0, sizeof(float), n.st);
  rg::forward(n, count, h, w);
  rg::k_head<true><<<(unsigned)((P + 255) / 256), 256, 0, n.st>>>(count, h, w, n.Z.p, n.noisy.p, n.ref.p, nullptr, n.gA.p,
                                                                   n.loss.p);
  rg::backward(n, count, h, w);
  const rg_status rs = rg::checkErr(n, "learned denoiser gradients");
  if (rs != RG_OK) return rs;
  RG_CUDA_CHECK(cudaMemcpy(grad, n.grad.p, sizeof(float) * rg::kNumParams, cudaMemcpyDeviceToHost));
  if (loss) RG_CUDA_CHECK(cudaMemcpy(loss, n.loss.p, sizeof(float), cudaMemcpyDeviceToHost));
  return RG_OK;
}

rg_status rg_denoiser_apply(rg_denoiser* d, int32_t w, int32_t h, const float* noisy_rgba, const float* normal,
                            const float* albedo, const float* depth, float spp, float* out_rgba) {
  if (!d || w <= 0 || h <= 0 || !noisy_rgba || !normal || !albedo || !depth || !out_rgba || !(spp >= 0.0f))
    return RG_ERR_INVALID_ARGUMENT;
  rg::KpcnNet& n = d->net;
  std::lock_guard<std::mutex> lk(n.mu);
  const size_t P = (size_t)w * h;
  if (!rg::ensureWork(n, P) || !rg::uploadInputs(n, P, noisy_rgba, normal, albedo, depth, spp, nullptr))
    return RG_ERR_OUT_OF_MEMORY;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, n.st);
  rg::forward(n, 1, h, w, n.noisy.p, n.out.p);
  cudaEventRecord(e1, n.st);
  const rg_status rs = rg::checkErr(n, "learned denoiser");
  if (rs == RG_OK) cudaEventElapsedTime(&n.lastApplyMs, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rs != RG_OK) return rs;
  RG_CUDA_CHECK(cudaMemcpy(out_rgba, n.out.p, sizeof(float4) * P, cudaMemcpyDeviceToHost));
  return RG_OK;
}

}  // extern "C"
