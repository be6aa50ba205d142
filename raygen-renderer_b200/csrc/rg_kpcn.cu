// rg_kpcn.cu - learned denoiser: a kernel-predicting CNN on the 5th-generation
// tensor cores (tcgen05, BF16 operands, FP32 accumulation in tensor memory).
//
// This part: the tensor-core GEMM building block and its stand-alone test
// entry point.  The convolution passes (forward, backward data, backward
// weights) stage their operands with their own gathers around the same block.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstring>
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
