// rg_post.cu - resolve, adaptive-sampling masks, A-Trous denoiser, HDR bloom
// and tonemap.
//
// Reference: renderPixel / hdrToPreview (rayrenderer.cpp:959-1009),
// computeTileNoise / renderAdaptive (:1038-1252), denoiseImage / atrousPass
// (:2536-2772), applyTonemapGamma (:2610-2647).  The denoiser keeps the
// reference's filter exactly (B3 5x5 taps at step 2^level, luminance /
// normal / depth edge stops, firefly pre-clamp, albedo demodulation) with
// FP32 colour and FP16 guide buffers; every pass is one kernel, one thread
// per pixel, reading its taps through the read-only cache.
#include <cuda_fp16.h>

#include <algorithm>
#include <vector>

#include "rg_device.cuh"
#include "rg_trace.cuh"

namespace rg {

namespace {

__device__ __forceinline__ float lum3(float r, float g, float b) { return 0.2126f * r + 0.7152f * g + 0.0722f * b; }

__global__ void k_resolve(int n, const float4* __restrict__ sum, const int* __restrict__ cnt, float exposure,
                          float4* __restrict__ hdr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = cnt[i];
  const float invN = c > 0 ? 1.0f / (float)c : 0.0f;
  const float4 s = sum[i];
  hdr[i] = make_float4(fmaxf(s.x * invN * exposure, 0.0f), fmaxf(s.y * invN * exposure, 0.0f),
                       fmaxf(s.z * invN * exposure, 0.0f), 1.0f);
}

// Firefly pre-clamp + albedo demodulation (rayrenderer.cpp:2685-2722).
__global__ void k_prepass(int w, int h, const float4* __restrict__ noisy, const __half* __restrict__ albedo,
                          const __half* __restrict__ albedoA, float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w * h) return;
  const int x = i % w, y = i / w;
  float4 c = noisy[i];
  float maxN = 0.0f;
  for (int dy = -1; dy <= 1; ++dy) {
    const int ny = y + dy;
    if (ny < 0 || ny >= h) continue;
    for (int dx = -1; dx <= 1; ++dx) {
      if (dx == 0 && dy == 0) continue;
      const int nx = x + dx;
      if (nx < 0 || nx >= w) continue;
      const float4 q = __ldg(&noisy[ny * w + nx]);
      const float l = lum3(q.x, q.y, q.z);
      if (l > maxN) maxN = l;
    }
  }
  const float cl = lum3(c.x, c.y, c.z);
  const float cap = 1.5f * maxN + 0.01f;
  if (cl > cap) {
    const float s = cap / cl;
    c.x *= s; c.y *= s; c.z *= s;
  }
  if (__half2float(albedoA[i]) > 0.5f) {
    const float ar = fmaxf(__half2float(albedo[i * 3]), 0.3f), ag = fmaxf(__half2float(albedo[i * 3 + 1]), 0.3f),
                ab = fmaxf(__half2float(albedo[i * 3 + 2]), 0.3f);
    out[i] = make_float4(fminf(c.x / ar, 3.0f), fminf(c.y / ag, 3.0f), fminf(c.z / ab, 3.0f), 1.0f);
  } else {
    out[i] = c;
  }
}

// One edge-avoiding A-Trous level (rayrenderer.cpp:2536-2608).
__global__ void __launch_bounds__(256) k_atrous(int w, int h, const float4* __restrict__ src, float4* __restrict__ dst,
                                                const __half* __restrict__ normal, const __half* __restrict__ depth,
                                                int step, float invC2, float sigN, float dScale) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const float kw[5] = {1.0f / 16.0f, 1.0f / 4.0f, 3.0f / 8.0f, 1.0f / 4.0f, 1.0f / 16.0f};
  const int ci = y * w + x;
  const float4 cc = src[ci];
  const float cnx = __half2float(normal[ci * 3]) * 2.0f - 1.0f, cny = __half2float(normal[ci * 3 + 1]) * 2.0f - 1.0f,
              cnz = __half2float(normal[ci * 3 + 2]) * 2.0f - 1.0f;
  const float cd = __half2float(depth[ci]);
  const float cl = lum3(cc.x, cc.y, cc.z);
  float sx = 0, sy = 0, sz = 0, ws = 0;
  for (int ky = 0; ky < 5; ++ky) {
    const int ny = y + (ky - 2) * step;
    if (ny < 0 || ny >= h) continue;
    for (int kx = 0; kx < 5; ++kx) {
      const int nx = x + (kx - 2) * step;
      if (nx < 0 || nx >= w) continue;
      const int si = ny * w + nx;
      const float4 sc = __ldg(&src[si]);
      const float snx = __half2float(normal[si * 3]) * 2.0f - 1.0f, sny = __half2float(normal[si * 3 + 1]) * 2.0f - 1.0f,
                  snz = __half2float(normal[si * 3 + 2]) * 2.0f - 1.0f;
      const float sl = lum3(sc.x, sc.y, sc.z);
      const float ld = sl - cl;
      float nd = snx * cnx + sny * cny + snz * cnz;
      if (nd < 0.0f) nd = 0.0f;
      // exp(-ld^2 / 2sc^2) * max(n.n', 0)^sigN * exp(-|dd| / (sd step)) as one
      // base-2 exponential of the summed logarithms (powf(0, 0) = 1 kept)
      const float lnC = -(ld * ld) * invC2 - fabsf(__half2float(depth[si]) - cd) * dScale;
      const float lg2N = sigN == 0.0f ? 0.0f : (nd > 0.0f ? sigN * __log2f(nd) : -INFINITY);
      const float wgt = kw[kx] * kw[ky] * exp2f(fmaf(lnC, 1.44269504088896341f, lg2N));
      sx += sc.x * wgt; sy += sc.y * wgt; sz += sc.z * wgt;
      ws += wgt;
    }
  }
  dst[ci] = ws > 1e-8f ? make_float4(sx / ws, sy / ws, sz / ws, cc.w) : cc;
}

// Remodulate and blend with the noisy input (rayrenderer.cpp:2752-2771).
__global__ void k_remod(int n, const float4* __restrict__ filtered, const float4* __restrict__ noisy,
                        const __half* __restrict__ albedo, const __half* __restrict__ albedoA, float intensity,
                        float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float t = fminf(fmaxf(intensity, 0.0f), 1.0f), s = 1.0f - t;
  const float4 f = filtered[i], nz = noisy[i];
  float4 r = f;
  if (__half2float(albedoA[i]) > 0.5f)
    r = make_float4(f.x * __half2float(albedo[i * 3]), f.y * __half2float(albedo[i * 3 + 1]),
                    f.z * __half2float(albedo[i * 3 + 2]), 1.0f);
  out[i] = make_float4(nz.x * s + r.x * t, nz.y * s + r.y * t, nz.z * s + r.z * t, 1.0f);
}

__global__ void k_tonemap(int n, const float4* __restrict__ src, float4* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 c = src[i];
  const float L = lum3(c.x, c.y, c.z);
  float mr = 0, mg = 0, mb = 0;
  if (L > 1e-6f) {
    const float sc = (L / (L + 1.0f)) / L;
    mr = c.x * sc; mg = c.y * sc; mb = c.z * sc;
    const float peak = fmaxf(fmaxf(mr, mg), mb);
    if (peak > 1.0f) {
      const float inv = 1.0f / peak;
      mr *= inv; mg *= inv; mb *= inv;
    }
  }
  const float g = 1.0f / 2.2f;
  float4 o = make_float4(powf(fmaxf(mr, 0.0f), g), powf(fmaxf(mg, 0.0f), g), powf(fmaxf(mb, 0.0f), g), c.w);
  o.x = fminf(o.x, 1.0f); o.y = fminf(o.y, 1.0f); o.z = fminf(o.z, 1.0f);
  dst[i] = o;
}

// Per-pixel relative standard error of the mean, max over channels
// (computeTileNoise, rayrenderer.cpp:1038-1087, evaluated per pixel).
__device__ __forceinline__ float relSem(const float4& s, const float4& q, int n, bool& counted) {
  counted = true;
  if (n <= 1) return 1e9f;
  const float invN = 1.0f / (float)n;
  const float mr = s.x * invN, mg = s.y * invN, mb = s.z * invN;
  if (fmaxf(fmaxf(mr, mg), mb) < 1e-3f) {
    counted = false;
    return 0.0f;
  }
  const float vr = fmaxf(0.0f, q.x * invN - mr * mr), vg = fmaxf(0.0f, q.y * invN - mg * mg),
              vb = fmaxf(0.0f, q.z * invN - mb * mb);
  const float rr = sqrtf(vr * invN) / fmaxf(mr, 1e-3f), rg_ = sqrtf(vg * invN) / fmaxf(mg, 1e-3f),
              rb = sqrtf(vb * invN) / fmaxf(mb, 1e-3f);
  return fmaxf(fmaxf(rr, rg_), rb);
}

__global__ void k_adaptivePixels(int n, const float4* __restrict__ sum, const float4* __restrict__ sumSq,
                                 const int* __restrict__ cnt, int target, float threshold, int* list, int* outCount) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool want = false;
  if (i < n && cnt[i] < target) {
    bool counted;
    const float r = relSem(sum[i], sumSq[i], cnt[i], counted);
    want = counted && r > threshold;
  }
  const unsigned act = __activemask();
  const unsigned m = __ballot_sync(act, want);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (m) {
    const int leader = __ffs(m) - 1;
    if (lane == leader) base = atomicAdd(outCount, __popc(m));
    base = __shfl_sync(act, base, leader);
  }
  if (want) list[base + __popc(m & ((1u << lane) - 1u))] = i;
}

// One block per 32x32 tile: mean relative SEM over counted pixels; active
// tiles append all their pixels (renderAdaptive tile mode, rayrenderer.cpp:1233-1251).
__global__ void k_adaptiveTiles(int w, int h, const float4* __restrict__ sum, const float4* __restrict__ sumSq,
                                const int* __restrict__ cnt, int target, float threshold, int* list, int* outCount) {
  const int tx = blockIdx.x * 32, ty = blockIdx.y * 32;
  __shared__ float acc[256];
  __shared__ int num[256];
  __shared__ int base;
  float a = 0.0f;
  int c = 0;
  int tileN = 0x7fffffff;
  for (int k = threadIdx.x; k < 1024; k += blockDim.x) {
    const int x = tx + (k & 31), y = ty + (k >> 5);
    if (x >= w || y >= h) continue;
    const int i = y * w + x;
    tileN = min(tileN, cnt[i]);
    bool counted;
    const float r = relSem(sum[i], sumSq[i], cnt[i], counted);
    if (counted) { a += r; c++; }
  }
  acc[threadIdx.x] = a;
  num[threadIdx.x] = c;
  __shared__ int minN[256];
  minN[threadIdx.x] = tileN;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      acc[threadIdx.x] += acc[threadIdx.x + s];
      num[threadIdx.x] += num[threadIdx.x + s];
      minN[threadIdx.x] = min(minN[threadIdx.x], minN[threadIdx.x + s]);
    }
    __syncthreads();
  }
  const float noise = num[0] > 0 ? acc[0] / (float)num[0] : 0.0f;
  const bool active = minN[0] < target && noise > threshold;
  if (!active) return;
  const int tw = min(32, w - tx), th = min(32, h - ty);
  if (threadIdx.x == 0) base = atomicAdd(outCount, tw * th);
  __syncthreads();
  for (int k = threadIdx.x; k < tw * th; k += blockDim.x) {
    const int x = tx + k % tw, y = ty + k / tw;
    list[base + k] = y * w + x;
  }
}

__global__ void k_h2f(int n, const __half* in, float* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __half2float(in[i]);
}
__global__ void k_f2h(int n, const float* in, __half* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2half(in[i]);
}

inline int g256(int n) { return (n + 255) / 256; }

// ---- HDR bloom (RayRenderer::applyPostProcess, rayrenderer.cpp:598-696) ------
// Every product that feeds a sum is rounded on its own (no contraction), in
// the reference's loop order, so the oracle's restatement agrees bit for bit
// (powf for a bloom curve other than 1 aside).
__device__ __forceinline__ float3 bloomExtract(float4 c, float threshold, float curve) {
  // excess luminance above the threshold (rayrenderer.cpp:614-633)
  const float L = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, c.x), __fmul_rn(0.7152f, c.y)), __fmul_rn(0.0722f, c.z));
  float3 g = make_float3(0.0f, 0.0f, 0.0f);
  if (L > threshold && L > 1e-6f) {
    float scale = __fdiv_rn(__fsub_rn(L, threshold), L);
    if (curve != 1.0f) scale = powf(scale, curve);
    g = make_float3(__fmul_rn(c.x, scale), __fmul_rn(c.y, scale), __fmul_rn(c.z, scale));
  }
  return g;
}

// extract + downsampleArea (rayrenderer.cpp:386-413): one thread per glow pixel,
// the box of full-resolution pixels it covers summed row by row.
__global__ void k_bloomDown(int W, int H, int gw, int gh, const float4* __restrict__ hdr, float threshold, float curve,
                            float4* __restrict__ small) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= gw * gh) return;
  const int x = i % gw, y = i / gw;
  const int y0 = (int)((long long)y * H / gh);
  const int y1 = max(y0 + 1, (int)((long long)(y + 1) * H / gh));
  const int x0 = (int)((long long)x * W / gw);
  const int x1 = max(x0 + 1, (int)((long long)(x + 1) * W / gw));
  float ar = 0.0f, ag = 0.0f, ab = 0.0f;
  int count = 0;
  for (int sy = y0; sy < y1 && sy < H; ++sy)
    for (int sx = x0; sx < x1 && sx < W; ++sx) {
      const float3 g = bloomExtract(__ldg(hdr + (size_t)sy * W + sx), threshold, curve);
      ar = __fadd_rn(ar, g.x);
      ag = __fadd_rn(ag, g.y);
      ab = __fadd_rn(ab, g.z);
      count++;
    }
  float4 o = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (count > 0) {
    const float inv = __fdiv_rn(1.0f, (float)count);
    o = make_float4(__fmul_rn(ar, inv), __fmul_rn(ag, inv), __fmul_rn(ab, inv), 0.0f);
  }
  small[i] = o;
}

// separableGaussianBlur, one direction (rayrenderer.cpp:423-475): clamp to edge,
// taps k = -r..r in order.
__global__ void k_bloomBlur(int w, int h, int r, const float* __restrict__ wts, int vertical,
                            const float4* __restrict__ src, float4* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= w * h) return;
  const int x = i % w, y = i / w;
  float ar = 0.0f, ag = 0.0f, ab = 0.0f;
  for (int k = -r; k <= r; ++k) {
    int sx = x, sy = y;
    if (vertical) sy = min(max(y + k, 0), h - 1);
    else sx = min(max(x + k, 0), w - 1);
    const float4 c = __ldg(src + (size_t)sy * w + sx);
    const float wk = __ldg(wts + k + r);
    ar = __fadd_rn(ar, __fmul_rn(c.x, wk));
    ag = __fadd_rn(ag, __fmul_rn(c.y, wk));
    ab = __fadd_rn(ab, __fmul_rn(c.z, wk));
  }
  dst[i] = make_float4(ar, ag, ab, 0.0f);
}

// Bilinear upsample of the glow (Image::resize; texel centres aligned, edges
// clamped) and the unclamped add hdr += glow * strength (rayrenderer.cpp:675-693).
__device__ __forceinline__ float lerpRn(float a, float b, float t) { return __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), t)); }

__global__ void k_bloomUpAdd(int W, int H, int gw, int gh, const float4* __restrict__ small, float strength,
                             float4* __restrict__ hdr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W * H) return;
  const int x = i % W, y = i / W;
  float sx = __fsub_rn(__fdiv_rn(__fmul_rn((float)x + 0.5f, (float)gw), (float)W), 0.5f);
  float sy = __fsub_rn(__fdiv_rn(__fmul_rn((float)y + 0.5f, (float)gh), (float)H), 0.5f);
  sx = fminf(fmaxf(sx, 0.0f), (float)(gw - 1));
  sy = fminf(fmaxf(sy, 0.0f), (float)(gh - 1));
  const int x0 = (int)sx, y0 = (int)sy;
  const int x1 = min(x0 + 1, gw - 1), y1 = min(y0 + 1, gh - 1);
  const float fx = __fsub_rn(sx, (float)x0), fy = __fsub_rn(sy, (float)y0);
  const float4 p00 = __ldg(small + (size_t)y0 * gw + x0), p10 = __ldg(small + (size_t)y0 * gw + x1);
  const float4 p01 = __ldg(small + (size_t)y1 * gw + x0), p11 = __ldg(small + (size_t)y1 * gw + x1);
  const float gr = lerpRn(lerpRn(p00.x, p10.x, fx), lerpRn(p01.x, p11.x, fx), fy);
  const float gg = lerpRn(lerpRn(p00.y, p10.y, fx), lerpRn(p01.y, p11.y, fx), fy);
  const float gb = lerpRn(lerpRn(p00.z, p10.z, fx), lerpRn(p01.z, p11.z, fx), fy);
  float4 a = hdr[i];
  a.x = __fadd_rn(a.x, __fmul_rn(gr, strength));
  a.y = __fadd_rn(a.y, __fmul_rn(gg, strength));
  a.z = __fadd_rn(a.z, __fmul_rn(gb, strength));
  hdr[i] = a;
}

}  // namespace

void launchResolve(int n, const float4* sum, const int* cnt, float exposure, float4* hdr, cudaStream_t st) {
  k_resolve<<<g256(n), 256, 0, st>>>(n, sum, cnt, exposure, hdr);
}

void launchDenoise(int w, int h, const float4* noisy, const __half* normal, const __half* depth, const __half* albedo,
                   const __half* albedoA, int levels, float sigC, float sigN, float sigD, float intensity,
                   float4* bufA, float4* bufB, float4* out, cudaStream_t st) {
  const int n = w * h;
  k_prepass<<<g256(n), 256, 0, st>>>(w, h, noisy, albedo, albedoA, bufA);
  float4* src = bufA;
  float4* dst = bufB;
  const float invC2 = 1.0f / (2.0f * sigC * sigC + 1e-8f);
  const dim3 blk(32, 8), grd((w + 31) / 32, (h + 7) / 8);
  for (int l = 0; l < (levels < 1 ? 1 : levels); ++l) {
    const int step = 1 << l;
    const float dScale = 1.0f / (sigD * (float)step + 1e-8f);
    k_atrous<<<grd, blk, 0, st>>>(w, h, src, dst, normal, depth, step, invC2, sigN, dScale);
    float4* t = src;
    src = dst;
    dst = t;
  }
  k_remod<<<g256(n), 256, 0, st>>>(n, src, noisy, albedo, albedoA, intensity, out);
}

void launchTonemap(int n, const float4* hdr, float4* ldr, cudaStream_t st) { k_tonemap<<<g256(n), 256, 0, st>>>(n, hdr, ldr); }

BloomPlan planBloom(int W, int H, float radius, float sizeAspect) {
  BloomPlan p;
  const float aspect = fmaxf(0.02f, sizeAspect);
  p.gw = std::max(1, (int)((float)W * aspect));
  p.gh = std::max(1, (int)((float)H * aspect));
  const float sigmaDown = fmaxf(0.0f, radius) * (float)W * aspect;
  p.r = 0;
  p.weights.clear();
  if (sigmaDown >= 0.5f) {
    // two passes of sigma / sqrt(2) (rayrenderer.cpp:660-666); kernel as separableGaussianBlur
    const float sigma = sigmaDown * 0.70710678f;
    if (sigma >= 0.25f) {
      p.r = std::max(1, (int)ceilf(sigma * 3.0f));
      const int k = 2 * p.r + 1;
      p.weights.resize(k);
      float sum = 0.0f;
      const float twoSigmaSq = 2.0f * sigma * sigma;
      for (int i = 0; i < k; ++i) {
        const float x = (float)(i - p.r);
        p.weights[i] = expf(-(x * x) / twoSigmaSq);
        sum += p.weights[i];
      }
      const float inv = 1.0f / sum;
      for (float& w : p.weights) w *= inv;
    }
  }
  return p;
}

void launchBloom(int W, int H, float4* hdr, const BloomPlan& p, const float* weightsDev, float threshold,
                 float strength, float curve, float4* smallA, float4* smallB, cudaStream_t st) {
  const int n = p.gw * p.gh;
  k_bloomDown<<<g256(n), 256, 0, st>>>(W, H, p.gw, p.gh, hdr, fmaxf(threshold, 0.0f), fmaxf(curve, 1e-3f), smallA);
  if (p.r > 0) {
    for (int pass = 0; pass < 2; ++pass) {
      k_bloomBlur<<<g256(n), 256, 0, st>>>(p.gw, p.gh, p.r, weightsDev, 0, smallA, smallB);
      k_bloomBlur<<<g256(n), 256, 0, st>>>(p.gw, p.gh, p.r, weightsDev, 1, smallB, smallA);
    }
  }
  k_bloomUpAdd<<<g256(W * H), 256, 0, st>>>(W, H, p.gw, p.gh, smallA, strength, hdr);
}

void launchAdaptivePixels(int n, const float4* sum, const float4* sumSq, const int* cnt, int target, float threshold,
                          int* list, int* outCount, cudaStream_t st) {
  k_adaptivePixels<<<g256(n), 256, 0, st>>>(n, sum, sumSq, cnt, target, threshold, list, outCount);
}

void launchAdaptiveTiles(int w, int h, const float4* sum, const float4* sumSq, const int* cnt, int target,
                         float threshold, int* list, int* outCount, cudaStream_t st) {
  const dim3 grd((w + 31) / 32, (h + 31) / 32);
  k_adaptiveTiles<<<grd, 256, 0, st>>>(w, h, sum, sumSq, cnt, target, threshold, list, outCount);
}

void launchHalfToFloat(int n, const __half* in, float* out, cudaStream_t st) { k_h2f<<<g256(n), 256, 0, st>>>(n, in, out); }
void launchFloatToHalf(int n, const float* in, __half* out, cudaStream_t st) { k_f2h<<<g256(n), 256, 0, st>>>(n, in, out); }

}  // namespace rg
