// rg_medium.cuh - procedural participating media on the device: the fBm
// value-noise field, procedural emission (cone, path tube), delta tracking,
// stratified emission integrals, heat-haze ray bending and equiangular
// volume-light sampling (medium.cpp:103-473, rayrenderer.cpp:2067-2203).
//
// The noise, density, emission and bending arithmetic is written with
// explicit round-to-nearest operations in the reference's evaluation order,
// so that these fields match the CPU oracle (built without contraction) bit
// for bit; expf / logf / powf / atanf / tanf are the library functions.
// Everything reads the medium through a global pointer and returns by value:
// these functions run only in the shade kernel's procedural-media variant.
#pragma once
#include "rg_device.cuh"

namespace rg {
namespace med {

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
// x*x + y*y + z*z, left to right
__device__ __forceinline__ float sq3(float x, float y, float z) { return fa(fa(fm(x, x), fm(y, y)), fm(z, z)); }
__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return fa(fa(fm(ax, bx), fm(ay, by)), fm(az, bz));
}

// Integer lattice hash -> [0, 1) (medium.cpp:127-136).
__device__ __forceinline__ float hash3(int x, int y, int z) {
  uint32_t h = (uint32_t)x * 374761393u + (uint32_t)y * 668265263u + (uint32_t)z * 2147483647u;
  h = (h ^ (h >> 13)) * 1274126177u;
  h ^= h >> 16;
  return fm((float)(h & 0x00FFFFFFu), 1.0f / 16777216.0f);
}

__device__ __forceinline__ float smooth01(float x) { return fm(fm(x, x), fs(3.0f, fm(2.0f, x))); }
__device__ __forceinline__ float lerp01(float a, float b, float t) { return fa(fm(a, fs(1.0f, t)), fm(b, t)); }

// Trilinear value noise with smoothstep weights, [0, 1] (medium.cpp:142-163).
__device__ float valueNoise(float x, float y, float z) {
  const float flx = floorf(x), fly = floorf(y), flz = floorf(z);
  const int xi = (int)flx, yi = (int)fly, zi = (int)flz;
  const float xf = smooth01(fs(x, (float)xi)), yf = smooth01(fs(y, (float)yi)), zf = smooth01(fs(z, (float)zi));
  const float x00 = lerp01(hash3(xi, yi, zi), hash3(xi + 1, yi, zi), xf);
  const float x10 = lerp01(hash3(xi, yi + 1, zi), hash3(xi + 1, yi + 1, zi), xf);
  const float x01 = lerp01(hash3(xi, yi, zi + 1), hash3(xi + 1, yi, zi + 1), xf);
  const float x11 = lerp01(hash3(xi, yi + 1, zi + 1), hash3(xi + 1, yi + 1, zi + 1), xf);
  return lerp01(lerp01(x00, x10, yf), lerp01(x01, x11, yf), zf);
}

// Normalised fractal sum over `oct` octaves of the point already shifted by
// the field's offset (fbmNormalised, medium.cpp:171-185; densityAt's loop,
// medium.cpp:276-301, is the same arithmetic).
__device__ float fbm(float x, float y, float z, float freq, int oct, float gain, float lac) {
  float fx = fm(x, freq), fy = fm(y, freq), fz = fm(z, freq);
  float amp = 1.0f, total = 0.0f, ampSum = 0.0f;
  const int n = oct > 0 ? oct : 1;
  for (int i = 0; i < n; i++) {
    total = fa(total, fm(amp, valueNoise(fx, fy, fz)));
    ampSum = fa(ampSum, amp);
    amp = fm(amp, gain);
    fx = fm(fx, lac);
    fy = fm(fy, lac);
    fz = fm(fz, lac);
  }
  return ampSum > 0.0f ? fd(total, ampSum) : 0.0f;
}

// densityAt (medium.cpp:276-301): max(0, amplitude * fbm + bias), 1 without a field.
__device__ float densityAt(const DevMedium* M, V3 p) {
  if (M->field == 0) return 1.0f;
  const float n = fbm(fs(p.x, M->nox), fs(p.y, M->noy), fs(p.z, M->noz), M->nFreq, M->nOct, M->nGain, M->nLac);
  return fmaxf(0.0f, fa(fm(M->nAmp, n), M->nBias));
}

__device__ __forceinline__ V3 scale3(V3 c, float s) { return v3(fm(c.x, s), fm(c.y, s), fm(c.z, s)); }

// emissionAt (medium.cpp:303-404): sigma_e at p for the three emission modes.
__device__ V3 emissionAt(const DevScene* S, const DevMedium* M, V3 p) {
  if (M->mode == 0) {
    const V3 base = v3(M->ser, M->seg, M->seb);
    return M->field == 0 ? base : scale3(base, densityAt(M, p));
  }
  if (M->mode == 2) {
    const int n = M->pathCount;
    if (n < 2) return v3(0, 0, 0);
    float bestD2 = __int_as_float(0x7f800000), bestT = 0.0f, bestR = 0.0f;
    for (int i = 0; i + 1 < n; i++) {
      const DevPathPoint A = S->pathPts[M->pathFirst + i], B = S->pathPts[M->pathFirst + i + 1];
      const float abx = fs(B.pr.x, A.pr.x), aby = fs(B.pr.y, A.pr.y), abz = fs(B.pr.z, A.pr.z);
      const float ab2 = sq3(abx, aby, abz);
      if (ab2 < 1e-12f) continue;
      const float apx = fs(p.x, A.pr.x), apy = fs(p.y, A.pr.y), apz = fs(p.z, A.pr.z);
      float u = fd(dot3(apx, apy, apz, abx, aby, abz), ab2);
      if (u < 0.0f) u = 0.0f;
      else if (u > 1.0f) u = 1.0f;
      const float qx = fa(A.pr.x, fm(abx, u)), qy = fa(A.pr.y, fm(aby, u)), qz = fa(A.pr.z, fm(abz, u));
      const float d2 = sq3(fs(p.x, qx), fs(p.y, qy), fs(p.z, qz));
      if (d2 < bestD2) {
        bestD2 = d2;
        bestT = fa(A.t.x, fm(fs(B.t.x, A.t.x), u));
        bestR = fa(A.pr.w, fm(fs(B.pr.w, A.pr.w), u));
      }
    }
    if (bestR <= 0.0f) return v3(0, 0, 0);
    if (bestD2 >= fm(bestR, bestR)) return v3(0, 0, 0);
    const float r = fd(__fsqrt_rn(bestD2), bestR);
    const float radial = powf(fmaxf(0.0f, fs(1.0f, r)), M->pathFalloff);
    if (radial <= 0.0f) return v3(0, 0, 0);
    const float tb = bestT < 0.0f ? 0.0f : (bestT > 1.0f ? 1.0f : bestT);
    const V3 col = v3(fa(fm(M->pir, fs(1.0f, tb)), fm(M->por, tb)), fa(fm(M->pig, fs(1.0f, tb)), fm(M->pog, tb)),
                      fa(fm(M->pib, fs(1.0f, tb)), fm(M->pob, tb)));
    float sc = fm(fm(radial, M->pathIntensity), M->densityScale);
    if (M->field != 0) sc = fm(sc, densityAt(M, p));
    return scale3(col, sc);
  }
  // cone: axial gaussian x (1 - v^2)^2 radial profile inside the bounding ellipsoid
  const float rx = fs(p.x, M->cox), ry = fs(p.y, M->coy), rz = fs(p.z, M->coz);
  const float axialT = dot3(rx, ry, rz, M->cax, M->cay, M->caz);
  if (M->coneLength <= 0.0f) return v3(0, 0, 0);
  const float u = fd(axialT, M->coneLength);
  if (u < 0.0f || u > 1.0f) return v3(0, 0, 0);
  const float px = fs(rx, fm(M->cax, axialT)), py = fs(ry, fm(M->cay, axialT)), pz = fs(rz, fm(M->caz, axialT));
  const float radial2 = sq3(px, py, pz);
  if (M->coneRadius <= 0.0f) return v3(0, 0, 0);
  const float v2 = fd(radial2, fm(M->coneRadius, M->coneRadius));
  if (v2 > 1.0f) return v3(0, 0, 0);
  const float dx = fm(fs(u, M->conePeakAxial), M->conePeakSharpness);
  const float axial = expf(-fm(dx, dx));
  const float om = fs(1.0f, v2);
  const float t = fm(axial, fm(om, om));
  if (t <= 0.0f) return v3(0, 0, 0);
  const float it = fs(1.0f, t);
  const V3 col = v3(fa(fm(M->cir, t), fm(M->cor, it)), fa(fm(M->cig, t), fm(M->cog, it)), fa(fm(M->cib, t), fm(M->cob, it)));
  float sc = fm(fm(t, M->coneIntensity), M->densityScale);
  if (M->field != 0) sc = fm(sc, densityAt(M, p));
  return scale3(col, sc);
}

// Beer-Lambert with the homogeneous sigma_t (medium.cpp:103-108).
__device__ __forceinline__ V3 transmittance(const DevMedium* M, float d) {
  if (d <= 0.0f) return v3(1, 1, 1);
  return v3(expf(-M->str * d), expf(-M->stg * d), expf(-M->stb * d));
}

__device__ __forceinline__ float emissionWeight(float st, float d) {
  return st < 1e-6f ? d : (1.0f - expf(-st * d)) / st;
}

// emissionIntegralAlongRay (medium.cpp:443-473): closed form for constant
// emission (the density field is not applied there), else one jittered
// sample per stratum of [0, maxT].
__device__ __noinline__ V3 emissionIntegral(const DevScene* S, const DevMedium* M, V3 o, V3 d, float maxT,
                                            const Rng& rng, int v) {
  if (M->mode == 0) {
    if (maxT <= 0.0f) return v3(0, 0, 0);
    return v3(M->ser * emissionWeight(M->str, maxT), M->seg * emissionWeight(M->stg, maxT),
              M->seb * emissionWeight(M->stb, maxT));
  }
  if (maxT <= 0.0f) return v3(0, 0, 0);
  const int ns = M->mode == 2 ? M->pathSamples : M->coneSamples;
  const int N = ns > 0 ? ns : 1;
  const float dt = fd(maxT, (float)N);
  V3 acc = v3(0, 0, 0);
  for (int i = 0; i < N; i++) {
    const float t = fm(fa((float)i, rng.prngk(v, S_EMIS, i)), dt);
    const V3 p = v3(fa(o.x, fm(d.x, t)), fa(o.y, fm(d.y, t)), fa(o.z, fm(d.z, t)));
    const V3 se = emissionAt(S, M, p);
    if (se.x == 0.0f && se.y == 0.0f && se.z == 0.0f) continue;
    const V3 tr = transmittance(M, t);
    acc = v3(fa(acc.x, fm(fm(se.x, tr.x), dt)), fa(acc.y, fm(fm(se.y, tr.y), dt)), fa(acc.z, fm(fm(se.z, tr.z), dt)));
  }
  return acc;
}

struct Collision {
  bool hit;
  float t, density;
};

// sampleDeltaTracking (medium.cpp:406-441): exponential steps at the majorant
// rate, each accepted as a real collision with probability density / peak;
// at most 64 steps.
__device__ __noinline__ Collision deltaTrack(const DevMedium* M, V3 o, V3 d, float maxT, const Rng& rng, int v) {
  Collision c{false, 0.0f, 1.0f};
  const float tmh = M->tMaxHero;
  if (tmh <= 0.0f || maxT <= 0.0f) return c;
  const float peak = M->hero > 0.0f ? fd(tmh, M->hero) : 1.0f;
  if (peak <= 0.0f) return c;
  float t = 0.0f;
  for (int i = 0; i < 64; i++) {
    const float xi = fminf(0.9999999f, fmaxf(0.0f, rng.prngk(v, S_DTSTEP, i)));
    t = fa(t, fd(-logf(fs(1.0f, xi)), tmh));
    if (t >= maxT) return c;
    const V3 p = v3(fa(o.x, fm(d.x, t)), fa(o.y, fm(d.y, t)), fa(o.z, fm(d.z, t)));
    const float dn = densityAt(M, p);
    const float pAccept = peak > 0.0f ? fd(dn, peak) : 1.0f;
    if (rng.prngk(v, S_DTACC, i) < pAccept) {
      c.hit = true;
      c.t = t;
      c.density = dn;
      return c;
    }
  }
  return c;
}

// iorAt (medium.cpp:186-215): 1 + amplitude * falloff * (2 fbm - 1).
__device__ float iorAt(const DevMedium* M, float x, float y, float z) {
  if (!M->hazeOn) return 1.0f;
  const float n = fbm(fs(x, M->iox), fs(y, M->ioy), fs(z, M->ioz), M->iFreq, M->iOct, M->iGain, M->iLac);
  float ampMul = 1.0f;
  if (M->iFalloff != 0.0f && M->coneLength > 0.0f) {
    const float axialT = dot3(fs(x, M->cox), fs(y, M->coy), fs(z, M->coz), M->cax, M->cay, M->caz);
    float u = fd(axialT, M->coneLength);
    if (u < 0.0f) u = 0.0f;
    else if (u > 1.0f) u = 1.0f;
    const float mag = M->iFalloff < 0.0f ? -M->iFalloff : M->iFalloff;
    const float tt = M->iFalloff >= 0.0f ? u : fs(1.0f, u);
    ampMul = fs(1.0f, fm(mag, tt));
    if (ampMul < 0.0f) ampMul = 0.0f;
  }
  return fa(1.0f, fm(fm(fm(M->iAmp, ampMul), fs(n, 0.5f)), 2.0f));
}

struct Ray6 {
  V3 o, d;
};

// bendRay (medium.cpp:237-274): midpoint-sampled eikonal steps,
// d(dir)/ds = (grad n - (grad n . dir) dir) / n, renormalised each step;
// the gradient by central differences of half a noise cell (iorGradientAt,
// medium.cpp:217-235).
__device__ __noinline__ Ray6 bendRay(const DevMedium* M, V3 o, V3 d, float length) {
  Ray6 r;
  if (length <= 0.0f || !M->haze) {
    r.o = v3(fa(o.x, fm(d.x, length)), fa(o.y, fm(d.y, length)), fa(o.z, fm(d.z, length)));
    r.d = d;
    return r;
  }
  const int N = M->iSteps;
  const float ds = fd(length, (float)N);
  const float h = M->iFreq > 0.0f ? fd(0.5f, M->iFreq) : 0.05f;
  const float inv2h = fd(0.5f, h);
  const float half = fm(ds, 0.5f);
  V3 pos = o, dir = d;
  for (int i = 0; i < N; i++) {
    const float mx = fa(pos.x, fm(dir.x, half)), my = fa(pos.y, fm(dir.y, half)), mz = fa(pos.z, fm(dir.z, half));
    const float n = iorAt(M, mx, my, mz);
    const float gx = fm(fs(iorAt(M, fa(mx, h), my, mz), iorAt(M, fs(mx, h), my, mz)), inv2h);
    const float gy = fm(fs(iorAt(M, mx, fa(my, h), mz), iorAt(M, mx, fs(my, h), mz)), inv2h);
    const float gz = fm(fs(iorAt(M, mx, my, fa(mz, h)), iorAt(M, mx, my, fs(mz, h))), inv2h);
    const float gd = dot3(gx, gy, gz, dir.x, dir.y, dir.z);
    const float px = fs(gx, fm(dir.x, gd)), py = fs(gy, fm(dir.y, gd)), pz = fs(gz, fm(dir.z, gd));
    const float invN = n > 1e-6f ? fd(1.0f, n) : 1.0f;
    const float k = fm(ds, invN);
    const float nx = fa(dir.x, fm(px, k)), ny = fa(dir.y, fm(py, k)), nz = fa(dir.z, fm(pz, k));
    const float l2 = sq3(nx, ny, nz);
    if (l2 > 1e-12f) {
      const float invL = fd(1.0f, __fsqrt_rn(l2));
      dir = v3(fm(nx, invL), fm(ny, invL), fm(nz, invL));
    }
    pos = v3(fa(pos.x, fm(dir.x, ds)), fa(pos.y, fm(dir.y, ds)), fa(pos.z, fm(dir.z, ds)));
  }
  r.o = pos;
  r.d = dir;
  return r;
}

struct VolSample {
  bool ok;
  V3 dir, Le;
  float pdf;
  V3 so, sd;  // shadow ray: SurfaceRay origin and the unnormalised direction (tmax 0.99999)
};

// sampleVolumeLightForNEE (rayrenderer.cpp:2067-2203): pick one emissive
// volume uniformly, sample a point on its cone axis (or its anchor point)
// equiangularly from `hit` (Kulla & Fajardo 2012), and return sigma_e there,
// attenuated by the volume's own homogeneous transmittance over the distance,
// with the solid-angle pdf (times the volume count).  The shadow ray is
// returned, not traced.
__device__ __noinline__ VolSample sampleVolumeLight(const DevScene* S, const Rng& rng, int v, V3 hit, V3 n) {
  VolSample out;
  out.ok = false;
  const int N = S->numVolLights;
  if (N <= 0) return out;
  const DevVolLight L = S->volLights[pickIndex(rng.prng(v, S_VOLPICK), N)];
  const DevMedium* M = S->media + L.medium;
  V3 a, b;
  if (M->mode == 1) {
    a = v3(M->cox, M->coy, M->coz);
    b = a + v3(M->cax, M->cay, M->caz) * M->coneLength;
  } else {
    a = v3(L.ax, L.ay, L.az);
    b = a;
  }
  const V3 sd = b - a;
  const float segLen = sqrtf(dot(sd, sd));
  const V3 axis = segLen > 1e-6f ? sd * (1.0f / segLen) : v3(0.0f, 0.0f, -1.0f);
  const V3 toA = a - hit;
  const float along = dot(toA, axis);
  const V3 perp = toA - axis * along;
  const float D = sqrtf(dot(perp, perp));
  if (!(D > 1e-5f) && segLen <= 1e-6f) return out;
  const float Dc = fmaxf(D, 1e-5f);
  const float thA = atanf(along / Dc), thB = atanf((along + segLen) / Dc);
  if (!(fabsf(thB - thA) > 1e-6f) && segLen > 1e-6f) return out;
  const float theta = thA + rng.prng(v, S_VOLU) * (thB - thA);
  const float tS = D * tanf(theta);
  const V3 sp = segLen > 1e-6f ? a + axis * (tS - along) : a;
  const V3 toS = sp - hit;
  const float r2 = dot(toS, toS);
  const float r = sqrtf(r2);
  if (!(r > 1e-5f)) return out;
  V3 se = emissionAt(S, M, sp);
  if (se.x == 0.0f && se.y == 0.0f && se.z == 0.0f) return out;
  if (M->hero > 0.0f) se = se * transmittance(M, r);
  const float pdfT = D / (fmaxf(1e-6f, fabsf(thB - thA)) * (D * D + tS * tS));
  out.ok = true;
  out.dir = toS * (1.0f / r);
  out.Le = se;
  out.pdf = pdfT * r2 * (float)N;
  const float side = dot(toS, n) >= 0.0f ? 1.0f : -1.0f;  // SurfaceRay, raycommon.h:82-85
  out.so = hit + n * (side * kSurfaceThickness);
  out.sd = toS;
  return out;
}

}  // namespace med
}  // namespace rg
