// rg_traverse.cuh - closest-hit and any-hit traversal of the device BVH.
//
// Node layout (64 B, one node holds the boxes of both children so a single
// fetch tests two boxes):
//   n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   n3 = (ref0, ref1, -, -)  ref >= 0: inner node, ref < 0: ~((first << 3) | (count - 1))
// Triangles (48 B, leaf order): (v1, mesh) (e1 = v2 - v1, occluder bits) (e2 = v3 - v1, -).
//
// The box test is the reference slab test (bvh.cpp:250-265) including its
// reciprocal guard; the triangle tests are Moller-Trumbore exactly as
// raycommon.cpp:151-235, evaluated without FMA contraction so hit ids, t,
// u and v are bit-identical to the CPU restatement when both find the same
// candidate.
#pragma once
#include "rg_device.cuh"

namespace rg {

// Traversal step bound read by every traversal loop (node steps per ray);
// kMaxTraversalSteps unless a test lowers it through
// rg_debug_set_traversal_step_cap to make the bound fire on a small scene.
__constant__ int c_traversalStepCap = kMaxTraversalSteps;

__device__ __forceinline__ float4 ldg4(const float4* p) { return __ldg(p); }
// BVH node and triangle fetches of the 8-wide traversal
__device__ __forceinline__ float4 ldNode4(const float4* p) { return __ldg(p); }
__device__ __forceinline__ float4 ldTri4(const float4* p) { return __ldg(p); }

__device__ __forceinline__ V3 safeInv(V3 d) {
  return v3(fabsf(d.x) > 1e-20f ? 1.0f / d.x : 1e30f, fabsf(d.y) > 1e-20f ? 1.0f / d.y : 1e30f,
            fabsf(d.z) > 1e-20f ? 1.0f / d.z : 1e30f);
}

// Slab test of both children. Returns a 2-bit mask and the entry distances.
__device__ __forceinline__ int boxPair(const float4 n0, const float4 n1, const float4 n2, V3 inv, V3 oi, float tcap,
                                       float& t0, float& t1) {
  const float a0 = fmaf(n0.x, inv.x, -oi.x), a1 = fmaf(n0.y, inv.x, -oi.x);
  const float b0 = fmaf(n0.z, inv.y, -oi.y), b1 = fmaf(n0.w, inv.y, -oi.y);
  const float c0 = fmaf(n2.x, inv.z, -oi.z), c1 = fmaf(n2.y, inv.z, -oi.z);
  const float tmin0 = fmaxf(fmaxf(fminf(a0, a1), fminf(b0, b1)), fminf(c0, c1));
  const float tmax0 = fminf(fminf(fmaxf(a0, a1), fmaxf(b0, b1)), fmaxf(c0, c1));
  const float d0 = fmaf(n1.x, inv.x, -oi.x), d1 = fmaf(n1.y, inv.x, -oi.x);
  const float e0 = fmaf(n1.z, inv.y, -oi.y), e1 = fmaf(n1.w, inv.y, -oi.y);
  const float f0 = fmaf(n2.z, inv.z, -oi.z), f1 = fmaf(n2.w, inv.z, -oi.z);
  const float tmin1 = fmaxf(fmaxf(fminf(d0, d1), fminf(e0, e1)), fminf(f0, f1));
  const float tmax1 = fminf(fminf(fmaxf(d0, d1), fmaxf(e0, e1)), fmaxf(f0, f1));
  t0 = tmin0;
  t1 = tmin1;
  const bool h0 = !(tmax0 < 0.0f || tmin0 > tmax0 || tmin0 > tcap);
  const bool h1 = !(tmax1 < 0.0f || tmin1 > tmax1 || tmin1 > tcap);
  return (h0 ? 1 : 0) | (h1 ? 2 : 0);
}

struct ClosestHit {
  float t, u, v;
  int prim;
};

// RenderMeshTriangle::intersectsRay(ray, info): raycommon.cpp:200-235
// (dot / cross in the fixed FMA form of dot_f / cross_f, as in the oracle)
__device__ __forceinline__ bool mtClosest(V3 o, V3 d, V3 p1, V3 e1, V3 e2, ClosestHit& h) {
  const V3 pvec = cross_f(d, e2);
  const float det = dot_f(e1, pvec);
  if (fabsf(det) < 1e-8f) return false;
  const float invDet = __frcp_rn(det);  // the correctly rounded 1 / det, as 1.0f / det
  const V3 tvec = sub_rn(o, p1);
  const float u = __fmul_rn(dot_f(tvec, pvec), invDet);
  if (u < 0.0f || u > 1.0f) return false;
  const V3 qvec = cross_f(tvec, e1);
  const float v = __fmul_rn(dot_f(d, qvec), invDet);
  if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
  const float t = __fmul_rn(dot_f(e2, qvec), invDet);
  if (t < 0.0f) return false;
  if (t >= h.t) return false;
  h.t = t;
  h.u = u;
  h.v = v;
  return true;
}

// RenderMeshTriangle::intersectsRay(ray, maxt, t, hit): raycommon.cpp:151-198
__device__ __forceinline__ bool mtAny(V3 o, V3 d, V3 p1, V3 e1, V3 e2, float maxt) {
  const V3 h = cross_f(d, e2);
  const float a = dot_f(e1, h);
  if (fabsf(a) < 1e-6f) return false;
  const float f = __frcp_rn(a);  // the correctly rounded 1 / a, as 1.0f / a
  const V3 s = sub_rn(o, p1);
  const float u = __fmul_rn(f, dot_f(s, h));
  if (u < 0.0f || u > 1.0f) return false;
  const V3 q = cross_f(s, e1);
  const float v = __fmul_rn(f, dot_f(d, q));
  if (v < 0.0f || __fadd_rn(u, v) > 1.0f) return false;
  const float t = __fmul_rn(f, dot_f(e2, q));
  return t > 1e-6f && t < maxt;
}

// Closest hit (TriangleBVH::intersectClosest, bvh.cpp:233-285). Near child
// first by entry distance. Returns the leaf-order primitive or -1.
__device__ __forceinline__ ClosestHit traceClosest2(const DevScene& S, V3 o, V3 d, uint32_t& nodeCount,
                                                    uint32_t& triCount) {
  ClosestHit h;
  h.t = kMaxRayDistance;
  h.u = h.v = 0.0f;
  h.prim = -1;
  const V3 inv = safeInv(d);
  const V3 oi = v3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
  int stack[kStackSize];
  int sp = 0;
  int ref = S.rootIsLeaf ? S.rootLeafRef : 0;
  if (S.numTris == 0) return h;
  int steps = 0;
  for (;;) {
    while (ref >= 0) {
      if (++steps > c_traversalStepCap || ref >= S.numNodes) {
        atomicCAS(S.error, 0, kErrTraversalSteps);
        return h;
      }
      const float4* np = S.nodes + (size_t)ref * 4;
      const float4 n0 = ldg4(np), n1 = ldg4(np + 1), n2 = ldg4(np + 2), n3 = ldg4(np + 3);
      nodeCount++;
      float t0, t1;
      const int m = boxPair(n0, n1, n2, inv, oi, h.t, t0, t1);
      const int r0 = __float_as_int(n3.x), r1 = __float_as_int(n3.y);
      if (m == 0) {
        ref = sp > 0 ? stack[--sp] : INT_MAX;
        if (ref == INT_MAX) break;
      } else if (m == 3) {
        const bool near0 = t0 <= t1;
        if (sp < kStackSize) stack[sp++] = near0 ? r1 : r0;
        else atomicCAS(S.error, 0, kErrStackOverflow);
        ref = near0 ? r0 : r1;
      } else {
        ref = (m == 1) ? r0 : r1;
      }
    }
    if (ref == INT_MAX) break;
    // leaf
    const int enc = ~ref;
    const int first = enc >> 3, cnt = (enc & 7) + 1;
    if (first + cnt > S.numTris) {
      atomicCAS(S.error, 0, kErrLeafRange);
      return h;
    }
    for (int i = first; i < first + cnt; i++) {
      const float4* tp = S.triVerts + (size_t)i * 3;
      const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
      triCount++;
      if (mtClosest(o, d, xyz(a), xyz(b), xyz(c), h)) h.prim = i;
    }
    if (sp == 0) break;
    ref = stack[--sp];
  }
  return h;
}

// Any hit with an occluder-class predicate (TriangleBVH::intersectAny, bvh.h:63-101).
__device__ __forceinline__ bool traceAny2(const DevScene& S, V3 o, V3 d, float maxT, uint32_t occMask,
                                          uint32_t& nodeCount, uint32_t& triCount) {
  if (S.numTris == 0) return false;
  const V3 inv = safeInv(d);
  const V3 oi = v3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
  int stack[kStackSize];
  int sp = 0;
  int ref = S.rootIsLeaf ? S.rootLeafRef : 0;
  int steps = 0;
  for (;;) {
    while (ref >= 0) {
      if (++steps > c_traversalStepCap || ref >= S.numNodes) {
        atomicCAS(S.error, 0, kErrTraversalSteps);
        return false;
      }
      const float4* np = S.nodes + (size_t)ref * 4;
      const float4 n0 = ldg4(np), n1 = ldg4(np + 1), n2 = ldg4(np + 2), n3 = ldg4(np + 3);
      nodeCount++;
      float t0, t1;
      const int m = boxPair(n0, n1, n2, inv, oi, maxT, t0, t1);
      const int r0 = __float_as_int(n3.x), r1 = __float_as_int(n3.y);
      if (m == 0) {
        ref = sp > 0 ? stack[--sp] : INT_MAX;
        if (ref == INT_MAX) break;
      } else if (m == 3) {
        if (sp < kStackSize) stack[sp++] = r1;
        else atomicCAS(S.error, 0, kErrStackOverflow);
        ref = r0;
      } else {
        ref = (m == 1) ? r0 : r1;
      }
    }
    if (ref == INT_MAX) break;
    const int enc = ~ref;
    const int first = enc >> 3, cnt = (enc & 7) + 1;
    if (first + cnt > S.numTris) {
      atomicCAS(S.error, 0, kErrLeafRange);
      return false;
    }
    for (int i = first; i < first + cnt; i++) {
      const float4* tp = S.triVerts + (size_t)i * 3;
      const float4 b = ldg4(tp + 1);
      if (!(__float_as_uint(b.w) & occMask)) continue;
      const float4 a = ldg4(tp), c = ldg4(tp + 2);
      triCount++;
      if (mtAny(o, d, xyz(a), xyz(b), xyz(c), maxT)) return true;
    }
    if (sp == 0) break;
    ref = stack[--sp];
  }
  return false;
}

// ---- 8-wide BVH ---------------------------------------------------------------
// Node layout: see k_collapse (rg_bvh.cu).  Traversal keeps a "node group"
// (child base, hit bits, inner-slot mask) and a "triangle group" (triangle base,
// 32-bit mask); hit inner children are visited in descending order of
// (slot XOR ray octant), an approximate front-to-back order.

struct Node8Hit {
  uint32_t inner;    // hit inner children, bit (slot ^ octant)
  uint32_t tris;     // triangle mask relative to triBase
  uint32_t imask;
  int childBase, triBase;
};

// Three-input minimum / maximum: one instruction each on sm_100 (PTX ISA 8.8).
__device__ __forceinline__ float fmax3f(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
__device__ __forceinline__ float fmin3f(float a, float b, float c) {
  float d;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}

// Bit 7 of each byte of w -> 4 bits (byte k -> bit k).
__device__ __forceinline__ uint32_t byteTopBits(uint32_t w) {
  return (((w >> 7) & 0x01010101u) * 0x01020408u) >> 24;
}

__device__ __forceinline__ Node8Hit intersectNode8(const float4* np, V3 o, V3 inv, float tcap, uint32_t oct) {
  const float4 h = ldNode4(np);
  Node8Hit r;
  r.childBase = __float_as_int(h.x);
  r.triBase = __float_as_int(h.y);
  const uint32_t m0 = __float_as_uint(h.z), m1 = __float_as_uint(h.w);
  r.imask = byteTopBits(m0) | (byteTopBits(m1) << 4);  // meta 0x80: inner child
  r.inner = 0;
  r.tris = 0;
  const V3 oi = v3(o.x * inv.x, o.y * inv.y, o.z * inv.z);
  // near / far plane arrays per axis from the ray direction signs (inv < 0: the hi planes are near)
  const int fx = (int)(oct & 1u), fy = (int)((oct >> 1) & 1u), fz = (int)((oct >> 2) & 1u);
  const float4 *nx = np + 1 + 2 * fx, *fxp = np + 3 - 2 * fx;
  const float4 *ny = np + 5 + 2 * fy, *fyp = np + 7 - 2 * fy;
  const float4 *nz = np + 9 + 2 * fz, *fzp = np + 11 - 2 * fz;
  uint32_t hits = 0;
#pragma unroll
  for (int half = 0; half < 2; half++) {
    const float4 a = ldNode4(nx + half), b = ldNode4(fxp + half), c = ldNode4(ny + half), d = ldNode4(fyp + half),
                 e = ldNode4(nz + half), f = ldNode4(fzp + half);
    const float pa[4] = {a.x, a.y, a.z, a.w}, pb[4] = {b.x, b.y, b.z, b.w}, pc[4] = {c.x, c.y, c.z, c.w},
                pd[4] = {d.x, d.y, d.z, d.w}, pe[4] = {e.x, e.y, e.z, e.w}, pf[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      // slab test (bvh.cpp:250-265): the interval [max(tnear, 0), min(tfar, tcap)] is not empty
      const float tmin = fmax3f(fmaf(pa[j], inv.x, -oi.x), fmaf(pc[j], inv.y, -oi.y), fmaf(pe[j], inv.z, -oi.z));
      const float tmax = fmin3f(fmaf(pb[j], inv.x, -oi.x), fmaf(pd[j], inv.y, -oi.y), fmaf(pf[j], inv.z, -oi.z));
      if (fmaxf(tmin, 0.0f) <= fminf(tmax, tcap)) hits |= 1u << (4 * half + j);
    }
  }
  // inner children: bit (slot ^ octant)
  uint32_t x = hits & r.imask;
  if (oct & 1u) x = ((x & 0x55u) << 1) | ((x >> 1) & 0x55u);
  if (oct & 2u) x = ((x & 0x33u) << 2) | ((x >> 2) & 0x33u);
  if (oct & 4u) x = ((x & 0x0fu) << 4) | ((x >> 4) & 0x0fu);
  r.inner = x;
  // leaf children: their triangle ranges
  const unsigned long long meta64 = ((unsigned long long)m1 << 32) | m0;
  for (uint32_t leaf = hits & ~r.imask; leaf; leaf &= leaf - 1u) {
    const uint32_t m = (uint32_t)(meta64 >> (8 * (__ffs(leaf) - 1))) & 0xffu;
    r.tris |= ((2u << (m >> 5)) - 1u) << (m & 31u);
  }
  return r;
}

// Octant from the guarded reciprocal (not from d): a tiny negative component
// has a positive reciprocal (1e30), and the near/far plane choice must follow it.
__device__ __forceinline__ uint32_t rayOctant(V3 inv) {
  return (inv.x < 0.0f ? 1u : 0u) | (inv.y < 0.0f ? 2u : 0u) | (inv.z < 0.0f ? 4u : 0u);
}

constexpr int kStack8 = 32;

__device__ __forceinline__ ClosestHit traceClosest8(const DevScene& S, V3 o, V3 d, uint32_t& nodeCount,
                                                    uint32_t& triCount) {
  ClosestHit h;
  h.t = kMaxRayDistance;
  h.u = h.v = 0.0f;
  h.prim = -1;
  if (S.numTris == 0) return h;
  const V3 inv = safeInv(d);
  const uint32_t oct = rayOctant(inv);
  uint2 stack[kStack8];
  int sp = 0;
  Node8Hit g = intersectNode8(S.nodes8, o, inv, h.t, oct);
  nodeCount++;
  uint32_t gInner = g.inner, gImask = g.imask, tMask = g.tris;
  int gBase = g.childBase, tBase = g.triBase;
  int steps = 0;
  for (;;) {
    while (tMask) {
      const int i = __ffs(tMask) - 1;
      tMask &= tMask - 1u;
      const int k = tBase + i;
      const float4* tp = S.triVerts + (size_t)k * 3;
      const float4 a = ldg4(tp), b = ldg4(tp + 1), c = ldg4(tp + 2);
      triCount++;
      if (mtClosest(o, d, xyz(a), xyz(b), xyz(c), h)) h.prim = k;
    }
    if (gInner == 0) {
      if (sp == 0) break;
      const uint2 e = stack[--sp];
      gBase = (int)e.x;
      gInner = e.y & 0xffu;
      gImask = e.y >> 8;
      continue;
    }
    if (++steps > c_traversalStepCap) {
      atomicCAS(S.error, 0, kErrTraversalSteps);
      break;
    }
    const int pos = 31 - __clz(gInner);
    gInner &= ~(1u << pos);
    const int slot = pos ^ (int)oct;
    const int node = gBase + __popc(gImask & ((1u << slot) - 1u));
    if (gInner) {
      if (sp < kStack8) stack[sp++] = make_uint2((uint32_t)gBase, gInner | (gImask << 8));
      else atomicCAS(S.error, 0, kErrStackOverflow);
    }
    if (node >= S.numNodes8) {
      atomicCAS(S.error, 0, kErrTraversalSteps);
      break;
    }
    g = intersectNode8(S.nodes8 + (size_t)node * kNode8Vec, o, inv, h.t, oct);
    nodeCount++;
    gInner = g.inner;
    gImask = g.imask;
    gBase = g.childBase;
    tMask = g.tris;
    tBase = g.triBase;
  }
  return h;
}

__device__ __forceinline__ bool traceAny8(const DevScene& S, V3 o, V3 d, float maxT, uint32_t occMask,
                                          uint32_t& nodeCount, uint32_t& triCount) {
  if (S.numTris == 0) return false;
  const V3 inv = safeInv(d);
  const uint32_t oct = rayOctant(inv);
  uint2 stack[kStack8];
  int sp = 0;
  Node8Hit g = intersectNode8(S.nodes8, o, inv, maxT, oct);
  nodeCount++;
  uint32_t gInner = g.inner, gImask = g.imask, tMask = g.tris;
  int gBase = g.childBase, tBase = g.triBase;
  int steps = 0;
  for (;;) {
    while (tMask) {
      const int i = __ffs(tMask) - 1;
      tMask &= tMask - 1u;
      const int k = tBase + i;
      const float4* tp = S.triVerts + (size_t)k * 3;
      const float4 b = ldg4(tp + 1);
      if (!(__float_as_uint(b.w) & occMask)) continue;
      const float4 a = ldg4(tp), c = ldg4(tp + 2);
      triCount++;
      if (mtAny(o, d, xyz(a), xyz(b), xyz(c), maxT)) return true;
    }
    if (gInner == 0) {
      if (sp == 0) break;
      const uint2 e = stack[--sp];
      gBase = (int)e.x;
      gInner = e.y & 0xffu;
      gImask = e.y >> 8;
      continue;
    }
    if (++steps > c_traversalStepCap) {
      atomicCAS(S.error, 0, kErrTraversalSteps);
      break;
    }
    const int pos = 31 - __clz(gInner);
    gInner &= ~(1u << pos);
    const int slot = pos ^ (int)oct;
    const int node = gBase + __popc(gImask & ((1u << slot) - 1u));
    if (gInner) {
      if (sp < kStack8) stack[sp++] = make_uint2((uint32_t)gBase, gInner | (gImask << 8));
      else atomicCAS(S.error, 0, kErrStackOverflow);
    }
    if (node >= S.numNodes8) {
      atomicCAS(S.error, 0, kErrTraversalSteps);
      break;
    }
    g = intersectNode8(S.nodes8 + (size_t)node * kNode8Vec, o, inv, maxT, oct);
    nodeCount++;
    gInner = g.inner;
    gImask = g.imask;
    gBase = g.childBase;
    tMask = g.tris;
    tBase = g.triBase;
  }
  return false;
}

__device__ __forceinline__ ClosestHit traceClosest(const DevScene& S, V3 o, V3 d, uint32_t& nodeCount,
                                                   uint32_t& triCount) {
  if (S.bvhWidth == 8) return traceClosest8(S, o, d, nodeCount, triCount);
  return traceClosest2(S, o, d, nodeCount, triCount);
}

__device__ __forceinline__ bool traceAny(const DevScene& S, V3 o, V3 d, float maxT, uint32_t occMask,
                                         uint32_t& nodeCount, uint32_t& triCount) {
  if (S.bvhWidth == 8) return traceAny8(S, o, d, maxT, occMask, nodeCount, triCount);
  return traceAny2(S, o, d, maxT, occMask, nodeCount, triCount);
}

}  // namespace rg
