// rg_bvh.cu - scene preparation and binned-SAH BVH build on the device.
//
// Reference: RayRenderer::transformScene / transformObject
// (rayrenderer.cpp:157-363), RenderMeshTriangle::precalc (raycommon.cpp:128-149)
// and TriangleBVH::build / buildRecursive (bvh.cpp:76-231).
//
// The reference builds top-down and recursively on one CPU thread: widest
// centroid axis, 16 bins, leaf <= 4, cost 1 + 1.5 (A_L N_L + A_R N_R)/A_P
// against 1.5 N.  Here the same split rule (bin count a parameter, 32 by
// default) runs breadth-first: every level bins all open nodes at once
// (shared-memory bins for blocks inside one node, global atomics across
// nodes), picks splits one thread per node, and scatters primitives with
// warp-aggregated atomics.  Leaves hold at most kMaxLeaf (8) triangles:
// where the reference would keep a larger leaf, the best SAH bin (or, for
// coincident centroids, an index median) splits it further.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cub/device/device_scan.cuh>

#include <cfloat>
#include <vector>

#include "rg_device.cuh"
#include "rg_host.h"

namespace rg {

namespace {

__device__ __forceinline__ uint32_t fenc(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fdec(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

struct BNode {
  float bmin[3], bmax[3];
  float cmin[3], cmax[3];
  int start, count;
  int left;      // first child (right = left + 1), -1 for leaves
  int axis;
  int binSlot;   // slot in the level's bin array while open
  int splitBin;  // bins <= splitBin go left; -2 = index median split
};

struct BinData {  // ordered-uint encoded bounds, 16 words
  uint32_t bmin[3], bmax[3], cmin[3], cmax[3];
  uint32_t count;
  uint32_t pad[3];
};

// ---- triangle preparation -------------------------------------------------
// World -> view (camera translation; angles handled on the host by rotating
// the input), edges, geometric normal, bounds, occluder bits.
__global__ void k_prepTriangles(int n, const float* __restrict__ pos, const float* __restrict__ nrm,
                                const float* __restrict__ uv, const int* __restrict__ triMesh,
                                const int* __restrict__ meshObj, const int* __restrict__ objMat,
                                const DevMaterial* __restrict__ mats, const float* __restrict__ view,
                                float4* __restrict__ verts, float4* __restrict__ shade, float2* __restrict__ uvOut,
                                float4* __restrict__ bmin, float4* __restrict__ bmax) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* p = pos + (size_t)i * 9;
  const float* q = nrm + (size_t)i * 9;
  V3 v[3], nn[3];
  for (int k = 0; k < 3; k++) {
    const V3 w = v3(p[k * 3], p[k * 3 + 1], p[k * 3 + 2]);
    // p_view = [p 1] * M (row vector, M row-major 4x4), non-contracted
    v[k].x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w.x, view[0]), __fmul_rn(w.y, view[4])), __fmul_rn(w.z, view[8])), view[12]);
    v[k].y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w.x, view[1]), __fmul_rn(w.y, view[5])), __fmul_rn(w.z, view[9])), view[13]);
    v[k].z = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(w.x, view[2]), __fmul_rn(w.y, view[6])), __fmul_rn(w.z, view[10])), view[14]);
    const V3 m = v3(q[k * 3], q[k * 3 + 1], q[k * 3 + 2]);
    // normals: [n 0] * inverse-transpose(M); M is rigid here, so its 3x3 block
    V3 r;
    r.x = __fadd_rn(__fadd_rn(__fmul_rn(m.x, view[0]), __fmul_rn(m.y, view[4])), __fmul_rn(m.z, view[8]));
    r.y = __fadd_rn(__fadd_rn(__fmul_rn(m.x, view[1]), __fmul_rn(m.y, view[5])), __fmul_rn(m.z, view[9]));
    r.z = __fadd_rn(__fadd_rn(__fmul_rn(m.x, view[2]), __fmul_rn(m.y, view[6])), __fmul_rn(m.z, view[10]));
    const float l = __fsqrt_rn(dot_rn(r, r));
    nn[k] = l > 0.0f ? v3(__fdiv_rn(r.x, l), __fdiv_rn(r.y, l), __fdiv_rn(r.z, l)) : r;
  }
  const V3 e1 = sub_rn(v[1], v[0]), e2 = sub_rn(v[2], v[0]);
  const V3 pd = cross_rn(sub_rn(v[1], v[0]), sub_rn(v[2], v[1]));
  const float pl = __fsqrt_rn(dot_rn(pd, pd));
  const V3 gn = pl > 0.0f ? v3(__fdiv_rn(pd.x, pl), __fdiv_rn(pd.y, pl), __fdiv_rn(pd.z, pl)) : pd;
  const int mesh = triMesh[i];
  const DevMaterial mt = mats[objMat[meshObj[mesh]]];
  uint32_t occ = kOccAll;
  if (mt.transparency < 0.01f && mt.emission <= 0.0f) occ |= kOccArea;
  if (mt.emission <= 0.0f && (mt.transparency < 0.01f || mt.refraction > 0.1f)) occ |= kOccPoint;
  if (mt.transparency < 0.01f) occ |= kOccAO;
  if (mt.emission <= 0.0f && mt.transparency < 0.01f && mt.refraction <= 0.1f) occ |= kOccVol;
  verts[(size_t)i * 3 + 0] = make_float4(v[0].x, v[0].y, v[0].z, __int_as_float(mesh));
  verts[(size_t)i * 3 + 1] = make_float4(e1.x, e1.y, e1.z, __uint_as_float(occ));
  verts[(size_t)i * 3 + 2] = make_float4(e2.x, e2.y, e2.z, 0.0f);
  shade[(size_t)i * 3 + 0] = make_float4(nn[0].x, nn[0].y, nn[0].z, nn[1].x);
  shade[(size_t)i * 3 + 1] = make_float4(nn[1].y, nn[1].z, nn[2].x, nn[2].y);
  shade[(size_t)i * 3 + 2] = make_float4(nn[2].z, gn.x, gn.y, gn.z);
  if (uvOut) {
    for (int k = 0; k < 3; k++) uvOut[(size_t)i * 3 + k] = uv ? make_float2(uv[(size_t)i * 6 + k * 2], uv[(size_t)i * 6 + k * 2 + 1]) : make_float2(0, 0);
  }
  const V3 lo = v3(fminf(v[0].x, fminf(v[1].x, v[2].x)), fminf(v[0].y, fminf(v[1].y, v[2].y)), fminf(v[0].z, fminf(v[1].z, v[2].z)));
  const V3 hi = v3(fmaxf(v[0].x, fmaxf(v[1].x, v[2].x)), fmaxf(v[0].y, fmaxf(v[1].y, v[2].y)), fmaxf(v[0].z, fmaxf(v[1].z, v[2].z)));
  bmin[i] = make_float4(lo.x, lo.y, lo.z, 0.0f);
  bmax[i] = make_float4(hi.x, hi.y, hi.z, 0.0f);
}

// ---- root bounds -------------------------------------------------------------
__global__ void k_rootBounds(int n, const float4* __restrict__ bmin, const float4* __restrict__ bmax, uint32_t* out) {
  // out: bmin[3] bmax[3] cmin[3] cmax[3] (encoded)
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 a = bmin[i], b = bmax[i];
    const float av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    for (int k = 0; k < 3; k++) {
      lo[k] = fminf(lo[k], av[k]);
      hi[k] = fmaxf(hi[k], bv[k]);
      const float c = (av[k] + bv[k]) * 0.5f;
      clo[k] = fminf(clo[k], c);
      chi[k] = fmaxf(chi[k], c);
    }
  }
  for (int k = 0; k < 3; k++) {
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
      clo[k] = fminf(clo[k], __shfl_xor_sync(0xffffffffu, clo[k], o));
      chi[k] = fmaxf(chi[k], __shfl_xor_sync(0xffffffffu, chi[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int k = 0; k < 3; k++) {
      atomicMin(&out[k], fenc(lo[k]));
      atomicMax(&out[3 + k], fenc(hi[k]));
      atomicMin(&out[6 + k], fenc(clo[k]));
      atomicMax(&out[9 + k], fenc(chi[k]));
    }
  }
}

__global__ void k_initRoot(int n, const uint32_t* rb, BNode* nodes, int* primIdx, int* primNode, int rootOpen) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) {
    BNode r;
    for (int k = 0; k < 3; k++) {
      r.bmin[k] = fdec(rb[k]); r.bmax[k] = fdec(rb[3 + k]);
      r.cmin[k] = fdec(rb[6 + k]); r.cmax[k] = fdec(rb[9 + k]);
    }
    r.start = 0; r.count = n; r.left = -1; r.axis = 0; r.binSlot = 0; r.splitBin = -1;
    nodes[0] = r;
  }
  if (i < n) {
    primIdx[i] = i;
    primNode[i] = rootOpen ? 0 : -1;
  }
}

// Prepare open nodes of a level: pick the widest centroid axis (bvh.cpp:125-131).
__global__ void k_prepareLevel(int numTasks, const int* tasks, BNode* nodes, BinData* bins, int nbins, bool resetBins) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < numTasks) {
    BNode& nd = nodes[tasks[t]];
    const float ex = nd.cmax[0] - nd.cmin[0], ey = nd.cmax[1] - nd.cmin[1], ez = nd.cmax[2] - nd.cmin[2];
    int axis = 0;
    if (ey > ex) axis = 1;
    if (ez > ((axis == 0) ? ex : ey)) axis = 2;
    nd.axis = axis;
    nd.binSlot = t;
  }
  // reset bins (one thread per bin) unless the split kernel leaves them reset
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (resetBins && b < numTasks * nbins) {
    BinData z;
    for (int k = 0; k < 3; k++) {
      z.bmin[k] = 0xFFFFFFFFu; z.bmax[k] = 0u; z.cmin[k] = 0xFFFFFFFFu; z.cmax[k] = 0u;
    }
    z.count = 0; z.pad[0] = z.pad[1] = z.pad[2] = 0;
    bins[b] = z;
  }
}

__device__ __forceinline__ int binOf(const BNode& nd, float c, int nbins) {
  const float cmin = nd.cmin[nd.axis];
  const float ext = nd.cmax[nd.axis] - cmin;
  const float scale = (float)nbins / ext;
  int b = (int)((c - cmin) * scale);
  if (b < 0) b = 0;
  if (b >= nbins) b = nbins - 1;
  return b;
}

__device__ __forceinline__ float axisOf(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Primitives binned per block (build-time overridable (-D) for sweeps).
#ifndef RG_BIN_CHUNK
#define RG_BIN_CHUNK 1024  // swept: 1024 / 2048 / 4096 / 16384 -> 12.5 / 13.0 / 13.9 / 19.4 ms (4M triangles)
#endif
constexpr int kBinChunk = RG_BIN_CHUNK;
// Largest leaf of the 8-wide BVH (<= 4: a node's leaves address at most 32 triangles
// through its 32-bit triangle mask); build-time overridable (-D) for sweeps.
#ifndef RG_WIDE_MAX_LEAF
#define RG_WIDE_MAX_LEAF 4
#endif
constexpr int kWideMaxLeaf = RG_WIDE_MAX_LEAF;
static_assert(kWideMaxLeaf >= 1 && kWideMaxLeaf <= 4, "8 leaves of at most 4 triangles fill the 32-bit mask");
constexpr int kMaxBins = 64;

// bmin / bmax are in the current primitive order (they move with primIdx in
// k_partition), so the passes over the primitives read them coalesced.
__global__ void __launch_bounds__(256) k_bin(int n, const int* __restrict__ primNode, const BNode* __restrict__ nodes,
                                             const float4* __restrict__ bmin, const float4* __restrict__ bmax,
                                             BinData* bins, int nbins) {
  __shared__ uint32_t sb[kMaxBins][13];
  const int first = blockIdx.x * kBinChunk;
  if (first >= n) return;
  const int last = min(n, first + kBinChunk) - 1;
  const int nodeA = primNode[first], nodeB = primNode[last];
  const bool uniform = (nodeA == nodeB) && nodeA >= 0;
  if (uniform) {
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
      for (int k = 0; k < 3; k++) {
        sb[b][k] = 0xFFFFFFFFu; sb[b][3 + k] = 0u; sb[b][6 + k] = 0xFFFFFFFFu; sb[b][9 + k] = 0u;
      }
      sb[b][12] = 0;
    }
    __syncthreads();
    const BNode nd = nodes[nodeA];
    if (nd.binSlot < 0) return;
    const float ext = nd.cmax[nd.axis] - nd.cmin[nd.axis];
    if (ext >= 1e-12f) {
      for (int i = first + threadIdx.x; i <= last; i += blockDim.x) {
        const float4 lo = bmin[i], hi = bmax[i];
        const float4 c = make_float4((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f, 0.0f);
        const int b = binOf(nd, axisOf(c, nd.axis), nbins);
        atomicMin(&sb[b][0], fenc(lo.x)); atomicMin(&sb[b][1], fenc(lo.y)); atomicMin(&sb[b][2], fenc(lo.z));
        atomicMax(&sb[b][3], fenc(hi.x)); atomicMax(&sb[b][4], fenc(hi.y)); atomicMax(&sb[b][5], fenc(hi.z));
        atomicMin(&sb[b][6], fenc(c.x)); atomicMin(&sb[b][7], fenc(c.y)); atomicMin(&sb[b][8], fenc(c.z));
        atomicMax(&sb[b][9], fenc(c.x)); atomicMax(&sb[b][10], fenc(c.y)); atomicMax(&sb[b][11], fenc(c.z));
        atomicAdd(&sb[b][12], 1u);
      }
    }
    __syncthreads();
    BinData* nb = bins + (size_t)nd.binSlot * nbins;
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
      if (sb[b][12] == 0) continue;
      for (int k = 0; k < 3; k++) {
        atomicMin(&nb[b].bmin[k], sb[b][k]);
        atomicMax(&nb[b].bmax[k], sb[b][3 + k]);
        atomicMin(&nb[b].cmin[k], sb[b][6 + k]);
        atomicMax(&nb[b].cmax[k], sb[b][9 + k]);
      }
      atomicAdd(&nb[b].count, sb[b][12]);
    }
    return;
  }
  for (int i = first + threadIdx.x; i <= last; i += blockDim.x) {
    const int node = primNode[i];
    if (node < 0) continue;
    const BNode& nd = nodes[node];
    if (nd.binSlot < 0) continue;
    const float ext = nd.cmax[nd.axis] - nd.cmin[nd.axis];
    if (ext < 1e-12f) continue;
    const float4 lo = bmin[i], hi = bmax[i];
    const float4 c = make_float4((lo.x + hi.x) * 0.5f, (lo.y + hi.y) * 0.5f, (lo.z + hi.z) * 0.5f, 0.0f);
    const int b = binOf(nd, axisOf(c, nd.axis), nbins);
    BinData& bd = bins[(size_t)nd.binSlot * nbins + b];
    atomicMin(&bd.bmin[0], fenc(lo.x)); atomicMin(&bd.bmin[1], fenc(lo.y)); atomicMin(&bd.bmin[2], fenc(lo.z));
    atomicMax(&bd.bmax[0], fenc(hi.x)); atomicMax(&bd.bmax[1], fenc(hi.y)); atomicMax(&bd.bmax[2], fenc(hi.z));
    atomicMin(&bd.cmin[0], fenc(c.x)); atomicMin(&bd.cmin[1], fenc(c.y)); atomicMin(&bd.cmin[2], fenc(c.z));
    atomicMax(&bd.cmax[0], fenc(c.x)); atomicMax(&bd.cmax[1], fenc(c.y)); atomicMax(&bd.cmax[2], fenc(c.z));
    atomicAdd(&bd.count, 1u);
  }
}

__device__ __forceinline__ float areaOf(const float lo[3], const float hi[3]) {
  const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

// Split decision per open node (bvh.cpp:133-211 cost model).
__global__ void k_split(int numTasks, const int* __restrict__ tasks, BNode* nodes, const BinData* __restrict__ bins,
                        int nbins, int* nodeCounter, int* nextTasks, int* nextCount, int maxLeaf) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numTasks) return;
  const int id = tasks[t];
  BNode nd = nodes[id];
  const BinData* nb = bins + (size_t)nd.binSlot * nbins;
  const float ext = nd.cmax[nd.axis] - nd.cmin[nd.axis];
  int best = -1;
  float bestCost = (float)nd.count * 1.5f;
  float forcedCost = FLT_MAX;
  int forced = -1;
  // sweeps
  float la[kMaxBins];
  int lc[kMaxBins];
  if (ext >= 1e-12f) {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    int c = 0;
    for (int i = 0; i < nbins - 1; i++) {
      if (nb[i].count > 0) {
        for (int k = 0; k < 3; k++) { lo[k] = fminf(lo[k], fdec(nb[i].bmin[k])); hi[k] = fmaxf(hi[k], fdec(nb[i].bmax[k])); }
      }
      c += nb[i].count;
      la[i] = c > 0 ? areaOf(lo, hi) : 0.0f;
      lc[i] = c;
    }
    const float pa = areaOf(nd.bmin, nd.bmax);
    const float invPa = pa > 0.0f ? 1.0f / pa : 0.0f;
    float rlo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, rhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    int rc = 0;
    for (int i = nbins - 1; i > 0; i--) {
      if (nb[i].count > 0) {
        for (int k = 0; k < 3; k++) { rlo[k] = fminf(rlo[k], fdec(nb[i].bmin[k])); rhi[k] = fmaxf(rhi[k], fdec(nb[i].bmax[k])); }
      }
      rc += nb[i].count;
      const float ra = rc > 0 ? areaOf(rlo, rhi) : 0.0f;
      const int s = i - 1;
      if (lc[s] == 0 || rc == 0) continue;
      const float cost = 1.0f + 1.5f * invPa * (la[s] * (float)lc[s] + ra * (float)rc);
      if (cost < bestCost || (cost == bestCost && best >= 0 && s < best)) { bestCost = cost; best = s; }
      if (cost < forcedCost || (cost == forcedCost && s < forced)) { forcedCost = cost; forced = s; }
    }
  }
  int split = best;
  if (split < 0 && nd.count > maxLeaf) split = forced >= 0 ? forced : -2;  // -2: index median
  nd.binSlot = -1;
  if (split == -1) {
    nd.left = -1;
    nodes[id] = nd;
    return;
  }
  const int left = atomicAdd(nodeCounter, 2);
  BNode ch[2];
  int cnt[2];
  if (split == -2) {
    cnt[0] = nd.count / 2;
    cnt[1] = nd.count - cnt[0];
    for (int s = 0; s < 2; s++) {
      for (int k = 0; k < 3; k++) {
        ch[s].bmin[k] = nd.bmin[k]; ch[s].bmax[k] = nd.bmax[k];
        ch[s].cmin[k] = nd.cmin[k]; ch[s].cmax[k] = nd.cmax[k];
      }
    }
  } else {
    for (int s = 0; s < 2; s++) {
      float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
      int c = 0;
      const int b0 = s == 0 ? 0 : split + 1, b1 = s == 0 ? split + 1 : nbins;
      for (int b = b0; b < b1; b++) {
        if (nb[b].count == 0) continue;
        c += nb[b].count;
        for (int k = 0; k < 3; k++) {
          lo[k] = fminf(lo[k], fdec(nb[b].bmin[k])); hi[k] = fmaxf(hi[k], fdec(nb[b].bmax[k]));
          clo[k] = fminf(clo[k], fdec(nb[b].cmin[k])); chi[k] = fmaxf(chi[k], fdec(nb[b].cmax[k]));
        }
      }
      cnt[s] = c;
      for (int k = 0; k < 3; k++) { ch[s].bmin[k] = lo[k]; ch[s].bmax[k] = hi[k]; ch[s].cmin[k] = clo[k]; ch[s].cmax[k] = chi[k]; }
    }
  }
  for (int s = 0; s < 2; s++) {
    ch[s].start = nd.start + (s == 0 ? 0 : cnt[0]);
    ch[s].count = cnt[s];
    ch[s].left = -1;
    ch[s].axis = 0;
    ch[s].binSlot = -1;
    ch[s].splitBin = -1;
    nodes[left + s] = ch[s];
    if (cnt[s] > 4) {  // BVH_LEAF_SIZE (bvh.cpp:23): larger children stay open
      const int slot = atomicAdd(nextCount, 1);
      nextTasks[slot] = left + s;
    }
  }
  nd.left = left;
  nd.splitBin = split;
  nodes[id] = nd;
}

// The same split decision with one warp per open node (nbins <= 32: lane b holds
// bin b).  Left and right bounds come from inclusive warp scans of min / max (exact,
// so the same values as the sequential sweeps), the cost of each split from the
// same formula, and the choice is the lowest bin index of the lowest cost, as the
// sweeps choose.  The warp then resets its bins for the next use, so levels need
// no separate clear.
__device__ __forceinline__ void resetBin(BinData* b) {
  uint4* w = reinterpret_cast<uint4*>(b);
  w[0] = make_uint4(0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u);  // bmin x y z, bmax x
  w[1] = make_uint4(0u, 0u, 0xFFFFFFFFu, 0xFFFFFFFFu);           // bmax y z, cmin x y
  w[2] = make_uint4(0xFFFFFFFFu, 0u, 0u, 0u);                    // cmin z, cmax x y z
  w[3] = make_uint4(0u, 0u, 0u, 0u);                             // count, pad
}

__global__ void k_resetBins(size_t count, BinData* bins) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) resetBin(bins + i);
}

template <bool MIN>
__device__ __forceinline__ float warpScanF(float v, int lane, bool reverse) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float u = reverse ? __shfl_down_sync(0xffffffffu, v, o) : __shfl_up_sync(0xffffffffu, v, o);
    const bool in = reverse ? lane + o < 32 : lane >= o;
    if (in) v = MIN ? fminf(v, u) : fmaxf(v, u);
  }
  return v;
}

__device__ __forceinline__ int warpScanI(int v, int lane, bool reverse) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = reverse ? __shfl_down_sync(0xffffffffu, v, o) : __shfl_up_sync(0xffffffffu, v, o);
    if (reverse ? lane + o < 32 : lane >= o) v += u;
  }
  return v;
}

__global__ void __launch_bounds__(128) k_splitWarp(int numTasks, const int* __restrict__ tasks, BNode* nodes,
                                                  BinData* bins, int nbins, int* nodeCounter, int* nextTasks,
                                                  int* nextCount, int maxLeaf) {
  const int t = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (t >= numTasks) return;
  const int id = tasks[t];
  BNode nd = nodes[id];
  BinData* nb = bins + (size_t)nd.binSlot * nbins;
  // this lane's bin (identity when empty or past nbins)
  int cnt = 0;
  float blo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, bhi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  float clo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, chi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  if (lane < nbins) {
    const BinData b = nb[lane];
    cnt = (int)b.count;
    if (cnt > 0)
      for (int k = 0; k < 3; k++) {
        blo[k] = fdec(b.bmin[k]); bhi[k] = fdec(b.bmax[k]); clo[k] = fdec(b.cmin[k]); chi[k] = fdec(b.cmax[k]);
      }
    resetBin(nb + lane);
  }
  // left: bins 0..lane, right: bins lane..nbins-1
  float llo[3], lhi[3], rlo[3], rhi[3];
  for (int k = 0; k < 3; k++) {
    llo[k] = warpScanF<true>(blo[k], lane, false);
    lhi[k] = warpScanF<false>(bhi[k], lane, false);
    rlo[k] = warpScanF<true>(blo[k], lane, true);
    rhi[k] = warpScanF<false>(bhi[k], lane, true);
  }
  const int lc = warpScanI(cnt, lane, false), rcAll = warpScanI(cnt, lane, true);
  // split s = lane: left = bins 0..s, right = bins s+1..nbins-1 (the right sums of lane s + 1)
  const int rc = __shfl_down_sync(0xffffffffu, rcAll, 1);
  float rl[3], rh[3];
  for (int k = 0; k < 3; k++) {
    rl[k] = __shfl_down_sync(0xffffffffu, rlo[k], 1);
    rh[k] = __shfl_down_sync(0xffffffffu, rhi[k], 1);
  }
  const float pa = areaOf(nd.bmin, nd.bmax);
  const float invPa = pa > 0.0f ? 1.0f / pa : 0.0f;
  float cost = FLT_MAX;
  const bool valid = lane < nbins - 1 && lc > 0 && rc > 0;
  if (valid) {
    const float la = areaOf(llo, lhi), ra = areaOf(rl, rh);
    cost = 1.0f + 1.5f * invPa * (la * (float)lc + ra * (float)rc);
  }
  // lowest cost, then lowest split index
  float bc = cost;
  int bs = valid ? lane : 0x7fffffff;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
    const int os = __shfl_xor_sync(0xffffffffu, bs, o);
    if (oc < bc || (oc == bc && os < bs)) { bc = oc; bs = os; }
  }
  const int forced = bs == 0x7fffffff ? -1 : bs;
  const int best = (forced >= 0 && bc < (float)nd.count * 1.5f) ? forced : -1;
  int split = best;
  if (split < 0 && nd.count > maxLeaf) split = forced >= 0 ? forced : -2;  // -2: index median
  // child bounds: reductions over the bins of each side
  float cb[2][12];
  int cc[2];
  for (int sd = 0; sd < 2; sd++) {
    const bool mine = split >= 0 && (sd == 0 ? lane <= split : lane > split);
    for (int k = 0; k < 3; k++) {
      float v0 = mine ? blo[k] : FLT_MAX, v1 = mine ? bhi[k] : -FLT_MAX, v2 = mine ? clo[k] : FLT_MAX,
            v3 = mine ? chi[k] : -FLT_MAX;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        v0 = fminf(v0, __shfl_xor_sync(0xffffffffu, v0, o));
        v1 = fmaxf(v1, __shfl_xor_sync(0xffffffffu, v1, o));
        v2 = fminf(v2, __shfl_xor_sync(0xffffffffu, v2, o));
        v3 = fmaxf(v3, __shfl_xor_sync(0xffffffffu, v3, o));
      }
      cb[sd][k] = v0; cb[sd][3 + k] = v1; cb[sd][6 + k] = v2; cb[sd][9 + k] = v3;
    }
    int c = mine ? cnt : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    cc[sd] = c;
  }
  if (lane != 0) return;
  nd.binSlot = -1;
  if (split == -1) {
    nd.left = -1;
    nodes[id] = nd;
    return;
  }
  const int left = atomicAdd(nodeCounter, 2);
  BNode ch[2];
  int cnts[2];
  for (int sd = 0; sd < 2; sd++) {
    if (split == -2) {
      cnts[0] = nd.count / 2;
      cnts[1] = nd.count - cnts[0];
      for (int k = 0; k < 3; k++) {
        ch[sd].bmin[k] = nd.bmin[k]; ch[sd].bmax[k] = nd.bmax[k];
        ch[sd].cmin[k] = nd.cmin[k]; ch[sd].cmax[k] = nd.cmax[k];
      }
    } else {
      cnts[sd] = cc[sd];
      for (int k = 0; k < 3; k++) {
        ch[sd].bmin[k] = cb[sd][k]; ch[sd].bmax[k] = cb[sd][3 + k];
        ch[sd].cmin[k] = cb[sd][6 + k]; ch[sd].cmax[k] = cb[sd][9 + k];
      }
    }
  }
  for (int sd = 0; sd < 2; sd++) {
    ch[sd].start = nd.start + (sd == 0 ? 0 : cnts[0]);
    ch[sd].count = cnts[sd];
    ch[sd].left = -1;
    ch[sd].axis = 0;
    ch[sd].binSlot = -1;
    ch[sd].splitBin = -1;
    nodes[left + sd] = ch[sd];
    if (cnts[sd] > 4) {  // BVH_LEAF_SIZE (bvh.cpp:23): larger children stay open
      const int slot = atomicAdd(nextCount, 1);
      nextTasks[slot] = left + sd;
    }
  }
  nd.left = left;
  nd.splitBin = split;
  nodes[id] = nd;
}

// Partition, pass 1: flag 1 for a primitive that goes to the left child of its
// node (the split bin, or the first half of the node's range for a median split).
__global__ void k_partitionFlags(int n, const int* __restrict__ primNode, const BNode* __restrict__ nodes,
                                 const float4* __restrict__ bmin, const float4* __restrict__ bmax, int nbins,
                                 int* __restrict__ flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int node = primNode[i];
  int flag = 0;
  if (node >= 0) {
    const BNode& nd = nodes[node];
    if (nd.left >= 0) {
      if (nd.splitBin == -2) {
        flag = (i - nd.start) < nd.count / 2 ? 1 : 0;
      } else {
        const float4 lo = bmin[i], hi = bmax[i];
        const float c = nd.axis == 0 ? (lo.x + hi.x) * 0.5f : (nd.axis == 1 ? (lo.y + hi.y) * 0.5f : (lo.z + hi.z) * 0.5f);
        flag = binOf(nd, c, nbins) <= nd.splitBin ? 1 : 0;
      }
    }
  }
  flags[i] = flag;
}

// Partition, pass 2 (after an exclusive scan of the flags into `before`): a stable
// scatter of each split node's primitives into its children's ranges, with their
// bounds; primitives of closed nodes and new leaves stay where they are.  No
// atomics, so the order (and the BVH) is the same on every run.
__global__ void k_partitionScatter(int n, const int* __restrict__ primIdx, const int* __restrict__ primNode,
                                   const BNode* __restrict__ nodes, const float4* __restrict__ bmin,
                                   const float4* __restrict__ bmax, const int* __restrict__ flags,
                                   const int* __restrict__ before, int* __restrict__ outIdx, int* __restrict__ outNode,
                                   float4* __restrict__ outMin, float4* __restrict__ outMax, int* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int node = primNode[i];
  int pos = i, outN = -1;
  if (node >= 0) {
    const BNode& nd = nodes[node];
    if (nd.left >= 0) {
      const int leftBefore = before[i] - before[nd.start];
      const int side = flags[i] ? 0 : 1;
      const int rank = side == 0 ? leftBefore : (i - nd.start) - leftBefore;
      const BNode& cn = nodes[nd.left + side];
      if (rank >= cn.count) {
        atomicCAS(err, 0, kErrPartition);
        return;
      }
      pos = cn.start + rank;
      outN = cn.count > 4 ? nd.left + side : -1;
    }
  }
  outIdx[pos] = primIdx[i];
  outNode[pos] = outN;
  outMin[pos] = bmin[i];
  outMax[pos] = bmax[i];
}

__global__ void k_innerFlags(int numNodes, const BNode* __restrict__ nodes, int* flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < numNodes) flags[i] = nodes[i].left >= 0 ? 1 : 0;
}

__device__ __forceinline__ float inflateLo(float x) { return x - fmaxf(fabsf(x), 1.0f) * 2e-6f; }
__device__ __forceinline__ float inflateHi(float x) { return x + fmaxf(fabsf(x), 1.0f) * 2e-6f; }

__global__ void k_emitNodes(int numNodes, const BNode* __restrict__ nodes, const int* __restrict__ travIdx,
                            float4* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= numNodes) return;
  const BNode nd = nodes[i];
  if (nd.left < 0) return;
  const BNode a = nodes[nd.left], b = nodes[nd.left + 1];
  int refs[2];
  const BNode* cs[2] = {&a, &b};
  for (int s = 0; s < 2; s++) {
    const BNode& c = *cs[s];
    if (c.left >= 0) refs[s] = travIdx[nd.left + s];
    else refs[s] = ~((c.start << 3) | (c.count - 1));
  }
  float4* o = out + (size_t)travIdx[i] * 4;
  o[0] = make_float4(inflateLo(a.bmin[0]), inflateHi(a.bmax[0]), inflateLo(a.bmin[1]), inflateHi(a.bmax[1]));
  o[1] = make_float4(inflateLo(b.bmin[0]), inflateHi(b.bmax[0]), inflateLo(b.bmin[1]), inflateHi(b.bmax[1]));
  o[2] = make_float4(inflateLo(a.bmin[2]), inflateHi(a.bmax[2]), inflateLo(b.bmin[2]), inflateHi(b.bmax[2]));
  o[3] = make_float4(__int_as_float(refs[0]), __int_as_float(refs[1]), 0.0f, 0.0f);
}

__global__ void k_gather(int n, const int* __restrict__ primIdx, const float4* __restrict__ vIn,
                         const float4* __restrict__ sIn, const float2* __restrict__ uvIn, float4* __restrict__ vOut,
                         float4* __restrict__ sOut, float2* __restrict__ uvOut, int* __restrict__ orig) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = primIdx[i];
  for (int k = 0; k < 3; k++) {
    vOut[(size_t)i * 3 + k] = vIn[(size_t)p * 3 + k];
    sOut[(size_t)i * 3 + k] = sIn[(size_t)p * 3 + k];
    if (uvOut) uvOut[(size_t)i * 3 + k] = uvIn[(size_t)p * 3 + k];
  }
  orig[i] = p;
}


// ---- 8-wide BVH (collapse of the binary build) ---------------------------------
// Node (208 B = kNode8Vec float4): (childBase, triBase, meta[0..3], meta[4..7]), then
// per axis x, y, z the 8 children's lo planes and their 8 hi planes (2 float4 each).
// meta[s] = 0x80: slot s is an inner child, stored at childBase + (inner slots
// below s); ((count - 1) << 5) | offset: a leaf of `count` (1..4) triangles at
// triBase + offset; an empty slot has an inverted box and is never entered.
// Slots are assigned per octant: a child whose centre lies on the negative side
// of the node centre along axis k prefers slots with bit k set, so visiting hit
// slots in descending order of (slot XOR ray octant) is roughly front to back.
// countOnly: the same child choices, nothing written but the node count and the
// next level's tasks (the host sizes the node array with it).
__global__ void k_collapse(int numTasks, const int2* __restrict__ tasks, const BNode* __restrict__ nodes,
                           const int* __restrict__ primIdx, float4* __restrict__ nodes8, int* counters,
                           int2* __restrict__ nextTasks, int* __restrict__ triOrder, int maxNodes8, bool countOnly) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= numTasks) return;
  const int2 task = tasks[t];
  const BNode& nd = nodes[task.x];
  int ch[8];
  int nc;
  if (nd.left < 0) {
    ch[0] = task.x;
    nc = 1;
  } else {
    ch[0] = nd.left;
    ch[1] = nd.left + 1;
    nc = 2;
    while (nc < 8) {
      int best = -1;
      float bestA = -1.0f;
      for (int i = 0; i < nc; i++) {
        const BNode& c = nodes[ch[i]];
        if (c.left < 0) continue;
        const float a = areaOf(c.bmin, c.bmax);
        if (a > bestA) { bestA = a; best = i; }
      }
      if (best < 0) break;
      const int l = nodes[ch[best]].left;
      ch[best] = l;
      ch[nc++] = l + 1;
    }
  }
  if (countOnly) {
    for (int i = 0; i < nc; i++)
      if (nodes[ch[i]].left >= 0) {
        atomicAdd(&counters[0], 1);
        nextTasks[atomicAdd(&counters[2], 1)] = make_int2(ch[i], 0);
      }
    return;
  }
  float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
  float cc[8][3];
  for (int i = 0; i < nc; i++) {
    const BNode& c = nodes[ch[i]];
    for (int k = 0; k < 3; k++) {
      const float a = inflateLo(c.bmin[k]), b = inflateHi(c.bmax[k]);
      lo[k] = fminf(lo[k], a);
      hi[k] = fmaxf(hi[k], b);
      cc[i][k] = 0.5f * (c.bmin[k] + c.bmax[k]);
    }
  }
  // greedy octant slot assignment
  int slotOf[8];
  bool slotUsed[8] = {false, false, false, false, false, false, false, false};
  bool childDone[8] = {false, false, false, false, false, false, false, false};
  const float ctr[3] = {0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2])};
  for (int it = 0; it < nc; it++) {
    float bestS = -FLT_MAX;
    int bj = -1, bs = -1;
    for (int j = 0; j < nc; j++) {
      if (childDone[j]) continue;
      for (int sl = 0; sl < 8; sl++) {
        if (slotUsed[sl]) continue;
        const float sc = (cc[j][0] - ctr[0]) * ((sl & 1) ? -1.0f : 1.0f) + (cc[j][1] - ctr[1]) * ((sl & 2) ? -1.0f : 1.0f) +
                         (cc[j][2] - ctr[2]) * ((sl & 4) ? -1.0f : 1.0f);
        if (sc > bestS) { bestS = sc; bj = j; bs = sl; }
      }
    }
    childDone[bj] = true;
    slotUsed[bs] = true;
    slotOf[bj] = bs;
  }
  int childAt[8];
  for (int sl = 0; sl < 8; sl++) childAt[sl] = -1;
  for (int j = 0; j < nc; j++) childAt[slotOf[j]] = ch[j];
  // float planes of the child boxes (each widened by the inflate margin); an empty
  // slot keeps an inverted box (+inf / -inf) that no ray enters
  float pl[3][2][8];
  for (int k = 0; k < 3; k++)
    for (int sl = 0; sl < 8; sl++) {
      pl[k][0][sl] = INFINITY;
      pl[k][1][sl] = -INFINITY;
    }
  uint32_t meta[2] = {0, 0};
  int ni = 0, ntri = 0;
  for (int sl = 0; sl < 8; sl++) {
    const int c = childAt[sl];
    if (c < 0) continue;
    const BNode& cn = nodes[c];
    for (int k = 0; k < 3; k++) {
      pl[k][0][sl] = inflateLo(cn.bmin[k]);
      pl[k][1][sl] = inflateHi(cn.bmax[k]);
    }
    if (cn.left >= 0) {
      meta[sl >> 2] |= 0x80u << (8 * (sl & 3));
      ni++;
    } else {
      meta[sl >> 2] |= (uint32_t)(((cn.count - 1) << 5) | ntri) << (8 * (sl & 3));
      ntri += cn.count;
    }
  }
  const int childBase = ni ? atomicAdd(&counters[0], ni) : 0;
  const int triBase = atomicAdd(&counters[1], ntri);
  if (childBase + ni > maxNodes8) {
    atomicCAS(&counters[3], 0, kErrPartition);
    return;
  }
  float4* o = nodes8 + (size_t)task.y * kNode8Vec;
  o[0] = make_float4(__int_as_float(childBase), __int_as_float(triBase), __uint_as_float(meta[0]), __uint_as_float(meta[1]));
  for (int k = 0; k < 3; k++)
    for (int h = 0; h < 2; h++) {
      const float* q = pl[k][h];
      o[1 + 4 * k + 2 * h] = make_float4(q[0], q[1], q[2], q[3]);
      o[2 + 4 * k + 2 * h] = make_float4(q[4], q[5], q[6], q[7]);
    }
  int k = 0, off = 0;
  for (int sl = 0; sl < 8; sl++) {
    const int c = childAt[sl];
    if (c < 0) continue;
    const BNode& cn = nodes[c];
    if (cn.left >= 0) {
      const int slot = atomicAdd(&counters[2], 1);
      nextTasks[slot] = make_int2(c, childBase + k);
      k++;
    } else {
      for (int q = 0; q < cn.count; q++) triOrder[triBase + off + q] = primIdx[cn.start + q];
      off += cn.count;
    }
  }
}

inline int gridFor(long long n, int block) { return (int)((n + block - 1) / block); }

}  // namespace

// Builds the view-space triangle arrays and the BVH for `n` triangles whose
// world-space inputs are already on the device (DeviceSceneBuild fields).
// Per-level host timing of the build, printed to stderr when RG_TRACE_HOST is set.
struct BuildTrace {
  bool on = std::getenv("RG_TRACE_HOST") != nullptr;
  std::chrono::steady_clock::time_point last = std::chrono::steady_clock::now();
  void mark(const char* what, int level, int tasks) {
    if (!on) return;
    const auto t = std::chrono::steady_clock::now();
    std::fprintf(stderr, "[rg] bvh %-10s %3d: %8d tasks %8.3f ms\n", what, level, tasks,
                 std::chrono::duration<double, std::milli>(t - last).count());
    last = t;
  }
};

// The build's working arrays; a scene rebuilt in place keeps them, so a build no
// larger than the last allocates nothing (DevBuf::alloc only grows).
struct BvhScratch {
  DevBuf<float4> vTmp, sTmp, lo, hi, lo2, hi2;
  DevBuf<float2> uvTmp;
  DevBuf<uint32_t> rb;
  DevBuf<BNode> nodes;
  DevBuf<int> idxA, idxB, nodeA, nodeB, tasksA, tasksB, counters, pflags, pbefore;
  DevBuf<BinData> bins;
  DevBuf<unsigned char> scanTmp, tmp;
  DevBuf<int2> ta, tb;
  DevBuf<int> order, c8, flags, trav;
};

void freeBvhScratch(BvhScratch* s) { delete s; }

rg_status buildDeviceBvh(DeviceScene& ds, int nbins, bool wide, cudaStream_t st, std::string& err) {
  BuildTrace trace;
  const int n = ds.numTris;
  nbins = nbins < 2 ? 2 : (nbins > kMaxBins ? kMaxBins : nbins);
  ds.rootIsLeaf = 0;
  ds.rootLeafRef = 0;
  ds.numNodes = 0;
  if (n == 0) return RG_OK;
  if (!ds.scratch) ds.scratch = new BvhScratch();
  BvhScratch& X = *ds.scratch;
  DevBuf<float4> &vTmp = X.vTmp, &sTmp = X.sTmp, &lo = X.lo, &hi = X.hi, &lo2 = X.lo2, &hi2 = X.hi2;
  DevBuf<float2>& uvTmp = X.uvTmp;
  if (!vTmp.alloc((size_t)n * 3) || !sTmp.alloc((size_t)n * 3) || !lo.alloc(n) || !hi.alloc(n)) {
    err = "out of device memory (triangle staging)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  if (ds.hasUV && !uvTmp.alloc((size_t)n * 3)) {
    err = "out of device memory (triangle staging)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  trace.mark("alloc stage", 0, n);
  k_prepTriangles<<<gridFor(n, 256), 256, 0, st>>>(n, ds.inPos.p, ds.inNrm.p, ds.hasUV ? ds.inUV.p : nullptr,
                                                   ds.inTriMesh.p, ds.meshObj.p, ds.objMat.p, ds.mats.p, ds.view.p,
                                                   vTmp.p, sTmp.p, ds.hasUV ? uvTmp.p : nullptr, lo.p, hi.p);
  // root bounds
  DevBuf<uint32_t>& rb = X.rb;
  if (!rb.alloc(12)) {
    err = "out of device memory (BVH build)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  {
    std::vector<uint32_t> init(12);
    for (int k = 0; k < 3; k++) { init[k] = 0xFFFFFFFFu; init[3 + k] = 0u; init[6 + k] = 0xFFFFFFFFu; init[9 + k] = 0u; }
    cudaMemcpyAsync(rb.p, init.data(), 12 * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
  }
  k_rootBounds<<<std::min(gridFor(n, 256), 1184), 256, 0, st>>>(n, lo.p, hi.p, rb.p);
  const size_t maxNodes = 2 * (size_t)n + 1;
  // bins for at most chunkTasks open nodes at a time (<= 256 MB)
  const int chunkTasks = (int)std::min<size_t>((size_t)n / 4 + 2, ((size_t)256 << 20) / (sizeof(BinData) * nbins));
  DevBuf<BNode>& nodes = X.nodes;
  DevBuf<int> &idxA = X.idxA, &idxB = X.idxB, &nodeA = X.nodeA, &nodeB = X.nodeB, &tasksA = X.tasksA,
  &tasksB = X.tasksB, &counters = X.counters, &pflags = X.pflags, &pbefore = X.pbefore;
  DevBuf<BinData>& bins = X.bins;
  trace.mark("prep kern", 0, n);
  if (!nodes.alloc(maxNodes) || !idxA.alloc(n) || !idxB.alloc(n) || !nodeA.alloc(n) || !nodeB.alloc(n) ||
      !lo2.alloc(n) || !hi2.alloc(n) || !pflags.alloc(n) || !pbefore.alloc(n) ||
      !tasksA.alloc((size_t)n / 4 + 2) || !tasksB.alloc((size_t)n / 4 + 2) || !counters.alloc(4) ||
      !bins.alloc((size_t)chunkTasks * nbins)) {
    err = "out of device memory (BVH build)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  const int rootOpen = n > 4 ? 1 : 0;
  k_initRoot<<<gridFor(n, 256), 256, 0, st>>>(n, rb.p, nodes.p, idxA.p, nodeA.p, rootOpen);
  int h_counters[4] = {1, 0, 0, 0};  // [0] node count, [1] next task count, [2] error
  cudaMemcpyAsync(counters.p, h_counters, sizeof(h_counters), cudaMemcpyHostToDevice, st);
  int numTasks = rootOpen;
  {
    const int zero = 0;
    cudaMemcpyAsync(tasksA.p, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
  }
  int* curIdx = idxA.p;
  int* curNode = nodeA.p;
  int* altIdx = idxB.p;
  int* altNode = nodeB.p;
  int* curTasks = tasksA.p;
  int* nxtTasks = tasksB.p;
  // up to 32 bins: one warp per node decides the split and resets its bins, which
  // therefore start reset once here
  const bool warpSplit = nbins <= 32;
  if (warpSplit) {
    const size_t nb = (size_t)chunkTasks * nbins;
    k_resetBins<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(nb, bins.p);
  }
  // scratch of the partition's prefix sum
  size_t scanBytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, pflags.p, pbefore.p, n, st);
  DevBuf<unsigned char>& scanTmp = X.scanTmp;
  if (!scanTmp.alloc(scanBytes + 16)) {
    err = "out of device memory (BVH build)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  float4* curLo = lo.p;
  float4* curHi = hi.p;
  float4* altLo = lo2.p;
  float4* altHi = hi2.p;
  int levels = 0;
  trace.mark("alloc tree", 0, n);
  trace.mark("prep", 0, numTasks);
  while (numTasks > 0) {
    levels++;
    const int tasksThisLevel = numTasks;
    cudaMemsetAsync(counters.p + 1, 0, sizeof(int), st);
    for (int c0 = 0; c0 < numTasks; c0 += chunkTasks) {
      const int nt = std::min(chunkTasks, numTasks - c0);
      const int prepN = warpSplit ? nt : std::max(nt, nt * nbins);
      k_prepareLevel<<<gridFor(prepN, 256), 256, 0, st>>>(nt, curTasks + c0, nodes.p, bins.p, nbins, !warpSplit);
      k_bin<<<gridFor(n, kBinChunk), 256, 0, st>>>(n, curNode, nodes.p, curLo, curHi, bins.p, nbins);
      if (warpSplit)
        k_splitWarp<<<gridFor((long long)nt * 32, 128), 128, 0, st>>>(nt, curTasks + c0, nodes.p, bins.p, nbins,
                                                                      counters.p, nxtTasks, counters.p + 1,
                                                                      wide ? kWideMaxLeaf : kMaxLeaf);
      else
        k_split<<<gridFor(nt, 128), 128, 0, st>>>(nt, curTasks + c0, nodes.p, bins.p, nbins, counters.p, nxtTasks,
                                                   counters.p + 1, wide ? kWideMaxLeaf : kMaxLeaf);
    }
    k_partitionFlags<<<gridFor(n, 256), 256, 0, st>>>(n, curNode, nodes.p, curLo, curHi, nbins, pflags.p);
    cub::DeviceScan::ExclusiveSum(scanTmp.p, scanBytes, pflags.p, pbefore.p, n, st);
    k_partitionScatter<<<gridFor(n, 256), 256, 0, st>>>(n, curIdx, curNode, nodes.p, curLo, curHi, pflags.p, pbefore.p,
                                                        altIdx, altNode, altLo, altHi, counters.p + 2);
    std::swap(curIdx, altIdx);
    std::swap(curNode, altNode);
    std::swap(curLo, altLo);
    std::swap(curHi, altHi);
    std::swap(curTasks, nxtTasks);
    cudaMemcpyAsync(&numTasks, counters.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      err = "BVH build level failed";
      return RG_ERR_CUDA;
    }
    trace.mark("level", levels, tasksThisLevel);
    if (levels > 200) {
      err = "BVH build did not converge";
      return RG_ERR_DEVICE_STATUS;
    }
  }
  int numNodes = 0, buildErr = 0;
  cudaMemcpyAsync(&numNodes, counters.p, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&buildErr, counters.p + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  if (buildErr != 0) {
    err = "BVH build scatter error " + std::to_string(buildErr);
    return RG_ERR_DEVICE_STATUS;
  }
  ds.buildLevels = levels;
  trace.mark("levels end", 0, n);
  if (!ds.triVerts.alloc((size_t)n * 3) || !ds.triShade.alloc((size_t)n * 3) || !ds.triOrig.alloc(n)) {
    err = "out of device memory (triangles)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  if (ds.hasUV && !ds.triUV.alloc((size_t)n * 3)) {
    err = "out of device memory (triangles)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  trace.mark("alloc tris", 0, n);
  if (wide) {
    // collapse to the 8-wide compressed layout, level by level
    ds.bvhWidth = 8;
    const int maxTasks8 = numNodes + 1;
    DevBuf<int2> &ta = X.ta, &tb = X.tb;
    DevBuf<int> &order = X.order, &c8 = X.c8;
    if (!ta.alloc(maxTasks8) || !tb.alloc(maxTasks8) || !order.alloc(n) || !c8.alloc(4)) {
      err = "out of device memory (wide BVH)";
      return RG_ERR_OUT_OF_MEMORY;
    }
    // two passes over the levels: the first counts the 8-wide nodes, so the node
    // array is allocated at its size (about a seventh of the binary node count)
    int numNodes8 = 0;
    for (int pass = 0; pass < 2; pass++) {
      const bool countOnly = pass == 0;
      if (!countOnly && !ds.nodes8.alloc((size_t)numNodes8 * kNode8Vec)) {
        err = "out of device memory (wide BVH)";
        return RG_ERR_OUT_OF_MEMORY;
      }
      trace.mark(countOnly ? "count wide" : "alloc wide", 0, numNodes8);
      const int init[4] = {1, 0, 0, 0};  // [0] nodes (root preallocated) [1] triangles [2] next tasks [3] error
      cudaMemcpyAsync(c8.p, init, sizeof(init), cudaMemcpyHostToDevice, st);
      const int2 root = make_int2(0, 0);
      cudaMemcpyAsync(ta.p, &root, sizeof(int2), cudaMemcpyHostToDevice, st);
      int nt = 1;
      int2* cur = ta.p;
      int2* nxt = tb.p;
      int lv = 0;
      while (nt > 0) {
        cudaMemsetAsync(c8.p + 2, 0, sizeof(int), st);
        k_collapse<<<gridFor(nt, 64), 64, 0, st>>>(nt, cur, nodes.p, curIdx, ds.nodes8.p, c8.p, nxt, order.p,
                                                   numNodes8, countOnly);
        cudaMemcpyAsync(&nt, c8.p + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) {
          err = "wide BVH collapse failed";
          return RG_ERR_CUDA;
        }
        if (!countOnly) trace.mark("collapse", lv + 1, nt);
        std::swap(cur, nxt);
        if (++lv > 200) {
          err = "wide BVH collapse did not converge";
          return RG_ERR_DEVICE_STATUS;
        }
      }
      if (countOnly) {
        if (cudaMemcpy(&numNodes8, c8.p, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || numNodes8 < 1 ||
            numNodes8 > maxTasks8) {
          err = "wide BVH node count failed";
          return RG_ERR_DEVICE_STATUS;
        }
      }
    }
    int h8[4];
    cudaMemcpy(h8, c8.p, sizeof(h8), cudaMemcpyDeviceToHost);
    if (h8[3] != 0 || h8[1] != n || h8[0] != numNodes8) {
      err = "wide BVH collapse error (nodes " + std::to_string(h8[0]) + ", triangles " + std::to_string(h8[1]) + ")";
      return RG_ERR_DEVICE_STATUS;
    }
    ds.numNodes8 = h8[0];
    ds.numNodes = 0;
    k_gather<<<gridFor(n, 256), 256, 0, st>>>(n, order.p, vTmp.p, sTmp.p, ds.hasUV ? uvTmp.p : nullptr, ds.triVerts.p,
                                              ds.triShade.p, ds.hasUV ? ds.triUV.p : nullptr, ds.triOrig.p);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
      err = std::string("BVH gather failed: ") + cudaGetErrorString(cudaGetLastError());
      return RG_ERR_CUDA;
    }
    trace.mark("gather", 0, n);
    return RG_OK;
  }
  // binary traversal layout
  ds.bvhWidth = 2;
  DevBuf<int> &flags = X.flags, &trav = X.trav;
  if (!flags.alloc(numNodes) || !trav.alloc(numNodes)) {
    err = "out of device memory (BVH layout)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  k_innerFlags<<<gridFor(numNodes, 256), 256, 0, st>>>(numNodes, nodes.p, flags.p);
  size_t tmpBytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmpBytes, flags.p, trav.p, numNodes, st);
  DevBuf<unsigned char>& tmp = X.tmp;
  if (!tmp.alloc(tmpBytes + 16)) {
    err = "out of device memory (BVH layout)";
    return RG_ERR_OUT_OF_MEMORY;
  }
  cub::DeviceScan::ExclusiveSum(tmp.p, tmpBytes, flags.p, trav.p, numNodes, st);
  int lastFlag = 0, lastTrav = 0;
  cudaMemcpyAsync(&lastFlag, flags.p + numNodes - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(&lastTrav, trav.p + numNodes - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  const int numInner = lastFlag + lastTrav;
  ds.numNodes = numInner;
  if (numInner == 0) {
    ds.rootIsLeaf = 1;
    ds.rootLeafRef = ~((0 << 3) | (n - 1));
    if (!ds.nodes.alloc(4)) {
      err = "out of device memory (BVH nodes)";
      return RG_ERR_OUT_OF_MEMORY;
    }
  } else {
    if (!ds.nodes.alloc((size_t)numInner * 4)) {
      err = "out of device memory (BVH nodes)";
      return RG_ERR_OUT_OF_MEMORY;
    }
    k_emitNodes<<<gridFor(numNodes, 256), 256, 0, st>>>(numNodes, nodes.p, trav.p, ds.nodes.p);
  }
  k_gather<<<gridFor(n, 256), 256, 0, st>>>(n, curIdx, vTmp.p, sTmp.p, ds.hasUV ? uvTmp.p : nullptr, ds.triVerts.p,
                                            ds.triShade.p, ds.hasUV ? ds.triUV.p : nullptr, ds.triOrig.p);
  if (cudaStreamSynchronize(st) != cudaSuccess) {
    err = std::string("BVH build failed: ") + cudaGetErrorString(cudaGetLastError());
    return RG_ERR_CUDA;
  }
  return RG_OK;
}

}  // namespace rg
