// rg_scene.cpp - procedural scene descriptions (host C++).
//
// The reference renders authored JSON scenes (resources/scenes/*); the
// workloads here are seeded procedural stand-ins with the shapes the
// benchmark configurations name:
//   kind 1  cube room: 10 wall triangles, two boxes (24), one ceiling quad
//   kind 2  displaced geodesic icosphere (~1M triangles) x4 in a 20x20 room,
//           16 emissive ceiling quads, metal / dielectric sphere materials
//   kind 3  kind 2 filled with a homogeneous medium (sigma_t 0.05, albedo 0.8, g 0.3)
//   kind 4  one job of the heterogeneous batch (triangle and emitter counts given)
// Triangles are emitted in the reference's DFS order (objects -> meshes ->
// triangles, rayrenderer.cpp:237-363); that index is the triangle id.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "rg_host.h"

namespace rg {

namespace {

struct F3 {
  float x, y, z;
};
inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 mul(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross3(F3 a, F3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline F3 norm3(F3 a) {
  const float l = std::sqrt(dot3(a, a));
  return l > 0 ? mul(a, 1.0f / l) : a;
}

// Small deterministic generator for scene parameters (splitmix64).
struct SceneRng {
  uint64_t s;
  explicit SceneRng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  float uniform(float a, float b) { return a + (b - a) * (float)((next() >> 40) * (1.0 / 16777216.0)); }
};

rg_material defaultMaterial() {  // Material defaults, material.h:20-70
  rg_material m;
  std::memset(&m, 0, sizeof(m));
  m.color[0] = m.color[1] = m.color[2] = 0.8f;
  m.diffuse = 0.8f;
  m.roughness = 0.5f;
  m.refraction_ratio = 1.45f;
  m.texture = -1;
  m.tex_tiling[0] = m.tex_tiling[1] = 1.0f;
  return m;
}

rg_material diffuseMat(float r, float g, float b) {
  rg_material m = defaultMaterial();
  m.color[0] = r; m.color[1] = g; m.color[2] = b;
  return m;
}

rg_material emitterMat(float radiance) {
  rg_material m = diffuseMat(1, 1, 1);
  m.emission = radiance;
  return m;
}

}  // namespace

// Growing description; the arrays are owned by SceneStore and exposed through rg_scene_desc.
struct SceneBuilder {
  SceneStore& st;
  int curMesh = -1;
  explicit SceneBuilder(SceneStore& s) : st(s) {}

  int material(const rg_material& m) {
    st.materials.push_back(m);
    return (int)st.materials.size() - 1;
  }
  int object(int mat, int medium = -1) {
    rg_object o{};
    o.material = mat;
    o.interior_medium = medium;
    st.objects.push_back(o);
    return (int)st.objects.size() - 1;
  }
  int mesh(int obj) {
    st.meshObject.push_back(obj);
    curMesh = (int)st.meshObject.size() - 1;
    return curMesh;
  }
  void tri(F3 a, F3 b, F3 c, F3 na, F3 nb, F3 nc) {
    const float p[9] = {a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z};
    const float n[9] = {na.x, na.y, na.z, nb.x, nb.y, nb.z, nc.x, nc.y, nc.z};
    st.positions.insert(st.positions.end(), p, p + 9);
    st.normals.insert(st.normals.end(), n, n + 9);
    for (int k = 0; k < 6; k++) st.uvs.push_back(0.0f);
    st.triMesh.push_back(curMesh);
  }
  void flatTri(F3 a, F3 b, F3 c) {
    const F3 n = norm3(cross3(sub(b, a), sub(c, a)));
    tri(a, b, c, n, n, n);
  }
  // Quad a-b-c-d (counter-clockwise seen from the side the normal points to).
  void quad(F3 a, F3 b, F3 c, F3 d) {
    flatTri(a, b, c);
    flatTri(a, c, d);
  }
  // Axis-aligned box of size (sx, sy, sz) standing on y = y0, rotated by yaw
  // degrees about its vertical axis through (cx, cz). 12 triangles.
  void box(float cx, float y0, float cz, float sx, float sy, float sz, float yawDeg) {
    const float a = yawDeg * 3.14159265358979f / 180.0f;
    const float ca = std::cos(a), sa = std::sin(a);
    auto P = [&](float lx, float ly, float lz) {
      return f3(cx + ca * lx + sa * lz, y0 + ly, cz - sa * lx + ca * lz);
    };
    const float hx = sx * 0.5f, hz = sz * 0.5f;
    const F3 v[8] = {P(-hx, 0, -hz), P(hx, 0, -hz), P(hx, 0, hz), P(-hx, 0, hz),
                     P(-hx, sy, -hz), P(hx, sy, -hz), P(hx, sy, hz), P(-hx, sy, hz)};
    quad(v[3], v[2], v[6], v[7]);  // +z
    quad(v[1], v[0], v[4], v[5]);  // -z
    quad(v[2], v[1], v[5], v[6]);  // +x
    quad(v[0], v[3], v[7], v[4]);  // -x
    quad(v[7], v[6], v[5], v[4]);  // top
    quad(v[0], v[1], v[2], v[3]);  // bottom
  }
};

namespace {

// Value noise on an integer lattice with smoothstep interpolation, seeded.
struct ValueNoise {
  uint32_t seed;
  float lattice(int x, int y, int z) const {
    uint32_t h = (uint32_t)x * 374761393u + (uint32_t)y * 668265263u + (uint32_t)z * 2147483647u + seed * 1274126177u;
    h = (h ^ (h >> 13)) * 1274126177u;
    h ^= h >> 16;
    return (float)(h & 0xFFFFFFu) * (1.0f / 16777216.0f) * 2.0f - 1.0f;
  }
  float noise(F3 p) const {
    const float fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
    const int ix = (int)fx, iy = (int)fy, iz = (int)fz;
    float tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
    tx = tx * tx * (3 - 2 * tx); ty = ty * ty * (3 - 2 * ty); tz = tz * tz * (3 - 2 * tz);
    auto L = [&](int a, int b, int c) { return lattice(ix + a, iy + b, iz + c); };
    const float x00 = L(0, 0, 0) + (L(1, 0, 0) - L(0, 0, 0)) * tx;
    const float x10 = L(0, 1, 0) + (L(1, 1, 0) - L(0, 1, 0)) * tx;
    const float x01 = L(0, 0, 1) + (L(1, 0, 1) - L(0, 0, 1)) * tx;
    const float x11 = L(0, 1, 1) + (L(1, 1, 1) - L(0, 1, 1)) * tx;
    const float y0 = x00 + (x10 - x00) * ty, y1 = x01 + (x11 - x01) * ty;
    return y0 + (y1 - y0) * tz;
  }
  // 4-octave fBm in [-1, 1].
  float fbm(F3 p) const {
    float sum = 0, amp = 0.5f, freq = 1.0f, norm = 0;
    for (int o = 0; o < 4; o++) {
      sum += amp * noise(mul(p, freq));
      norm += amp;
      amp *= 0.5f;
      freq *= 2.0f;
    }
    return sum / norm;
  }
};

// Indexed geodesic sphere (class-I subdivision of the icosahedron with
// frequency f: 20 f^2 triangles), displaced along the radius by
// amplitude * fBm(dir * 3). Shared edge points are computed with a
// vertex-order-canonical formula so the mesh is watertight.
struct IndexedMesh {
  std::vector<F3> pos, nrm;
  std::vector<uint32_t> idx;
};

IndexedMesh geodesicSphere(int f, float radius, float amplitude, uint32_t seed) {
  const float t = (1.0f + std::sqrt(5.0f)) * 0.5f;
  F3 ico[12] = {f3(-1, t, 0), f3(1, t, 0), f3(-1, -t, 0), f3(1, -t, 0), f3(0, -1, t), f3(0, 1, t),
                f3(0, -1, -t), f3(0, 1, -t), f3(t, 0, -1), f3(t, 0, 1), f3(-t, 0, -1), f3(-t, 0, 1)};
  for (auto& v : ico) v = norm3(v);
  static const int faces[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11},
                                   {1, 5, 9}, {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8},
                                   {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8}, {3, 8, 9},
                                   {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
  ValueNoise vn{seed};
  IndexedMesh m;
  std::unordered_map<uint64_t, uint32_t> lookup;
  lookup.reserve((size_t)10 * f * f + 16);
  auto vertex = [&](int fa, int ia, int fb, int ib, int fc, int ic) -> uint32_t {
    // canonical order: nonzero weights by icosahedron vertex id, zero weights last
    int vid[3] = {fa, fb, fc}, w[3] = {ia, ib, ic};
    auto before = [&](int p, int q) {
      if ((w[p] == 0) != (w[q] == 0)) return w[p] != 0;
      return vid[p] < vid[q];
    };
    for (int a = 0; a < 3; a++)
      for (int b = a + 1; b < 3; b++)
        if (before(b, a)) { std::swap(vid[a], vid[b]); std::swap(w[a], w[b]); }
    for (int k = 0; k < 3; k++) if (w[k] == 0) vid[k] = 0;
    // key: the nonzero (vertex, weight) pairs
    uint64_t key = 0;
    for (int k = 0; k < 3; k++) {
      const uint64_t part = w[k] ? ((uint64_t)vid[k] << 16 | (uint64_t)w[k]) : 0;
      key = key * 0x200000ull + part;
    }
    auto it = lookup.find(key);
    if (it != lookup.end()) return it->second;
    const float inv = 1.0f / (float)f;
    F3 p = add(add(mul(ico[vid[0]], (float)w[0] * inv), mul(ico[vid[1]], (float)w[1] * inv)), mul(ico[vid[2]], (float)w[2] * inv));
    const F3 dir = norm3(p);
    const float r = radius + amplitude * vn.fbm(mul(dir, 3.0f));
    m.pos.push_back(mul(dir, r));
    const uint32_t id = (uint32_t)m.pos.size() - 1;
    lookup.emplace(key, id);
    return id;
  };
  for (int fi = 0; fi < 20; fi++) {
    const int A = faces[fi][0], B = faces[fi][1], C = faces[fi][2];
    // grid point (i, j): weights A: f-i-j, B: i, C: j
    auto V = [&](int i, int j) { return vertex(A, f - i - j, B, i, C, j); };
    for (int j = 0; j < f; j++)
      for (int i = 0; i + j < f; i++) {
        const uint32_t a = V(i, j), b = V(i + 1, j), c = V(i, j + 1);
        m.idx.push_back(a); m.idx.push_back(b); m.idx.push_back(c);
        if (i + j + 1 < f) {
          const uint32_t d = V(i + 1, j + 1);
          m.idx.push_back(b); m.idx.push_back(d); m.idx.push_back(c);
        }
      }
  }
  // area-weighted vertex normals
  m.nrm.assign(m.pos.size(), f3(0, 0, 0));
  for (size_t k = 0; k < m.idx.size(); k += 3) {
    const F3 a = m.pos[m.idx[k]], b = m.pos[m.idx[k + 1]], c = m.pos[m.idx[k + 2]];
    const F3 n = cross3(sub(b, a), sub(c, a));
    for (int q = 0; q < 3; q++) m.nrm[m.idx[k + q]] = add(m.nrm[m.idx[k + q]], n);
  }
  for (auto& n : m.nrm) n = norm3(n);
  return m;
}

void addIndexed(SceneBuilder& b, const IndexedMesh& m, F3 offset) {
  const size_t nt = m.idx.size() / 3;
  b.st.positions.reserve(b.st.positions.size() + nt * 9);
  b.st.normals.reserve(b.st.normals.size() + nt * 9);
  b.st.uvs.reserve(b.st.uvs.size() + nt * 6);
  b.st.triMesh.reserve(b.st.triMesh.size() + nt);
  for (size_t k = 0; k < m.idx.size(); k += 3) {
    const F3 a = add(m.pos[m.idx[k]], offset), bb = add(m.pos[m.idx[k + 1]], offset), c = add(m.pos[m.idx[k + 2]], offset);
    b.tri(a, bb, c, m.nrm[m.idx[k]], m.nrm[m.idx[k + 1]], m.nrm[m.idx[k + 2]]);
  }
}

rg_camera defaultCamera() {  // Camera defaults, scene.h:118-137
  rg_camera c;
  std::memset(&c, 0, sizeof(c));
  c.field_of_view = 75.0f;
  c.view_near = 0.1f;
  c.view_far = 50.0f;
  c.depth_of_field = 0.0f;
  c.aperture = 1.8f;
  c.exposure = 1.0f;
  return c;
}

void buildCubeRoom(SceneStore& st) {
  SceneBuilder b(st);
  const int white = b.material(diffuseMat(0.73f, 0.73f, 0.73f));
  const int red = b.material(diffuseMat(0.65f, 0.05f, 0.05f));
  const int green = b.material(diffuseMat(0.12f, 0.45f, 0.15f));
  const int light = b.material(emitterMat(15.0f));
  // room x [-5,5], y [0,10], z [-5,5]; open towards +z (the camera)
  b.mesh(b.object(white));
  b.quad(f3(-5, 0, 5), f3(5, 0, 5), f3(5, 0, -5), f3(-5, 0, -5));      // floor (+y)
  b.quad(f3(-5, 10, -5), f3(5, 10, -5), f3(5, 10, 5), f3(-5, 10, 5));  // ceiling (-y)
  b.quad(f3(-5, 0, -5), f3(5, 0, -5), f3(5, 10, -5), f3(-5, 10, -5));  // back (+z)
  b.mesh(b.object(red));
  b.quad(f3(-5, 0, 5), f3(-5, 0, -5), f3(-5, 10, -5), f3(-5, 10, 5));  // left (+x)
  b.mesh(b.object(green));
  b.quad(f3(5, 0, -5), f3(5, 0, 5), f3(5, 10, 5), f3(5, 10, -5));      // right (-x)
  b.mesh(b.object(white));
  b.box(1.6f, 0.0f, 1.2f, 3.0f, 3.0f, 3.0f, -17.0f);
  b.mesh(b.object(white));
  b.box(-1.7f, 0.0f, -1.6f, 3.0f, 6.0f, 3.0f, 17.0f);
  b.mesh(b.object(light));
  b.quad(f3(-1.25f, 9.99f, -1.25f), f3(1.25f, 9.99f, -1.25f), f3(1.25f, 9.99f, 1.25f), f3(-1.25f, 9.99f, 1.25f));
  st.camera = defaultCamera();
  st.camera.location[0] = 0.0f; st.camera.location[1] = 5.0f; st.camera.location[2] = 18.5f;
  st.camera.field_of_view = 40.0f;
}

void buildRoom20(SceneBuilder& b, int nLights, SceneRng& rng) {
  const int floorM = b.material(diffuseMat(0.6f, 0.6f, 0.6f));
  const int wallM = b.material(diffuseMat(0.73f, 0.71f, 0.68f));
  const int redM = b.material(diffuseMat(0.65f, 0.08f, 0.06f));
  const int blueM = b.material(diffuseMat(0.08f, 0.15f, 0.55f));
  b.mesh(b.object(floorM));
  b.quad(f3(-10, 0, 10), f3(10, 0, 10), f3(10, 0, -10), f3(-10, 0, -10));
  b.mesh(b.object(wallM));
  b.quad(f3(-10, 10, -10), f3(10, 10, -10), f3(10, 10, 10), f3(-10, 10, 10));  // ceiling
  b.quad(f3(-10, 0, -10), f3(10, 0, -10), f3(10, 10, -10), f3(-10, 10, -10));  // back
  b.quad(f3(10, 0, 10), f3(-10, 0, 10), f3(-10, 10, 10), f3(10, 10, 10));      // front (behind camera)
  b.mesh(b.object(redM));
  b.quad(f3(-10, 0, 10), f3(-10, 0, -10), f3(-10, 10, -10), f3(-10, 10, 10));  // left
  b.mesh(b.object(blueM));
  b.quad(f3(10, 0, -10), f3(10, 0, 10), f3(10, 10, 10), f3(10, 10, -10));      // right
  // emissive ceiling quads on a square-ish grid, radiance U[5, 20]
  int gx = 1;
  while (gx * gx < nLights) gx++;
  const float cell = 20.0f / (float)gx;
  const float half = std::fmin(0.75f, cell * 0.3f);
  for (int i = 0; i < nLights; i++) {
    const float cx = -10.0f + cell * ((float)(i % gx) + 0.5f);
    const float cz = -10.0f + cell * ((float)(i / gx) + 0.5f);
    const int m = b.material(emitterMat(rng.uniform(5.0f, 20.0f)));
    b.mesh(b.object(m));
    b.quad(f3(cx - half, 9.99f, cz - half), f3(cx + half, 9.99f, cz - half), f3(cx + half, 9.99f, cz + half),
           f3(cx - half, 9.99f, cz + half));
  }
}

rg_material sphereMaterial(int kind, SceneRng& rng) {
  rg_material m = defaultMaterial();
  if (kind == 0) {  // metal: GGX roughness U[0.05,1], F0 U[0.5,1]
    m.glossy = 1.0f;
    m.metallic = 1.0f;
    m.roughness = rng.uniform(0.05f, 1.0f);
    m.color[0] = rng.uniform(0.5f, 1.0f); m.color[1] = rng.uniform(0.5f, 1.0f); m.color[2] = rng.uniform(0.5f, 1.0f);
  } else {          // dielectric IOR 1.5
    m.refraction = 1.0f;
    m.refraction_ratio = 1.5f;
    m.roughness = 0.0f;
    m.color[0] = m.color[1] = m.color[2] = 1.0f;
  }
  return m;
}

void buildHeavy(SceneStore& st, uint32_t seed, int trisPerSphere, bool medium) {
  SceneRng rng(seed);
  SceneBuilder b(st);
  buildRoom20(b, 16, rng);
  int f = (int)std::lround(std::sqrt((double)trisPerSphere / 20.0));
  if (f < 1) f = 1;
  const IndexedMesh sphere = geodesicSphere(f, 2.5f, 0.15f, seed);
  const F3 centers[4] = {f3(-4.5f, 2.8f, -4.0f), f3(4.5f, 2.8f, -4.0f), f3(-4.5f, 2.8f, 3.0f), f3(4.5f, 2.8f, 3.0f)};
  for (int i = 0; i < 4; i++) {
    const int kind = i == 0 ? 0 : (i == 1 ? 1 : (int)(rng.next() & 1));
    const int m = b.material(sphereMaterial(kind, rng));
    b.mesh(b.object(m));
    addIndexed(b, sphere, centers[i]);
  }
  if (medium) {
    rg_medium md;
    std::memset(&md, 0, sizeof(md));
    for (int k = 0; k < 3; k++) { md.sigma_s[k] = 0.04f; md.sigma_a[k] = 0.01f; }
    md.g = 0.3f;
    md.density = 1.0f;
    st.media.push_back(md);
    st.globalMedium = 0;
  }
  st.camera = defaultCamera();
  st.camera.location[0] = 0.0f; st.camera.location[1] = 5.0f; st.camera.location[2] = 9.5f;
  st.camera.field_of_view = 55.0f;
}

void buildBatchJob(SceneStore& st, uint32_t seed, int tris, int emitters) {
  SceneRng rng(seed ^ 0xB47C0DEu);
  SceneBuilder b(st);
  if (emitters < 1) emitters = 1;
  buildRoom20(b, emitters, rng);
  int f = (int)std::lround(std::sqrt((double)tris / 20.0));
  if (f < 1) f = 1;
  const IndexedMesh sphere = geodesicSphere(f, rng.uniform(2.0f, 4.0f), 0.15f, seed);
  const int m = b.material(sphereMaterial((int)(rng.next() % 2), rng));
  b.mesh(b.object(m));
  addIndexed(b, sphere, f3(rng.uniform(-3, 3), 4.5f, rng.uniform(-5, 0)));
  st.camera = defaultCamera();
  st.camera.location[0] = 0.0f; st.camera.location[1] = 5.0f; st.camera.location[2] = 9.5f;
  st.camera.field_of_view = 55.0f;
}

}  // namespace

void SceneStore::finalize() {
  std::memset(&desc, 0, sizeof(desc));
  desc.num_triangles = (int32_t)triMesh.size();
  desc.positions = positions.data();
  desc.normals = normals.data();
  desc.uvs = uvs.data();
  desc.tri_mesh = triMesh.data();
  desc.num_meshes = (int32_t)meshObject.size();
  desc.mesh_object = meshObject.data();
  desc.num_objects = (int32_t)objects.size();
  desc.objects = objects.data();
  desc.num_materials = (int32_t)materials.size();
  desc.materials = materials.data();
  mediumPaths.resize(media.size());
  for (size_t i = 0; i < media.size(); i++) {
    media[i].num_path_points = (int32_t)mediumPaths[i].size();
    media[i].path_points = mediumPaths[i].empty() ? nullptr : mediumPaths[i].data();
  }
  desc.num_media = (int32_t)media.size();
  desc.media = media.data();
  desc.global_medium = globalMedium;
  desc.num_point_lights = (int32_t)pointLights.size();
  desc.point_lights = pointLights.data();
  textureDescs.clear();
  for (auto& t : textures) {
    rg_texture d;
    d.width = t.width; d.height = t.height; d.is_hdr = t.isHdr; d.rgba = t.rgba.data();
    textureDescs.push_back(d);
  }
  desc.num_textures = (int32_t)textureDescs.size();
  desc.textures = textureDescs.data();
  desc.camera = camera;
  desc.has_envmap = envmapTexture >= 0 ? 1 : 0;
  desc.envmap_texture = envmapTexture;
  desc.envmap_intensity = envmapIntensity;
  desc.envmap_rotation = envmapRotation;
  desc.envmap_cube = envCube;
  for (int f = 0; f < 6; f++) desc.envmap_cube_faces[f] = envCubeFaces[f];
}

}  // namespace rg

// HomogeneousMedium's member defaults (medium.h:80-199, PathSample medium.h:55-59).
extern "C" void rg_medium_defaults(rg_medium* m) {
  if (!m) return;
  std::memset(m, 0, sizeof(*m));
  m->density = 1.0f;
  m->cone_axis[2] = -1.0f;
  m->cone_length = 1.0f;
  m->cone_radius = 0.3f;
  const float inner[3] = {0.6f, 0.7f, 1.0f}, outer[3] = {1.0f, 0.4f, 0.05f};
  const float pInner[3] = {0.6f, 0.7f, 1.0f}, pOuter[3] = {0.3f, 0.4f, 0.6f};
  for (int k = 0; k < 3; k++) {
    m->cone_inner[k] = inner[k];
    m->cone_outer[k] = outer[k];
    m->path_inner[k] = pInner[k];
    m->path_outer[k] = pOuter[k];
  }
  m->cone_intensity = 50.0f;
  m->cone_emission_samples = 4;
  m->cone_peak_axial = 0.15f;
  m->cone_peak_sharpness = 5.0f;
  m->path_intensity = 1.0f;
  m->path_falloff_power = 2.0f;
  m->path_emission_samples = 6;
  m->noise_frequency = 1.0f;
  m->noise_octaves = 4;
  m->noise_gain = 0.5f;
  m->noise_lacunarity = 2.0f;
  m->noise_amplitude = 1.0f;
  m->ior_amplitude = 0.005f;
  m->ior_frequency = 4.0f;
  m->ior_octaves = 3;
  m->ior_gain = 0.5f;
  m->ior_lacunarity = 2.0f;
  m->ior_march_steps = 16;
}

namespace rg {

rg_status buildBuiltinScene(int kind, uint32_t seed, const int32_t* ip, int nip, SceneStore** out) {
  SceneStore* st = new (std::nothrow) SceneStore();
  if (!st) return RG_ERR_OUT_OF_MEMORY;
  switch (kind) {
    case 1: buildCubeRoom(*st); break;
    case 2: buildHeavy(*st, seed, nip > 0 ? ip[0] : 1003520, false); break;
    case 3: buildHeavy(*st, seed, nip > 0 ? ip[0] : 1003520, true); break;
    case 4: buildBatchJob(*st, seed, nip > 0 ? ip[0] : 10000, nip > 1 ? ip[1] : 4); break;
    default: delete st; return RG_ERR_INVALID_ARGUMENT;
  }
  st->finalize();
  *out = st;
  return RG_OK;
}

}  // namespace rg
