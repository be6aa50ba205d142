// rg_json.cpp - the reference scene JSON schema -> flattened scene description.
//
// Reference: SceneJsonLoader (src/raygen/sceneloader.cpp:101-883), mesh
// primitives (src/raygen/polygons.cpp:13-288) and the transform stack of
// transformObject (src/raygen/rayrenderer.cpp:237-363).
//  * JSONC: '//' and '/* */' comments, trailing commas and bare identifier
//    keys tolerated; containers still open at the end of input are closed
//    there (one sample scene lacks its final brace).
//  * Root keys: mainCamera, _materials, envmap (equirectangular Radiance
//    .hdr / .pfm, or a cubemap directory of six faces), medium (global), and
//    child objects.
//  * Object keys: location, angle (degrees), scale, mesh (path | [paths] |
//    {type: plane|cube|sphere|cone, ...}), mat (name | object), visible,
//    medium (interior), children.  Keys are applied in file order.  Objects
//    are flattened depth first, each object's meshes before its children; a
//    mesh-less emissive object becomes a point light.
//  * Materials: color ([r,g,b] | "#rgb" | "#rrggbb[aa]"), emission, diffuse,
//    glossy, roughness, transparency, refraction, refractionRatio,
//    chromaDispersion, metallic, anisotropy, anisoRotation, spotRange,
//    texTiling, tex (Radiance .hdr, PFM, JPEG or PNG; one texture per path).
//  * Transforms: world = parent * T(location) * R(angle) * S(scale) with
//    R = Ry(y) Rx(x) Rz(z), active right-handed rotations (the single-axis
//    rotations of the sample scenes, e.g. cubeRoom's walls, face inward).
//  * Meshes: primitives as polygons.cpp; Wavefront .obj (v / vn / vt / f with
//    polygon fans, 'o'/'g' objects, .mtl Kd / Tf) and the binary .mesh
//    format.  .toba bundles (tob:// / sob:// URIs, "_bundle") are reported
//    as unsupported.
//  * The multi-axis rotation order and the colour packing come from the
//    graphics-module submodule, which the reference tree does not vendor.
#include <cctype>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "rg_host.h"

namespace rg {

namespace {

// ------------------------------------------------------------------ JSON ----
struct JVal {
  enum Type { Null, Bool, Num, Str, Arr, Obj } type = Null;
  bool b = false;
  double n = 0;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;  // insertion order
  const JVal* get(const char* k) const {
    for (auto& p : obj)
      if (p.first == k) return &p.second;
    return nullptr;
  }
  bool num(const char* k, float& out) const {
    const JVal* v = get(k);
    if (v && v->type == Num) {
      out = (float)v->n;
      return true;
    }
    return false;
  }
};

struct Parser {
  const std::string& t;
  size_t i = 0;
  std::string err;
  explicit Parser(const std::string& s) : t(s) {}
  void ws() {
    for (;;) {
      while (i < t.size() && std::isspace((unsigned char)t[i])) i++;
      if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '/') {
        while (i < t.size() && t[i] != '\n') i++;
      } else if (i + 1 < t.size() && t[i] == '/' && t[i + 1] == '*') {
        i += 2;
        while (i + 1 < t.size() && !(t[i] == '*' && t[i + 1] == '/')) i++;
        i += 2;
      } else {
        return;
      }
    }
  }
  bool fail(const std::string& m) {
    if (err.empty()) err = m + " at offset " + std::to_string(i);
    return false;
  }
  bool str(std::string& out) {
    if (t[i] != '"') return fail("expected string");
    i++;
    while (i < t.size() && t[i] != '"') {
      if (t[i] == '\\' && i + 1 < t.size()) {
        i++;
        const char c = t[i];
        out += c == 'n' ? '\n' : c == 't' ? '\t' : c;
      } else {
        out += t[i];
      }
      i++;
    }
    if (i >= t.size()) return fail("unterminated string");
    i++;
    return true;
  }
  // Object keys: a string, or a bare identifier as in JavaScript object
  // literals (the sample scenes use both).
  bool key(std::string& out) {
    if (t[i] == '"') return str(out);
    while (i < t.size() && (std::isalnum((unsigned char)t[i]) || t[i] == '_' || t[i] == '$')) out += t[i++];
    if (out.empty()) return fail("expected key");
    return true;
  }
  bool val(JVal& v) {
    ws();
    if (i >= t.size()) return fail("unexpected end");
    const char c = t[i];
    if (c == '{') {
      v.type = JVal::Obj;
      i++;
      for (;;) {
        ws();
        if (i >= t.size()) return true;  // unterminated object closed at end of input
        if (t[i] == '}') { i++; return true; }
        std::string k;
        if (!key(k)) return false;
        ws();
        if (i >= t.size() || t[i] != ':') return fail("expected ':'");
        i++;
        JVal e;
        if (!val(e)) return false;
        v.obj.emplace_back(std::move(k), std::move(e));
        ws();
        if (i >= t.size()) return true;
        if (t[i] == ',') { i++; continue; }
        if (i < t.size() && t[i] == '}') { i++; return true; }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      v.type = JVal::Arr;
      i++;
      for (;;) {
        ws();
        if (i >= t.size()) return true;  // unterminated array closed at end of input
        if (t[i] == ']') { i++; return true; }
        JVal e;
        if (!val(e)) return false;
        v.arr.push_back(std::move(e));
        ws();
        if (i >= t.size()) return true;
        if (t[i] == ',') { i++; continue; }
        if (i < t.size() && t[i] == ']') { i++; return true; }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') { v.type = JVal::Str; return str(v.s); }
    if (t.compare(i, 4, "true") == 0) { v.type = JVal::Bool; v.b = true; i += 4; return true; }
    if (t.compare(i, 5, "false") == 0) { v.type = JVal::Bool; v.b = false; i += 5; return true; }
    if (t.compare(i, 4, "null") == 0) { v.type = JVal::Null; i += 4; return true; }
    char* end = nullptr;
    v.n = std::strtod(t.c_str() + i, &end);
    if (end == t.c_str() + i) return fail("unexpected character");
    v.type = JVal::Num;
    i = (size_t)(end - t.c_str());
    return true;
  }
};

// ------------------------------------------------------------------ math ----
struct M4 {
  double m[4][4];  // column-vector convention: p' = M p
  static M4 ident() {
    M4 r;
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) r.m[a][b] = a == b ? 1 : 0;
    return r;
  }
  M4 operator*(const M4& o) const {
    M4 r;
    for (int a = 0; a < 4; a++)
      for (int b = 0; b < 4; b++) {
        r.m[a][b] = 0;
        for (int k = 0; k < 4; k++) r.m[a][b] += m[a][k] * o.m[k][b];
      }
    return r;
  }
};

M4 trs(const float loc[3], const float ang[3], const float scl[3]) {
  const double d2r = 3.14159265358979323846 / 180.0;
  const double ax = ang[0] * d2r, ay = ang[1] * d2r, az = ang[2] * d2r;
  M4 T = M4::ident(), Rx = M4::ident(), Ry = M4::ident(), Rz = M4::ident(), S = M4::ident();
  T.m[0][3] = loc[0]; T.m[1][3] = loc[1]; T.m[2][3] = loc[2];
  Rx.m[1][1] = std::cos(ax); Rx.m[1][2] = -std::sin(ax); Rx.m[2][1] = std::sin(ax); Rx.m[2][2] = std::cos(ax);
  Ry.m[0][0] = std::cos(ay); Ry.m[0][2] = std::sin(ay); Ry.m[2][0] = -std::sin(ay); Ry.m[2][2] = std::cos(ay);
  Rz.m[0][0] = std::cos(az); Rz.m[0][1] = -std::sin(az); Rz.m[1][0] = std::sin(az); Rz.m[1][1] = std::cos(az);
  S.m[0][0] = scl[0]; S.m[1][1] = scl[1]; S.m[2][2] = scl[2];
  return T * Ry * Rx * Rz * S;
}

// inverse-transpose of the upper 3x3 (for normals)
void normalMatrix(const M4& M, double N[3][3]) {
  const double a = M.m[0][0], b = M.m[0][1], c = M.m[0][2], d = M.m[1][0], e = M.m[1][1], f = M.m[1][2], g = M.m[2][0],
               h = M.m[2][1], k = M.m[2][2];
  const double A = e * k - f * h, B = -(d * k - f * g), Cc = d * h - e * g;
  const double D = -(b * k - c * h), E = a * k - c * g, F = -(a * h - b * g);
  const double G = b * f - c * e, H = -(a * f - c * d), K = a * e - b * d;
  double det = a * A + b * B + c * Cc;
  if (std::fabs(det) < 1e-30) det = 1e-30;
  // inverse = adj^T / det ; transpose(inverse) = adj / det (cofactor matrix)
  N[0][0] = A / det; N[0][1] = B / det; N[0][2] = Cc / det;
  N[1][0] = D / det; N[1][1] = E / det; N[1][2] = F / det;
  N[2][0] = G / det; N[2][1] = H / det; N[2][2] = K / det;
}

struct Vtx {
  float p[3], n[3], uv[2];
};
using MeshTris = std::vector<Vtx>;  // 3 per triangle

// ------------------------------------------------------------ primitives ----
// PlaneMesh::create (polygons.cpp:29-59), 1x1 in XZ, normal +Y
MeshTris planeMesh() {
  const float h = 0.5f;
  const float P[6][3] = {{-h, 0, -h}, {-h, 0, h}, {h, 0, -h}, {-h, 0, h}, {h, 0, h}, {h, 0, -h}};
  const float T[6][2] = {{0, 0}, {0, 1}, {1, 0}, {0, 1}, {1, 1}, {1, 0}};
  MeshTris m(6);
  for (int i = 0; i < 6; i++) {
    m[i] = Vtx{{P[i][0], P[i][1], P[i][2]}, {0, 1, 0}, {T[i][0], T[i][1]}};
  }
  return m;
}

// CubeMesh (polygons.cpp:61-130)
MeshTris cubeMesh() {
  const float P[8][3] = {{-0.5f, -0.5f, -0.5f}, {0.5f, -0.5f, -0.5f}, {0.5f, 0.5f, -0.5f}, {-0.5f, 0.5f, -0.5f},
                         {-0.5f, -0.5f, 0.5f},  {0.5f, -0.5f, 0.5f},  {0.5f, 0.5f, 0.5f},  {-0.5f, 0.5f, 0.5f}};
  const int F[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 4, 7, 3}, {1, 5, 6, 2}, {3, 2, 6, 7}, {0, 1, 5, 4}};
  const float N[6][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
  const float T[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
  MeshTris m;
  for (int f = 0; f < 6; f++) {
    const int order[6] = {0, 1, 2, 0, 2, 3};
    for (int k : order) {
      const float* p = P[F[f][k]];
      m.push_back(Vtx{{p[0], p[1], p[2]}, {N[f][0], N[f][1], N[f][2]}, {T[k][0], T[k][1]}});
    }
  }
  return m;
}

// SphereMesh (polygons.cpp:132-180), indexed stacks x slices
MeshTris sphereMesh(float radius, int stacks, int slices) {
  std::vector<Vtx> v;
  for (int i = 0; i <= stacks; ++i) {
    const float fv = (float)i / stacks, phi = fv * 3.14159265358979f;
    for (int j = 0; j <= slices; ++j) {
      const float u = (float)j / slices, th = u * 2.0f * 3.14159265358979f;
      const float x = std::sin(phi) * std::cos(th), y = std::cos(phi), z = std::sin(phi) * std::sin(th);
      v.push_back(Vtx{{x * radius, y * radius, z * radius}, {x, y, z}, {u, fv}});
    }
  }
  MeshTris m;
  for (int i = 0; i < stacks; ++i)
    for (int j = 0; j < slices; ++j) {
      const int cur = i * (slices + 1) + j, nxt = (i + 1) * (slices + 1) + j;
      const int idx[6] = {cur, nxt, cur + 1, cur + 1, nxt, nxt + 1};
      for (int k : idx) m.push_back(v[k]);
    }
  return m;
}

// ConeMesh (polygons.cpp:182-288)
MeshTris coneMesh(float r0, float r1, int slices) {
  if (slices < 3) slices = 3;
  const float z0 = -0.5f, z1 = 0.5f, hgt = 1.0f;
  const float slope = (r0 - r1) / hgt, invLen = 1.0f / std::sqrt(1.0f + slope * slope);
  const float rn = invLen, an = slope * invLen;
  const float tw = 2.0f * 3.14159265358979f;
  MeshTris m;
  for (int i = 0; i < slices; ++i) {
    const float t0 = (float)i / slices, t1 = (float)(i + 1) / slices;
    const float c0 = std::cos(t0 * tw), s0 = std::sin(t0 * tw), c1 = std::cos(t1 * tw), s1 = std::sin(t1 * tw);
    const Vtx S0{{c0 * r0, s0 * r0, z0}, {c0 * rn, s0 * rn, an}, {t0, 0}};
    const Vtx S1{{c1 * r0, s1 * r0, z0}, {c1 * rn, s1 * rn, an}, {t1, 0}};
    const Vtx E0{{c0 * r1, s0 * r1, z1}, {c0 * rn, s0 * rn, an}, {t0, 1}};
    const Vtx E1{{c1 * r1, s1 * r1, z1}, {c1 * rn, s1 * rn, an}, {t1, 1}};
    m.push_back(S0); m.push_back(E0); m.push_back(E1);
    m.push_back(S0); m.push_back(E1); m.push_back(S1);
  }
  if (r0 > 0.0f)
    for (int i = 0; i < slices; ++i) {
      const float a0 = (float)i / slices * tw, a1 = (float)(i + 1) / slices * tw;
      m.push_back(Vtx{{0, 0, z0}, {0, 0, -1}, {0.5f, 0.5f}});
      m.push_back(Vtx{{std::cos(a1) * r0, std::sin(a1) * r0, z0}, {0, 0, -1}, {0.5f + 0.5f * std::cos(a1), 0.5f + 0.5f * std::sin(a1)}});
      m.push_back(Vtx{{std::cos(a0) * r0, std::sin(a0) * r0, z0}, {0, 0, -1}, {0.5f + 0.5f * std::cos(a0), 0.5f + 0.5f * std::sin(a0)}});
    }
  if (r1 > 0.0f)
    for (int i = 0; i < slices; ++i) {
      const float a0 = (float)i / slices * tw, a1 = (float)(i + 1) / slices * tw;
      m.push_back(Vtx{{0, 0, z1}, {0, 0, 1}, {0.5f, 0.5f}});
      m.push_back(Vtx{{std::cos(a0) * r1, std::sin(a0) * r1, z1}, {0, 0, 1}, {0.5f + 0.5f * std::cos(a0), 0.5f + 0.5f * std::sin(a0)}});
      m.push_back(Vtx{{std::cos(a1) * r1, std::sin(a1) * r1, z1}, {0, 0, 1}, {0.5f + 0.5f * std::cos(a1), 0.5f + 0.5f * std::sin(a1)}});
    }
  return m;
}

// ------------------------------------------------------------------- OBJ ----
// ObjFileReader (objreader.cpp:93-460): an object starts at every 'o' and at
// every 'g' except "g default"; 'usemtl' names the object's material (the last
// one wins, objects are not split); faces are fan-triangulated (v0, vi, vi+1);
// 'vt' v is flipped (1 - v); a header comment naming "3ds Max" or
// "uses millimeters as units" scales vertices by 0.01.  Faces without normals
// get the geometric face normal.
struct ObjGroup {
  std::string name, material;
  MeshTris tris;
};

// ObjMaterial after readMaterialLibrary (objreader.cpp:500-560): 'newmtl'
// resets diffuse to 0 but not the transparency, which carries over from the
// previous material; Tf gives transparency = 1 - mean(Tf); d / Tr are ignored.
struct ObjMtl {
  float kd[3] = {0.0f, 0.0f, 0.0f};
  float transparency = 0.0f;
};

void readMtl(const std::string& path, std::map<std::string, ObjMtl>& out) {
  std::ifstream f(path);
  std::string line, cur;
  ObjMtl m;
  bool has = false;
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    std::istringstream ss(line);
    std::string k;
    ss >> k;
    if (k == "newmtl") {
      if (has) out[cur] = m;
      cur = line.size() > 7 ? line.substr(7) : "";
      m.kd[0] = m.kd[1] = m.kd[2] = 0.0f;
      has = true;
    } else if (k == "Kd") {
      ss >> m.kd[0] >> m.kd[1] >> m.kd[2];
    } else if (k == "Tf") {
      float t[3] = {1, 1, 1};
      ss >> t[0] >> t[1] >> t[2];
      m.transparency = 1.0f - (t[0] + t[1] + t[2]) / 3.0f;
    }
  }
  if (has) out[cur] = m;
}

bool readObj(const std::string& path, std::vector<ObjGroup>& groups, std::map<std::string, ObjMtl>& mtls,
             std::string& err) {
  std::ifstream f(path);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  const std::string dir = path.find_last_of('/') == std::string::npos ? "" : path.substr(0, path.find_last_of('/') + 1);
  std::vector<float> P, N, T;
  groups.emplace_back();
  std::string line;
  bool headComments = true, autoScale = false;
  auto rest = [](const std::string& l, size_t n) { return l.size() > n ? l.substr(n) : std::string(); };
  auto startObject = [&](const std::string& name) {
    if (groups.back().tris.empty()) groups.back() = ObjGroup();
    else groups.emplace_back();
    groups.back().name = name;
  };
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (headComments && !line.empty() && line[0] == '#') {
      if (line.find("3ds Max") != std::string::npos || line.find("uses millimeters as units") != std::string::npos) {
        autoScale = true;
        headComments = false;
      }
      continue;
    }
    headComments = false;
    std::istringstream ss(line);
    std::string k;
    ss >> k;
    if (k == "v") {
      float x = 0, y = 0, z = 0;
      ss >> x >> y >> z;
      if (autoScale) { x *= 0.01f; y *= 0.01f; z *= 0.01f; }
      P.insert(P.end(), {x, y, z});
    } else if (k == "vn") {
      float x = 0, y = 0, z = 0;
      ss >> x >> y >> z;
      N.insert(N.end(), {x, y, z});
    } else if (k == "vt") {
      float u = 0, v = 0;
      ss >> u >> v;
      T.insert(T.end(), {u, 1.0f - v});
    } else if (k == "o") {
      startObject(rest(line, 2));
    } else if (k == "g") {
      const std::string nm = rest(line, 2);
      if (nm == "default") continue;
      std::istringstream gs(nm);
      std::string part, joined;
      while (gs >> part) joined += (joined.empty() ? "" : "_") + part;
      startObject(joined);
    } else if (k == "usemtl") {
      groups.back().material = rest(line, 7);
    } else if (k == "mtllib") {
      readMtl(dir + rest(line, 7), mtls);
    } else if (k == "f") {
      std::vector<Vtx> poly;
      bool faceHasNormal = true;
      std::string tok;
      while (ss >> tok) {
        int idx[3] = {0, 0, 0}, part = 0;
        std::string cur;
        for (size_t c = 0; c <= tok.size(); c++) {
          if (c == tok.size() || tok[c] == '/') {
            if (!cur.empty() && part < 3) idx[part] = std::atoi(cur.c_str());
            cur.clear();
            part++;
          } else {
            cur += tok[c];
          }
        }
        const int nv = (int)P.size() / 3, nt = (int)T.size() / 2, nn = (int)N.size() / 3;
        if (idx[0] < 0) idx[0] += nv + 1;
        if (idx[1] < 0) idx[1] += nt + 1;
        if (idx[2] < 0) idx[2] += nn + 1;
        if (idx[0] <= 0 || idx[0] > nv) {
          err = "bad vertex index in " + path;
          return false;
        }
        Vtx v{};
        for (int a = 0; a < 3; a++) v.p[a] = P[(size_t)(idx[0] - 1) * 3 + a];
        if (idx[1] > 0 && idx[1] <= nt) { v.uv[0] = T[(size_t)(idx[1] - 1) * 2]; v.uv[1] = T[(size_t)(idx[1] - 1) * 2 + 1]; }
        if (idx[2] > 0 && idx[2] <= nn) {
          for (int a = 0; a < 3; a++) v.n[a] = N[(size_t)(idx[2] - 1) * 3 + a];
        } else {
          faceHasNormal = false;
        }
        poly.push_back(v);
      }
      if (poly.size() < 3) {
        err = "face with fewer than 3 vertices in " + path;
        return false;
      }
      for (size_t q = 1; q + 1 < poly.size(); q++) {
        Vtx a = poly[0], b = poly[q], c = poly[q + 1];
        if (!faceHasNormal) {
          const float e1[3] = {b.p[0] - a.p[0], b.p[1] - a.p[1], b.p[2] - a.p[2]};
          const float e2[3] = {c.p[0] - a.p[0], c.p[1] - a.p[1], c.p[2] - a.p[2]};
          float fn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
          const float l = std::sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
          if (l > 0) { fn[0] /= l; fn[1] /= l; fn[2] /= l; }
          for (Vtx* v : {&a, &b, &c}) std::memcpy(v->n, fn, sizeof(fn));
        }
        groups.back().tris.push_back(a);
        groups.back().tris.push_back(b);
        groups.back().tris.push_back(c);
      }
    }
  }
  return true;
}

// ------------------------------------------------------------------ .mesh ---
// Binary mesh file, MeshLoader::load (meshloader.cpp:25-130, meshloader.h):
//   header  u32 tag 'mesh' (0x6873656d), u16 ver, u16 flags, u32 length
//   ver < 0x0102: meta {vertexCount, normalCount, uvCount, texcoordCount,
//                 indexCount}; normals iff normalCount > 0, texcoords iff
//                 texcoordCount > 0, tangents iff flags & 0x2
//   ver >= 0x0102: meta {vertexCount, uvCount, indexCount, ...}; normals iff
//                 flags & 0x2, texcoords iff & 0x4, tangents iff & 0x10,
//                 colours iff & 0x20 (ver >= 0x0103)
//   vertex data starts at byte `length`.  Files without the tag are the
//   0x0100 layout {vertexCount, normalCount, texcoordCount} followed by
//   vertices only (the Mesh flags keep their false defaults).
//   data: vec3 vertices[vc]; vec3 normals[vc]; vec2 uv[uvCount][vc];
//   vec3 tangents[vc], bitangents[vc]; vec3 colours[vc]; u32 indexes[ic].
// Triangles: ic > 0 ? (idx[3k], idx[3k+1], idx[3k+2]) : (3k, 3k+1, 3k+2)
// (Mesh::getVertex, mesh.cpp:93-110).  A mesh without normals gets the
// geometric face normal.
bool readMeshFile(const std::string& path, MeshTris& out, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::vector<unsigned char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
  auto u32 = [&](size_t o) { uint32_t v; std::memcpy(&v, &b[o], 4); return v; };
  auto u16 = [&](size_t o) { uint16_t v; std::memcpy(&v, &b[o], 2); return v; };
  auto bad = [&](const char* why) {
    err = std::string("malformed .mesh file (") + why + "): " + path;
    return false;
  };
  if (b.size() < 12) return bad("short header");
  uint64_t vc = 0, uvCount = 0, ic = 0;
  bool hasN = false, hasT = false, hasTan = false, hasC = false;
  size_t pos;
  if (u32(0) == 0x6873656du) {
    const uint16_t ver = u16(4), flags = u16(6);
    const uint32_t length = u32(8);
    if (ver < 0x0102) {
      if (b.size() < 32) return bad("short meta");
      vc = u32(12);
      hasN = u32(16) > 0;
      uvCount = u32(20);
      hasT = u32(24) > 0;
      ic = u32(28);
      hasTan = (flags & 0x2) != 0;
    } else {
      if (b.size() < 24) return bad("short meta");
      vc = u32(12);
      uvCount = u32(16);
      ic = u32(20);
      hasN = (flags & 0x2) != 0;
      hasT = (flags & 0x4) != 0;
      hasTan = (flags & 0x10) != 0;
      hasC = ver >= 0x0103 && (flags & 0x20) != 0;
    }
    pos = length;
  } else {
    vc = u32(0);
    uvCount = 1;
    pos = 12;
  }
  if (!hasT) uvCount = 0;
  const uint64_t need = vc * 12 + (hasN ? vc * 12 : 0) + vc * 8 * uvCount + (hasTan ? vc * 24 : 0) +
                        (hasC ? vc * 12 : 0) + ic * 4;
  if (pos > b.size() || need > b.size() - pos) return bad("truncated data");
  const float* V = reinterpret_cast<const float*>(&b[pos]);
  std::vector<float> vbuf(V, V + vc * 3);  // aligned copies
  size_t o = pos + vc * 12;
  std::vector<float> nbuf, tbuf;
  if (hasN) {
    nbuf.resize(vc * 3);
    std::memcpy(nbuf.data(), &b[o], vc * 12);
    o += vc * 12;
  }
  if (uvCount > 0) {
    tbuf.resize(vc * 2);  // first uv set
    std::memcpy(tbuf.data(), &b[o], vc * 8);
    o += vc * 8 * uvCount;
  }
  if (hasTan) o += vc * 24;
  if (hasC) o += vc * 12;
  std::vector<uint32_t> idx(ic);
  if (ic) std::memcpy(idx.data(), &b[o], ic * 4);
  const uint64_t nt = ic > 0 ? ic / 3 : vc / 3;
  for (uint64_t k = 0; k < nt; k++) {
    uint32_t id[3];
    for (int q = 0; q < 3; q++) {
      id[q] = ic > 0 ? idx[k * 3 + q] : (uint32_t)(k * 3 + q);
      if (id[q] >= vc) return bad("index out of range");
    }
    Vtx t[3];
    for (int q = 0; q < 3; q++) {
      std::memset(&t[q], 0, sizeof(Vtx));
      std::memcpy(t[q].p, &vbuf[(size_t)id[q] * 3], 12);
      if (hasN) std::memcpy(t[q].n, &nbuf[(size_t)id[q] * 3], 12);
      if (uvCount > 0) std::memcpy(t[q].uv, &tbuf[(size_t)id[q] * 2], 8);
    }
    if (!hasN) {
      const float e1[3] = {t[1].p[0] - t[0].p[0], t[1].p[1] - t[0].p[1], t[1].p[2] - t[0].p[2]};
      const float e2[3] = {t[2].p[0] - t[0].p[0], t[2].p[1] - t[0].p[1], t[2].p[2] - t[0].p[2]};
      float fn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
      const float l = std::sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
      if (l > 0) { fn[0] /= l; fn[1] /= l; fn[2] /= l; }
      for (auto& v : t) std::memcpy(v.n, fn, sizeof(fn));
    }
    for (auto& v : t) out.push_back(v);
  }
  return true;
}

// ---------------------------------------------------------------- loader ----
rg_material defaultMat() {  // Material member defaults, material.h:27-52
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

// tryParseColorString (sceneloader.cpp:167-199).  The 6/8-digit forms are
// 0xRRGGBB[AA].  The 3/4-digit forms take the reference's expression
// literally: the hex value of the 3 (4) digits times 2, read as a packed
// 0xRRGGBB (0xRRGGBBAA) word by tocolor3f (tocolor4f) -- so "#fff" is not
// white.  The packing of tocolor3f/tocolor4f comes from the graphics-module
// submodule, which is not part of the reference tree; byte order assumed
// R high.  Alpha is not used by the renderer.
bool parseColorString(const std::string& s0, float c[3]) {
  std::string s = s0;
  if (s.size() < 3) return false;
  if (s[0] == '#' && (s.size() == 4 || s.size() == 5 || s.size() == 7 || s.size() == 9)) s = s.substr(1);
  auto hex = [](const std::string& h) {
    uint64_t v = 0;
    for (char ch : h) {
      const int d = std::isdigit((unsigned char)ch) ? ch - '0'
                    : (std::tolower((unsigned char)ch) >= 'a' && std::tolower((unsigned char)ch) <= 'f')
                        ? std::tolower((unsigned char)ch) - 'a' + 10
                        : 0;
      v = v * 16 + (uint64_t)d;
    }
    return v;
  };
  uint64_t v;
  bool rgba;
  switch (s.size()) {
    case 3: v = hex(s) * 2; rgba = false; break;
    case 4: v = hex(s) * 2; rgba = true; break;
    case 6: v = hex(s); rgba = false; break;
    case 8: v = hex(s); rgba = true; break;
    default: return false;
  }
  const int shift = rgba ? 8 : 0;
  for (int k = 0; k < 3; k++) c[k] = (float)((v >> (shift + 8 * (2 - k))) & 0xff) / 255.0f;
  return true;
}

// tryReadVec3Property: an [x,y,z] array or an {x,y,z} object; absent keys
// leave the value untouched.
bool readVec3(const JVal* v, float out[3]) {
  if (!v) return false;
  if (v->type == JVal::Arr) {
    for (size_t k = 0; k < 3 && k < v->arr.size(); k++)
      if (v->arr[k].type == JVal::Num) out[k] = (float)v->arr[k].n;
    return true;
  }
  if (v->type == JVal::Obj) {
    v->num("x", out[0]);
    v->num("y", out[1]);
    v->num("z", out[2]);
    return true;
  }
  return false;
}

// readMaterial (sceneloader.cpp:101-165).  `texture` resolves a 'tex' path
// to a texture index (-1: the material keeps its flat colour).
void readMaterial(const JVal& j, rg_material& m, const std::function<int(const std::string&)>& texture) {
  if (const JVal* t = j.get("tex"))
    if (t->type == JVal::Str && !t->s.empty()) m.texture = texture(t->s);
  if (const JVal* t = j.get("texTiling")) {
    if (t->type == JVal::Arr && t->arr.size() >= 2) {
      m.tex_tiling[0] = (float)t->arr[0].n;
      m.tex_tiling[1] = (float)t->arr[1].n;
    } else if (t->type == JVal::Obj) {
      t->num("x", m.tex_tiling[0]);
      t->num("y", m.tex_tiling[1]);
    }
  }
  j.num("emission", m.emission);
  j.num("diffuse", m.diffuse);
  j.num("glossy", m.glossy);
  j.num("roughness", m.roughness);
  j.num("transparency", m.transparency);
  j.num("refraction", m.refraction);
  j.num("refractionRatio", m.refraction_ratio);
  j.num("chromaDispersion", m.chroma_dispersion);
  j.num("metallic", m.metallic);
  j.num("anisotropy", m.anisotropy);
  j.num("anisoRotation", m.aniso_rotation);
  j.num("spotRange", m.spot_range);
  if (const JVal* c = j.get("color")) {
    if (c->type == JVal::Str) parseColorString(c->s, m.color);
    else if (c->type == JVal::Arr) readVec3(c, m.color);
  }
}

// A medium as read from JSON; the owning object's transform is applied when
// the object is flattened (coneFollowObject / pathFollowObject).
struct MediumSpec {
  rg_medium m;
  std::vector<rg_medium_path_point> pts;
  bool coneFollow = false, pathFollow = false;
};

bool readBool(const JVal& j, const char* k, bool& out) {
  const JVal* v = j.get(k);
  if (!v || v->type != JVal::Bool) return false;
  out = v->b;
  return true;
}

bool readInt(const JVal& j, const char* k, int32_t& out) {
  const JVal* v = j.get(k);
  if (!v || v->type != JVal::Num) return false;
  out = (int32_t)v->n;
  return true;
}

bool isString(const JVal& j, const char* k, const char* value) {
  const JVal* v = j.get(k);
  return v && v->type == JVal::Str && v->s == value;
}

// HomogeneousMedium::isActive after prepare() (medium.h:226-234, medium.cpp:18-57).
bool mediumActive(const rg_medium& m, size_t numPathPoints) {
  const float d = std::fmax(0.0f, m.density);
  float st[3], se[3];
  for (int k = 0; k < 3; k++) {
    st[k] = m.sigma_a[k] * d + m.sigma_s[k] * d;
    se[k] = m.sigma_e[k] * d;
  }
  const float hero = (st[0] + st[1] + st[2]) * (1.0f / 3.0f);
  if (hero > 0.0f) return true;
  if (m.emission_mode == RG_EMISSION_CONE && m.cone_intensity > 0.0f) return true;
  if (m.emission_mode == RG_EMISSION_PATH && m.path_intensity > 0.0f && numPathPoints >= 2) return true;
  if (m.heat_haze && m.ior_amplitude > 0.0f) return true;
  return se[0] != 0.0f || se[1] != 0.0f || se[2] != 0.0f;
}

// An emissive volume registered for volume-light NEE (rayrenderer.cpp:193-203).
bool emissiveVolume(const rg_medium& m) {
  if (m.emission_mode == RG_EMISSION_CONE) return m.cone_intensity > 0.0f;
  if (m.emission_mode != RG_EMISSION_CONSTANT) return false;
  const float d = std::fmax(0.0f, m.density);
  return m.sigma_e[0] * d != 0.0f || m.sigma_e[1] * d != 0.0f || m.sigma_e[2] * d != 0.0f;
}

// readMedium (sceneloader.cpp:202-334): every key over the member defaults;
// false when the result is inactive, which the reference drops (the object
// or scene keeps what it had).  The JSON key of sigma_e is "emission".
bool readMedium(const JVal& j, MediumSpec& sp) {
  rg_medium& md = sp.m;
  rg_medium_defaults(&md);
  sp.pts.clear();
  readVec3(j.get("sigma_a"), md.sigma_a);
  readVec3(j.get("sigma_s"), md.sigma_s);
  readVec3(j.get("emission"), md.sigma_e);
  j.num("g", md.g);
  j.num("density", md.density);
  if (isString(j, "emissionMode", "cone")) md.emission_mode = RG_EMISSION_CONE;
  else if (isString(j, "emissionMode", "path")) md.emission_mode = RG_EMISSION_PATH;
  readVec3(j.get("coneAxis"), md.cone_axis);
  readVec3(j.get("coneOrigin"), md.cone_origin);
  j.num("coneLength", md.cone_length);
  j.num("coneRadius", md.cone_radius);
  readVec3(j.get("coneInner"), md.cone_inner);
  readVec3(j.get("coneOuter"), md.cone_outer);
  j.num("coneIntensity", md.cone_intensity);
  j.num("conePeakAxial", md.cone_peak_axial);
  j.num("conePeakSharpness", md.cone_peak_sharpness);
  readInt(j, "coneEmissionSamples", md.cone_emission_samples);
  readBool(j, "coneFollowObject", sp.coneFollow);
  readVec3(j.get("pathInner"), md.path_inner);
  readVec3(j.get("pathOuter"), md.path_outer);
  j.num("pathIntensity", md.path_intensity);
  j.num("pathFalloffPower", md.path_falloff_power);
  readInt(j, "pathEmissionSamples", md.path_emission_samples);
  readBool(j, "pathFollowObject", sp.pathFollow);
  if (const JVal* arr = j.get("pathPoints")) {
    if (arr->type == JVal::Arr)
      for (const JVal& el : arr->arr) {
        if (el.type != JVal::Obj) continue;
        rg_medium_path_point q{{0.0f, 0.0f, 0.0f}, 0.1f, 0.0f};
        readVec3(el.get("p"), q.p);
        el.num("radius", q.radius);
        el.num("t", q.t);
        sp.pts.push_back(q);
      }
  }
  if (isString(j, "densityField", "fbm")) md.density_field = RG_DENSITY_FBM;
  j.num("noiseFrequency", md.noise_frequency);
  readInt(j, "noiseOctaves", md.noise_octaves);
  j.num("noiseGain", md.noise_gain);
  j.num("noiseLacunarity", md.noise_lacunarity);
  j.num("noiseAmplitude", md.noise_amplitude);
  j.num("noiseBias", md.noise_bias);
  readVec3(j.get("noiseOffset"), md.noise_offset);
  bool haze = false;
  if (readBool(j, "heatHaze", haze)) md.heat_haze = haze ? 1 : 0;
  j.num("iorAmplitude", md.ior_amplitude);
  j.num("iorFrequency", md.ior_frequency);
  readInt(j, "iorOctaves", md.ior_octaves);
  j.num("iorGain", md.ior_gain);
  j.num("iorLacunarity", md.ior_lacunarity);
  readInt(j, "iorMarchSteps", md.ior_march_steps);
  readVec3(j.get("iorOffset"), md.ior_offset);
  j.num("iorFalloff", md.ior_falloff);
  return mediumActive(md, sp.pts.size());
}

struct Loader {
  SceneStore& st;
  std::string baseDir;
  // SceneResourcePool::getTexture (scene.cpp:597-681): one texture per path,
  // relative paths from the scene's directory (transformPath,
  // sceneloader.cpp:50-62); a file that cannot be read or decoded gives no
  // texture, and bundle paths (sob:// / tob://) are not read.
  std::map<std::string, int> texPool;
  int texture(const std::string& rel) {
    if (rel.rfind("sob://", 0) == 0 || rel.rfind("tob://", 0) == 0) return -1;
    const std::string path = (rel[0] == '/' || rel[0] == '\\') ? rel : baseDir + rel;
    const auto it = texPool.find(path);
    if (it != texPool.end()) return it->second;
    TextureStore t;
    std::string e;
    int idx = -1;
    if (readImageFile(path, t, e) && t.width > 0 && t.height > 0) {
      st.textures.push_back(std::move(t));
      idx = (int)st.textures.size() - 1;
    }
    texPool[path] = idx;
    return idx;
  }
  std::function<int(const std::string&)> texFn = [this](const std::string& r) { return texture(r); };
  // Named materials, one scope per object being read; lookups search the
  // innermost scope first (SceneJsonLoader::findMaterialByName).
  std::vector<std::map<std::string, rg_material>> scopes;
  std::string err;
  rg_status code = RG_ERR_IO;  // status returned with err

  const rg_material* findMaterial(const std::string& name) const {
    for (size_t i = scopes.size(); i-- > 0;) {
      auto it = scopes[i].find(name);
      if (it != scopes[i].end()) return &it->second;
    }
    return nullptr;
  }

  int addMaterial(const rg_material& m) {
    st.materials.push_back(m);
    return (int)st.materials.size() - 1;
  }

  // transformObject (rayrenderer.cpp:237-300): positions by the model matrix,
  // normals by its inverse transpose, renormalised.
  void emitMesh(const MeshTris& m, const M4& W, int mesh) {
    double Nm[3][3];
    normalMatrix(W, Nm);
    for (size_t k = 0; k + 2 < m.size(); k += 3) {
      for (int q = 0; q < 3; q++) {
        const Vtx& v = m[k + q];
        for (int a = 0; a < 3; a++) {
          const double p = W.m[a][0] * v.p[0] + W.m[a][1] * v.p[1] + W.m[a][2] * v.p[2] + W.m[a][3];
          st.positions.push_back((float)p);
        }
        double n[3];
        for (int a = 0; a < 3; a++) n[a] = Nm[a][0] * v.n[0] + Nm[a][1] * v.n[1] + Nm[a][2] * v.n[2];
        double l = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        if (l <= 0) l = 1;
        for (int a = 0; a < 3; a++) st.normals.push_back((float)(n[a] / l));
        st.uvs.push_back(v.uv[0]);
        st.uvs.push_back(v.uv[1]);
      }
      st.triMesh.push_back(mesh);
    }
  }

  // One flattened object: its meshes, its material, its medium.
  struct Node {
    std::vector<MeshTris> meshes;
    rg_material mat;
    bool hasMedium = false;
    MediumSpec medium;
    bool visible = true;
    bool isCamera = false;
    float loc[3] = {0, 0, 0}, ang[3] = {0, 0, 0}, scl[3] = {1, 1, 1};
    std::vector<std::unique_ptr<Node>> children;  // file order
  };

  bool loadObjFile(const std::string& path, Node& parent) {
    std::vector<ObjGroup> groups;
    std::map<std::string, ObjMtl> mtls;
    if (!readObj(path, groups, mtls, err)) return false;
    // readObjAsSceneObjects (sceneloader.cpp:424-479): each .obj object is a
    // child; material = scene override by name > .mtl defaults > the loading
    // object's material as it stands when the mesh key is read.
    for (auto& g : groups) {
      if (g.tris.empty()) continue;
      std::unique_ptr<Node> c(new Node());
      c->mat = parent.mat;
      const rg_material* over = g.material.empty() ? nullptr : findMaterial(g.material);
      auto mt = mtls.find(g.material);
      if (over) {
        c->mat = *over;
      } else if (!g.material.empty() && mt != mtls.end()) {
        c->mat = defaultMat();
        for (int a = 0; a < 3; a++) c->mat.color[a] = mt->second.kd[a];
        c->mat.transparency = mt->second.transparency;
      }
      c->meshes.push_back(std::move(g.tris));
      parent.children.push_back(std::move(c));
    }
    return true;
  }

  bool readMeshPath(const std::string& rel, Node& n) {
    const std::string path = (!rel.empty() && rel[0] == '/') ? rel : baseDir + rel;
    const size_t dot = path.find_last_of('.');
    std::string ext = dot == std::string::npos ? "" : path.substr(dot);
    for (char& ch : ext) ch = (char)std::tolower((unsigned char)ch);
    if (rel.compare(0, 6, "tob://") == 0 || rel.compare(0, 6, "sob://") == 0) {
      err = "bundle mesh URIs (tob:// and sob://) are not read: " + rel;
      code = RG_ERR_UNSUPPORTED;
      return false;
    }
    if (ext == ".obj") {
      // ObjFileReader::read returns without objects when the file cannot be
      // opened (objreader.cpp:99), so a missing .obj adds no geometry.
      std::ifstream probe(path);
      if (!probe) return true;
      return loadObjFile(path, n);
    }
    MeshTris m;
    if (!readMeshFile(path, m, err)) return false;
    n.meshes.push_back(std::move(m));
    return true;
  }

  // readSceneObject (sceneloader.cpp:505-780): keys in file order.
  bool read(const JVal& jo, Node& n, bool root) {
    if (const JVal* b = jo.get("_bundle")) {
      if (b->type == JVal::Str && !b->s.empty()) {
        err = ".toba bundles (\"_bundle\") are not read: " + b->s;
        code = RG_ERR_UNSUPPORTED;
        return false;
      }
    }
    scopes.emplace_back();
    if (const JVal* mats = jo.get("_materials"))
      if (mats->type == JVal::Obj)
        for (auto& p : mats->obj)
          if (p.second.type == JVal::Obj) {
            rg_material m = defaultMat();
            readMaterial(p.second, m, texFn);
            scopes.back()[p.first] = m;
          }
    if (n.isCamera) readCamera(jo);
    for (auto& p : jo.obj) {
      const std::string& k = p.first;
      const JVal& v = p.second;
      if (k == "_materials" || k == "_bundles" || k == "_bundle") continue;
      if (k == "location") readVec3(&v, n.loc);
      else if (k == "angle") readVec3(&v, n.ang);
      else if (k == "scale") readVec3(&v, n.scl);
      else if (k == "mesh") {
        if (v.type == JVal::Str) {
          if (!readMeshPath(v.s, n)) return false;
        } else if (v.type == JVal::Arr) {
          for (auto& e : v.arr)
            if (e.type == JVal::Str && !readMeshPath(e.s, n)) return false;
        } else if (v.type == JVal::Obj) {
          const JVal* ty = v.get("type");
          const std::string t = ty && ty->type == JVal::Str ? ty->s : "";
          if (t == "plane") {
            n.meshes.push_back(planeMesh());
          } else if (t == "cube") {
            n.meshes.push_back(cubeMesh());
          } else if (t == "sphere") {
            float r = 1, stacks = 16, slices = 32;
            v.num("radius", r);
            v.num("stacks", stacks);
            v.num("slices", slices);
            if (stacks < 1 || slices < 1) { err = "sphere needs stacks >= 1 and slices >= 1"; return false; }
            n.meshes.push_back(sphereMesh(r, (int)stacks, (int)slices));
          } else if (t == "cone") {
            float r0 = 0.5f, r1 = 0.5f, slices = 32;
            v.num("radiusStart", r0);
            v.num("radiusEnd", r1);
            v.num("slices", slices);
            n.meshes.push_back(coneMesh(r0, r1, (int)slices));
          }
        }
      } else if (k == "mat") {
        if (v.type == JVal::Str) {
          if (const rg_material* m = findMaterial(v.s)) n.mat = *m;
        } else if (v.type == JVal::Obj) {
          readMaterial(v, n.mat, texFn);
        }
      } else if (k == "visible" && v.type == JVal::Bool) {
        n.visible = v.b;
      } else if (k == "medium") {
        MediumSpec sp;
        if (v.type == JVal::Obj && readMedium(v, sp)) {
          if (root) {
            st.globalMedium = addMedium(sp, M4::ident());
          } else {
            n.medium = sp;
            n.hasMedium = true;
          }
        }
      } else if (k == "envmap") {
        if (!readEnvmap(v)) return false;
      } else if (v.type == JVal::Obj) {
        std::unique_ptr<Node> c(new Node());
        c->mat = defaultMat();
        const JVal* ty = v.get("type");
        c->isCamera = k == "mainCamera" || (ty && ty->type == JVal::Num && (int)ty->n == 801);
        if (!read(v, *c, false)) return false;
        if (k == "mainCamera") {
          haveCamera = true;
          cameraNode = c.get();
        }
        n.children.push_back(std::move(c));
      }
    }
    scopes.pop_back();
    return true;
  }

  // "envmap": a path, or {texture, intensity, rotation, cubemap, ext}
  // (sceneloader.cpp:700-748); the last one read wins.  As in the reference,
  // an image that cannot be opened leaves the scene without an environment
  // (Texture::loadFromFile yields an empty image, which samples black).  A
  // malformed file or a cubemap (six JPEG faces, no decoder here) is an error.
  bool readEnvmap(const JVal& v) {
    std::string rel;
    float intensity = 1.0f, rotation = 0.0f;
    if (v.type == JVal::Str) {
      rel = v.s;
    } else if (v.type == JVal::Obj) {
      // cubemap: six faces px nx py ny pz nz.<ext> (ext "jpg" by default) in a
      // directory, read through the texture pool; all six or none
      // (sceneloader.cpp:725-744, scene.cpp:348)
      if (const JVal* c = v.get("cubemap"))
        if (c->type == JVal::Str && !c->s.empty()) {
          std::string dir = c->s;
          if (dir.back() != '/' && dir.back() != '\\') dir += "/";
          std::string ext = "jpg";
          if (const JVal* e = v.get("ext"))
            if (e->type == JVal::Str && !e->s.empty()) ext = e->s;
          static const char* names[6] = {"px", "nx", "py", "ny", "pz", "nz"};
          int faces[6];
          bool all = true;
          for (int f = 0; f < 6; f++) {
            faces[f] = texture(dir + names[f] + "." + ext);
            all = all && faces[f] >= 0;
          }
          st.envCube = all ? 1 : 0;
          for (int f = 0; f < 6; f++) st.envCubeFaces[f] = all ? faces[f] : -1;
        }
      if (const JVal* t = v.get("texture"))
        if (t->type == JVal::Str) rel = t->s;
      v.num("intensity", intensity);
      v.num("rotation", rotation);
    }
    st.envmapIntensity = intensity;
    st.envmapRotation = rotation;
    if (rel.empty()) return true;
    const std::string path = rel[0] == '/' ? rel : baseDir + rel;
    {
      std::ifstream probe(path, std::ios::binary);
      if (!probe) {
        st.envmapTexture = -1;
        return true;
      }
    }
    TextureStore tex;
    if (!readImageFile(path, tex, err)) {
      code = RG_ERR_PARSE;
      return false;
    }
    st.textures.push_back(std::move(tex));
    st.envmapTexture = (int)st.textures.size() - 1;
    return true;
  }

  void readCamera(const JVal& c) {  // sceneloader.cpp:552-588
    rg_camera& cam = st.camera;
    c.num("fieldOfView", cam.field_of_view);
    c.num("depthOfField", cam.depth_of_field);
    c.num("aperture", cam.aperture);
    float blades = (float)cam.aperture_blades;
    if (c.num("apertureBlades", blades)) cam.aperture_blades = (int)blades;
    c.num("apertureRotation", cam.aperture_rotation);
    c.num("exposure", cam.exposure);
  }

  bool haveCamera = false;
  const Node* cameraNode = nullptr;

  // A medium into the scene, with the owning object's transform W applied to
  // the cone and the path points when they follow the object
  // (HomogeneousMedium::bake, medium.cpp:59-101; the camera part is applied
  // at render set-up).  Returns its index.
  int addMedium(const MediumSpec& sp, const M4& W) {
    rg_medium md = sp.m;
    std::vector<rg_medium_path_point> pts = sp.pts;
    auto point = [&](float p[3]) {
      double o[3];
      for (int a = 0; a < 3; a++) o[a] = W.m[a][0] * p[0] + W.m[a][1] * p[1] + W.m[a][2] * p[2] + W.m[a][3];
      for (int a = 0; a < 3; a++) p[a] = (float)o[a];
    };
    if (sp.coneFollow && md.emission_mode == RG_EMISSION_CONE) {
      point(md.cone_origin);
      double ax[3];
      for (int a = 0; a < 3; a++)
        ax[a] = W.m[a][0] * md.cone_axis[0] + W.m[a][1] * md.cone_axis[1] + W.m[a][2] * md.cone_axis[2];
      for (int a = 0; a < 3; a++) md.cone_axis[a] = (float)ax[a];
    }
    if (sp.pathFollow && md.emission_mode == RG_EMISSION_PATH)
      for (auto& q : pts) point(q.p);
    md.num_path_points = 0;
    md.path_points = nullptr;  // set by SceneStore::finalize
    st.media.push_back(md);
    st.mediumPaths.resize(st.media.size() - 1);
    st.mediumPaths.push_back(std::move(pts));
    return (int)st.media.size() - 1;
  }

  // transformObject / transformScene (rayrenderer.cpp:156-363): depth first,
  // an object's own meshes before its children; invisible objects are
  // skipped together with their children, except that any object whose
  // interior medium emits (cone or constant sigma_e) is a volume light
  // whether it is visible or has meshes (rayrenderer.cpp:180-206); such an
  // object without rendered meshes becomes an object without meshes.
  void flatten(const Node& n, const M4& parent, bool parentVisible = true) {
    if (n.isCamera) return;
    const bool vis = parentVisible && n.visible;
    const M4 W = parent * trs(n.loc, n.ang, n.scl);
    const bool meshObject = vis && !n.meshes.empty();
    const bool volume = n.hasMedium && emissiveVolume(n.medium.m);
    int medium = -1;
    if (n.hasMedium && (meshObject || volume)) medium = addMedium(n.medium, W);
    if (meshObject || volume) {
      rg_object o{};
      o.material = addMaterial(n.mat);
      o.interior_medium = medium;
      for (int a = 0; a < 3; a++) o.location[a] = n.loc[a];
      st.objects.push_back(o);
    }
    if (meshObject) {
      const int obj = (int)st.objects.size() - 1;
      for (auto& m : n.meshes) {
        st.meshObject.push_back(obj);
        emitMesh(m, W, (int)st.meshObject.size() - 1);
      }
    } else if (vis && n.mat.emission > 0.0f) {
      // Mesh-less emissive object -> point light at the object's origin
      // (rayrenderer.cpp:333-353).  The reference builds the object-space
      // normal from sin/cos of RADIAN_TO_DEGREE(angle) although the angle is
      // already in degrees; kept as is (angle 0 gives +Y), then mapped by the
      // object's normal matrix and normalised.
      const double k = 180.0 / 3.14159265358979323846;
      const float s1 = std::sin((float)(n.ang[0] * k)), c1 = std::cos((float)(n.ang[0] * k));
      const float s2 = std::sin((float)(n.ang[1] * k)), c2 = std::cos((float)(n.ang[1] * k));
      double no[3] = {(double)(c2 * s1), (double)(c2 * c1), (double)s2};
      const double lo = std::sqrt(no[0] * no[0] + no[1] * no[1] + no[2] * no[2]);
      for (double& c : no) c /= lo;
      double Nm[3][3];
      normalMatrix(W, Nm);
      rg_point_light pl;
      double nw[3];
      for (int a = 0; a < 3; a++) {
        pl.position[a] = (float)W.m[a][3];
        nw[a] = Nm[a][0] * no[0] + Nm[a][1] * no[1] + Nm[a][2] * no[2];
      }
      const double l = std::sqrt(nw[0] * nw[0] + nw[1] * nw[1] + nw[2] * nw[2]);
      for (int a = 0; a < 3; a++) pl.normal[a] = (float)(l > 0 ? nw[a] / l : (a == 1 ? 1.0 : 0.0));
      pl.material = addMaterial(n.mat);
      st.pointLights.push_back(pl);
    }
    for (auto& c : n.children) flatten(*c, W, vis);
  }
};

}  // namespace

rg_status loadSceneJson(const char* path, SceneStore** out, std::string& err) {
  *out = nullptr;
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = std::string("cannot open scene file ") + path;
    return RG_ERR_IO;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  Parser P(text);
  JVal root;
  if (text.empty() || !P.val(root) || root.type != JVal::Obj) {
    err = "scene JSON parse error: " +
          (text.empty() ? std::string("empty file") : P.err.empty() ? std::string("root is not an object") : P.err);
    return RG_ERR_PARSE;
  }
  std::unique_ptr<SceneStore> st(new SceneStore());
  // Camera member defaults (scene.h, Camera)
  std::memset(&st->camera, 0, sizeof(st->camera));
  st->camera.field_of_view = 75.0f;
  st->camera.view_near = 0.1f;
  st->camera.view_far = 50.0f;
  st->camera.aperture = 1.8f;
  st->camera.aperture_blades = 0;
  st->camera.exposure = 1.0f;
  Loader L{*st};
  const std::string p(path);
  L.baseDir = p.find_last_of('/') == std::string::npos ? "" : p.substr(0, p.find_last_of('/') + 1);
  Loader::Node top;
  top.mat = defaultMat();
  if (!L.read(root, top, true)) {
    err = L.err;
    return L.code;
  }
  // The root's own transform and meshes are not rendered (transformScene
  // walks the root's children).
  for (auto& c : top.children) L.flatten(*c, M4::ident());
  if (L.cameraNode) {
    for (int a = 0; a < 3; a++) {
      st->camera.location[a] = L.cameraNode->loc[a];
      st->camera.angle[a] = L.cameraNode->ang[a];
    }
  }
  if (st->materials.empty()) L.addMaterial(defaultMat());
  st->finalize();
  *out = st.release();
  return RG_OK;
}

}  // namespace rg
