// rg_decode.cpp - JPEG and PNG readers for material textures ('tex') and
// environment maps.
//
// The reference decodes these through its image-module submodule
// (ugm::loadImage, texture.cpp:189), which is not in its tree, so both are
// written here from the public specifications:
//  * JPEG, ITU-T T.81: baseline and extended sequential DCT with Huffman
//    coding, 8-bit samples, one or three components (YCbCr, or RGB when an
//    Adobe marker says so), any sampling factors, interleaved or
//    single-component scans, restart intervals.  Inverse DCT straight from
//    its definition (A.3.3) in double precision, rounded to 8 bits; chroma
//    is upsampled by linear interpolation between sample centres (the JFIF
//    centred siting), and YCbCr -> RGB uses the JFIF equations.  Progressive
//    and arithmetic-coded files are refused.
//  * PNG, RFC 2083: every colour type and bit depth, palette transparency,
//    Adam7 interlacing, the five row filters; zlib inflates the data.
// Pixels come out as RGBA floats in [0, 1] (the byte value / 255, 16-bit
// samples / 65535), row 0 at the top, marked LDR: the renderer applies the
// sRGB decode when it samples them (Texture::sample, texture.cpp:210-241).
#include <zlib.h>

#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "rg_host.h"

namespace rg {

namespace {

// zig-zag scan position -> natural (row-major) index in an 8x8 block (T.81 Figure A.6)
const int kNatural[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                          41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                          30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

// Canonical Huffman decoding table (T.81 Annex C / F.2.2.3): codes of length
// l run from mincode[l] to maxcode[l] and index vals from valptr[l].
struct Huffman {
  bool defined = false;
  int mincode[17], maxcode[17], valptr[17];
  uint8_t vals[256];
};

bool buildHuffman(Huffman& h, const uint8_t* counts, const uint8_t* symbols, int total) {
  int code = 0, k = 0;
  for (int l = 1; l <= 16; l++) {
    const int n = counts[l - 1];
    h.valptr[l] = k;
    h.mincode[l] = code;
    code += n;
    k += n;
    if (code > (1 << l)) return false;  // over-subscribed code lengths
    h.maxcode[l] = n ? code - 1 : -1;
    code <<= 1;
  }
  if (k != total || total > 256) return false;
  std::memcpy(h.vals, symbols, (size_t)total);
  h.defined = true;
  return true;
}

// Entropy-coded segment reader: removes the 0xFF00 stuffing, stops at a marker
// (feeding zero bits past it, F.2.2.5).
struct Bits {
  const uint8_t* p = nullptr;
  size_t n = 0, pos = 0;
  uint32_t buf = 0;
  int cnt = 0;
  bool atMarker = false;

  void fill() {
    while (cnt <= 24) {
      uint32_t b = 0;
      if (!atMarker && pos < n) {
        b = p[pos];
        if (b == 0xFF) {
          const uint32_t nx = pos + 1 < n ? p[pos + 1] : 0xD9;
          if (nx == 0x00) {
            pos += 2;
          } else {
            atMarker = true;
            b = 0;
          }
        } else {
          pos++;
        }
      }
      buf |= b << (24 - cnt);
      cnt += 8;
    }
  }
  uint32_t peek16() {
    fill();
    return buf >> 16;
  }
  void skip(int k) {
    buf <<= k;
    cnt -= k;
  }
  int get(int k) {
    if (k == 0) return 0;
    fill();
    const int v = (int)(buf >> (32 - k));
    skip(k);
    return v;
  }
  // RECEIVE + EXTEND (F.2.2.1)
  int extend(int s) {
    if (s == 0) return 0;
    const int v = get(s);
    return v < (1 << (s - 1)) ? v - (1 << s) + 1 : v;
  }
  int decode(const Huffman& h) {
    const uint32_t c16 = peek16();
    for (int l = 1; l <= 16; l++) {
      const int code = (int)(c16 >> (16 - l));
      if (h.maxcode[l] >= 0 && code <= h.maxcode[l]) {
        skip(l);
        return h.vals[h.valptr[l] + code - h.mincode[l]];
      }
    }
    return -1;
  }
  // expect RSTn at the current byte position (after the padding bits)
  bool restart() {
    buf = 0;
    cnt = 0;
    atMarker = false;
    while (pos + 1 < n && !(p[pos] == 0xFF && p[pos + 1] >= 0xD0 && p[pos + 1] <= 0xD7)) {
      if (p[pos] == 0xFF && p[pos + 1] != 0x00 && p[pos + 1] != 0xFF) return false;  // another marker
      pos++;
    }
    if (pos + 1 >= n) return false;
    pos += 2;
    return true;
  }
};

struct JComp {
  int id = 0, h = 1, v = 1, tq = 0, td = 0, ta = 0;
  int bw = 0, bh = 0;   // blocks per row / column of the padded plane
  int w = 0, ht = 0;    // samples of the component inside the image
  int dc = 0;
  std::vector<uint8_t> plane;  // bw*8 x bh*8 samples
};

// 8x8 inverse DCT from its definition (T.81 A.3.3): 128 + 1/4 sum C(u)C(v) F cos cos.
struct Idct {
  double c[8][8];  // c[x][u] = C(u)/2 cos((2x+1) u pi / 16)
  Idct() {
    for (int x = 0; x < 8; x++)
      for (int u = 0; u < 8; u++)
        c[x][u] = (u == 0 ? std::sqrt(0.5) : 1.0) * 0.5 * std::cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0);
  }
  void run(const int* F, uint8_t* out, int stride) const {
    double tmp[64];
    for (int v = 0; v < 8; v++)
      for (int x = 0; x < 8; x++) {
        double s = 0;
        for (int u = 0; u < 8; u++) s += c[x][u] * F[v * 8 + u];
        tmp[v * 8 + x] = s;
      }
    for (int y = 0; y < 8; y++)
      for (int x = 0; x < 8; x++) {
        double s = 0;
        for (int v = 0; v < 8; v++) s += c[y][v] * tmp[v * 8 + x];
        const double val = std::floor(s + 128.0 + 0.5);
        out[y * stride + x] = (uint8_t)(val < 0 ? 0 : (val > 255 ? 255 : val));
      }
  }
};

inline int be16(const uint8_t* p) { return (p[0] << 8) | p[1]; }

}  // namespace

bool decodeJpeg(const std::vector<unsigned char>& b, TextureStore& out, std::string& err) {
  const size_t n = b.size();
  if (n < 4 || b[0] != 0xFF || b[1] != 0xD8) {
    err = "not a JPEG file";
    return false;
  }
  uint16_t qt[4][64];
  bool qdef[4] = {false, false, false, false};
  Huffman hdc[4], hac[4];
  std::vector<JComp> comp;
  int W = 0, H = 0, hmax = 1, vmax = 1, restartInterval = 0, adobeTransform = -1;
  bool frame = false, anyScan = false;
  const Idct idct;
  size_t pos = 2;
  auto fail = [&](const std::string& m) {
    err = "JPEG: " + m;
    return false;
  };
  while (pos + 4 <= n) {
    if (b[pos] != 0xFF) return fail("marker expected");
    const int m = b[pos + 1];
    if (m == 0xFF) {  // fill byte
      pos++;
      continue;
    }
    pos += 2;
    if (m == 0xD9) break;                     // EOI
    if (m == 0x01 || (m >= 0xD0 && m <= 0xD7)) continue;
    if (pos + 2 > n) return fail("truncated segment");
    const int len = be16(&b[pos]);
    if (len < 2 || pos + len > n) return fail("bad segment length");
    const uint8_t* s = &b[pos + 2];
    const int sl = len - 2;
    if (m == 0xDB) {  // DQT
      int k = 0;
      while (k < sl) {
        const int pq = s[k] >> 4, tq = s[k] & 15;
        if (tq > 3 || k + 1 + 64 * (pq + 1) > sl) return fail("bad quantisation table");
        for (int i = 0; i < 64; i++) qt[tq][i] = pq ? (uint16_t)be16(&s[k + 1 + 2 * i]) : s[k + 1 + i];
        qdef[tq] = true;
        k += 1 + 64 * (pq + 1);
      }
    } else if (m == 0xC4) {  // DHT
      int k = 0;
      while (k < sl) {
        if (k + 17 > sl) return fail("bad Huffman table");
        const int tc = s[k] >> 4, th = s[k] & 15;
        int total = 0;
        for (int i = 0; i < 16; i++) total += s[k + 1 + i];
        if (tc > 1 || th > 3 || k + 17 + total > sl) return fail("bad Huffman table");
        if (!buildHuffman(tc ? hac[th] : hdc[th], &s[k + 1], &s[k + 17], total)) return fail("bad Huffman code lengths");
        k += 17 + total;
      }
    } else if (m == 0xDD) {  // DRI
      if (sl < 2) return fail("bad restart interval");
      restartInterval = be16(s);
    } else if (m == 0xEE) {  // APP14 "Adobe": colour transform flag
      if (sl >= 12 && std::memcmp(s, "Adobe", 5) == 0) adobeTransform = s[11];
    } else if (m == 0xC0 || m == 0xC1) {  // SOF0 / SOF1
      if (frame) return fail("second frame");
      if (sl < 6 || s[0] != 8) return fail("only 8-bit samples are supported");
      H = be16(&s[1]);
      W = be16(&s[3]);
      const int nf = s[5];
      if (W <= 0 || H <= 0) return fail("zero image size (DNL) is not supported");
      if ((nf != 1 && nf != 3) || sl < 6 + 3 * nf) return fail("only 1 or 3 components are supported");
      comp.resize(nf);
      for (int i = 0; i < nf; i++) {
        comp[i].id = s[6 + 3 * i];
        comp[i].h = s[7 + 3 * i] >> 4;
        comp[i].v = s[7 + 3 * i] & 15;
        comp[i].tq = s[8 + 3 * i];
        if (comp[i].h < 1 || comp[i].h > 4 || comp[i].v < 1 || comp[i].v > 4 || comp[i].tq > 3)
          return fail("bad component parameters");
        hmax = std::max(hmax, comp[i].h);
        vmax = std::max(vmax, comp[i].v);
      }
      const int mcux = (W + 8 * hmax - 1) / (8 * hmax), mcuy = (H + 8 * vmax - 1) / (8 * vmax);
      for (auto& c : comp) {
        c.bw = mcux * c.h;
        c.bh = mcuy * c.v;
        c.w = (W * c.h + hmax - 1) / hmax;
        c.ht = (H * c.v + vmax - 1) / vmax;
        c.plane.assign((size_t)c.bw * 8 * c.bh * 8, 0);
      }
      frame = true;
    } else if ((m >= 0xC2 && m <= 0xC3) || (m >= 0xC5 && m <= 0xC7) || (m >= 0xC9 && m <= 0xCB) ||
               (m >= 0xCD && m <= 0xCF)) {
      return fail("progressive, lossless, hierarchical or arithmetic-coded files are not supported");
    } else if (m == 0xDA) {  // SOS + entropy-coded data
      if (!frame) return fail("scan before frame");
      const int ns = s[0];
      if (ns < 1 || ns > 4 || sl < 1 + 2 * ns + 3) return fail("bad scan header");
      std::vector<JComp*> sc;
      for (int i = 0; i < ns; i++) {
        JComp* c = nullptr;
        for (auto& q : comp)
          if (q.id == s[1 + 2 * i]) c = &q;
        if (!c) return fail("scan names an unknown component");
        c->td = s[2 + 2 * i] >> 4;
        c->ta = s[2 + 2 * i] & 15;
        if (c->td > 3 || c->ta > 3 || !hdc[c->td].defined || !hac[c->ta].defined || !qdef[c->tq])
          return fail("scan uses an undefined table");
        c->dc = 0;
        sc.push_back(c);
      }
      Bits bits;
      bits.p = b.data();
      bits.n = n;
      bits.pos = pos + len;
      int F[64];
      auto block = [&](JComp& c, int bx, int by) -> bool {
        std::memset(F, 0, sizeof(F));
        const uint16_t* q = qt[c.tq];
        const int t = bits.decode(hdc[c.td]);
        if (t < 0 || t > 11) return false;
        c.dc += bits.extend(t);
        F[0] = c.dc * q[0];
        for (int k = 1; k < 64;) {
          const int rs = bits.decode(hac[c.ta]);
          if (rs < 0) return false;
          const int r = rs >> 4, sz = rs & 15;
          if (sz == 0) {
            if (r != 15) break;  // EOB
            k += 16;
            continue;
          }
          k += r;
          if (k > 63) return false;
          F[kNatural[k]] = bits.extend(sz) * q[k];
          k++;
        }
        idct.run(F, &c.plane[((size_t)by * 8) * c.bw * 8 + (size_t)bx * 8], c.bw * 8);
        return true;
      };
      long long mcus, done = 0;
      int perRow;
      if (ns == 1) {  // non-interleaved: one block per MCU over the component's own grid
        perRow = (sc[0]->w + 7) / 8;
        mcus = (long long)perRow * ((sc[0]->ht + 7) / 8);
      } else {
        perRow = (W + 8 * hmax - 1) / (8 * hmax);
        mcus = (long long)perRow * ((H + 8 * vmax - 1) / (8 * vmax));
      }
      for (long long mcu = 0; mcu < mcus; mcu++) {
        if (restartInterval > 0 && mcu > 0 && mcu % restartInterval == 0) {
          if (!bits.restart()) return fail("missing restart marker");
          for (auto* c : sc) c->dc = 0;
        }
        const int mx = (int)(mcu % perRow), my = (int)(mcu / perRow);
        if (ns == 1) {
          if (!block(*sc[0], mx, my)) return fail("corrupt entropy-coded data");
        } else {
          for (auto* c : sc)
            for (int yy = 0; yy < c->v; yy++)
              for (int xx = 0; xx < c->h; xx++)
                if (!block(*c, mx * c->h + xx, my * c->v + yy)) return fail("corrupt entropy-coded data");
        }
        done++;
      }
      (void)done;
      anyScan = true;
      // continue after the entropy-coded data: the next marker that is not RSTn
      size_t p2 = bits.pos;
      while (p2 + 1 < n && !(b[p2] == 0xFF && b[p2 + 1] != 0x00 && !(b[p2 + 1] >= 0xD0 && b[p2 + 1] <= 0xD7)))
        p2++;
      pos = p2;
      continue;
    }
    pos += len;
  }
  if (!frame || !anyScan) return fail("no image data");
  // upsample to full resolution, convert to RGB
  out.width = W;
  out.height = H;
  out.isHdr = 0;
  out.rgba.assign((size_t)W * H * 4, 1.0f);
  auto sample = [&](const JComp& c, int x, int y) -> double {
    const int stride = c.bw * 8;
    if (c.h == hmax && c.v == vmax) return c.plane[(size_t)y * stride + x];
    // centre of output pixel x in component sample units, minus the sample-centre offset
    const double sx = (x + 0.5) * c.h / hmax - 0.5, sy = (y + 0.5) * c.v / vmax - 0.5;
    const int x0 = (int)std::floor(sx), y0 = (int)std::floor(sy);
    const double fx = sx - x0, fy = sy - y0;
    auto at = [&](int xx, int yy) -> double {
      xx = std::min(std::max(xx, 0), c.w - 1);
      yy = std::min(std::max(yy, 0), c.ht - 1);
      return c.plane[(size_t)yy * stride + xx];
    };
    return (at(x0, y0) * (1 - fx) + at(x0 + 1, y0) * fx) * (1 - fy) + (at(x0, y0 + 1) * (1 - fx) + at(x0 + 1, y0 + 1) * fx) * fy;
  };
  auto to8 = [](double v) { v = std::floor(v + 0.5); return (float)((v < 0 ? 0 : (v > 255 ? 255 : v)) / 255.0); };
  const bool rgb = comp.size() == 3 && (adobeTransform == 0 || (adobeTransform < 0 && comp[0].id == 'R' && comp[1].id == 'G'));
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      float* o = &out.rgba[((size_t)y * W + x) * 4];
      if (comp.size() == 1) {
        o[0] = o[1] = o[2] = to8(sample(comp[0], x, y));
      } else if (rgb) {
        for (int k = 0; k < 3; k++) o[k] = to8(sample(comp[k], x, y));
      } else {  // JFIF YCbCr -> RGB
        const double Y = sample(comp[0], x, y), cb = sample(comp[1], x, y) - 128.0, cr = sample(comp[2], x, y) - 128.0;
        o[0] = to8(Y + 1.402 * cr);
        o[1] = to8(Y - 0.344136 * cb - 0.714136 * cr);
        o[2] = to8(Y + 1.772 * cb);
      }
    }
  return true;
}

// ---- PNG ---------------------------------------------------------------------
namespace {

inline uint32_t be32(const uint8_t* p) {
  return ((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | p[3];
}

inline int paeth(int a, int b, int c) {
  const int p = a + b - c, pa = std::abs(p - a), pb = std::abs(p - b), pc = std::abs(p - c);
  if (pa <= pb && pa <= pc) return a;
  return pb <= pc ? b : c;
}

// Undo the row filters of one (sub)image of w x h pixels; `in` holds filter byte + row bytes per row.
bool unfilter(const uint8_t* in, int w, int h, int bitsPerPixel, std::vector<uint8_t>& rows) {
  const size_t rowBytes = ((size_t)w * bitsPerPixel + 7) / 8;
  const int bpp = std::max(1, bitsPerPixel / 8);
  rows.assign(rowBytes * h, 0);
  for (int y = 0; y < h; y++) {
    const uint8_t ft = in[(size_t)y * (rowBytes + 1)];
    const uint8_t* src = in + (size_t)y * (rowBytes + 1) + 1;
    uint8_t* cur = &rows[(size_t)y * rowBytes];
    const uint8_t* prev = y ? &rows[(size_t)(y - 1) * rowBytes] : nullptr;
    for (size_t i = 0; i < rowBytes; i++) {
      const int a = i >= (size_t)bpp ? cur[i - bpp] : 0, up = prev ? prev[i] : 0,
                c = (prev && i >= (size_t)bpp) ? prev[i - bpp] : 0;
      int v = src[i];
      switch (ft) {
        case 0: break;
        case 1: v += a; break;
        case 2: v += up; break;
        case 3: v += (a + up) >> 1; break;
        case 4: v += paeth(a, up, c); break;
        default: return false;
      }
      cur[i] = (uint8_t)v;
    }
  }
  return true;
}

}  // namespace

bool decodePng(const std::vector<unsigned char>& b, TextureStore& out, std::string& err) {
  static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
  auto fail = [&](const std::string& m) {
    err = "PNG: " + m;
    return false;
  };
  if (b.size() < 8 || std::memcmp(b.data(), sig, 8) != 0) return fail("bad signature");
  int W = 0, H = 0, depth = 0, ctype = -1, interlace = 0;
  std::vector<uint8_t> idat, palette, trns;
  size_t pos = 8;
  bool ihdr = false, iend = false;
  while (pos + 12 <= b.size() && !iend) {
    const uint32_t len = be32(&b[pos]);
    if (len > b.size() - pos - 12) return fail("truncated chunk");
    const uint8_t* type = &b[pos + 4];
    const uint8_t* d = &b[pos + 8];
    const uint32_t crc = be32(&b[pos + 8 + len]);
    if ((uint32_t)crc32(crc32(0L, Z_NULL, 0), type, len + 4) != crc) return fail("chunk CRC mismatch");
    if (!std::memcmp(type, "IHDR", 4)) {
      if (len < 13) return fail("bad IHDR");
      W = (int)be32(d);
      H = (int)be32(d + 4);
      depth = d[8];
      ctype = d[9];
      interlace = d[12];
      if (W <= 0 || H <= 0 || W > (1 << 16) || H > (1 << 16) || d[10] != 0 || d[11] != 0 || interlace > 1)
        return fail("unsupported header");
      const bool ok = (ctype == 0 && (depth == 1 || depth == 2 || depth == 4 || depth == 8 || depth == 16)) ||
                      (ctype == 3 && (depth == 1 || depth == 2 || depth == 4 || depth == 8)) ||
                      ((ctype == 2 || ctype == 4 || ctype == 6) && (depth == 8 || depth == 16));
      if (!ok) return fail("bad colour type / bit depth");
      ihdr = true;
    } else if (!std::memcmp(type, "PLTE", 4)) {
      palette.assign(d, d + len);
    } else if (!std::memcmp(type, "tRNS", 4)) {
      trns.assign(d, d + len);
    } else if (!std::memcmp(type, "IDAT", 4)) {
      idat.insert(idat.end(), d, d + len);
    } else if (!std::memcmp(type, "IEND", 4)) {
      iend = true;
    }
    pos += 12 + len;
  }
  if (!ihdr || idat.empty()) return fail("missing IHDR or IDAT");
  if (ctype == 3 && palette.size() < 3) return fail("palette image without PLTE");
  const int chans = ctype == 0 ? 1 : ctype == 2 ? 3 : ctype == 3 ? 1 : ctype == 4 ? 2 : 4;
  const int bitsPerPixel = chans * depth;
  // Adam7 passes (RFC 2083 2.6); one pass covering everything when not interlaced
  static const int a7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
  const int passes = interlace ? 7 : 1;
  size_t total = 0;
  int pw[7], ph[7];
  for (int p = 0; p < passes; p++) {
    const int x0 = interlace ? a7[p][0] : 0, y0 = interlace ? a7[p][1] : 0, dx = interlace ? a7[p][2] : 1,
              dy = interlace ? a7[p][3] : 1;
    pw[p] = W > x0 ? (W - x0 + dx - 1) / dx : 0;
    ph[p] = H > y0 ? (H - y0 + dy - 1) / dy : 0;
    if (pw[p] > 0 && ph[p] > 0) total += (size_t)ph[p] * (1 + ((size_t)pw[p] * bitsPerPixel + 7) / 8);
  }
  std::vector<uint8_t> raw(total);
  uLongf rawLen = (uLongf)total;
  if (uncompress(raw.data(), &rawLen, idat.data(), (uLong)idat.size()) != Z_OK || rawLen != total)
    return fail("bad compressed data");
  out.width = W;
  out.height = H;
  out.isHdr = 0;
  out.rgba.assign((size_t)W * H * 4, 1.0f);
  const double maxv = (double)((1 << depth) - 1);
  size_t off = 0;
  std::vector<uint8_t> rows;
  for (int p = 0; p < passes; p++) {
    if (pw[p] <= 0 || ph[p] <= 0) continue;
    const size_t rowBytes = ((size_t)pw[p] * bitsPerPixel + 7) / 8;
    if (!unfilter(&raw[off], pw[p], ph[p], bitsPerPixel, rows)) return fail("bad filter type");
    off += (size_t)ph[p] * (rowBytes + 1);
    const int x0 = interlace ? a7[p][0] : 0, y0 = interlace ? a7[p][1] : 0, dx = interlace ? a7[p][2] : 1,
              dy = interlace ? a7[p][3] : 1;
    for (int y = 0; y < ph[p]; y++) {
      const uint8_t* r = &rows[(size_t)y * rowBytes];
      auto samp = [&](int i) -> int {  // i-th sample of the row
        if (depth == 8) return r[i];
        if (depth == 16) return (r[2 * i] << 8) | r[2 * i + 1];
        const int perByte = 8 / depth;
        return (r[i / perByte] >> ((perByte - 1 - i % perByte) * depth)) & ((1 << depth) - 1);
      };
      for (int x = 0; x < pw[p]; x++) {
        float* o = &out.rgba[((size_t)(y0 + y * dy) * W + (x0 + x * dx)) * 4];
        if (ctype == 3) {
          const int idx = samp(x);
          if ((size_t)idx * 3 + 2 >= palette.size()) return fail("palette index out of range");
          for (int k = 0; k < 3; k++) o[k] = palette[idx * 3 + k] / 255.0f;
          o[3] = (size_t)idx < trns.size() ? trns[idx] / 255.0f : 1.0f;
        } else {
          const int base = x * chans;
          if (ctype == 0 || ctype == 4) {
            o[0] = o[1] = o[2] = (float)(samp(base) / maxv);
            if (ctype == 4) o[3] = (float)(samp(base + 1) / maxv);
          } else {
            for (int k = 0; k < 3; k++) o[k] = (float)(samp(base + k) / maxv);
            if (ctype == 6) o[3] = (float)(samp(base + 3) / maxv);
          }
        }
      }
    }
  }
  return true;
}

}  // namespace rg
