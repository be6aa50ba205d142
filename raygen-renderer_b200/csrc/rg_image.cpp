// rg_image.cpp - image file readers for textures and environment maps.
//
// Radiance RGBE (.hdr): header lines up to a blank line ("#?RADIANCE" or
// "#?RGBE" magic, FORMAT=32-bit_rle_rgbe), then "-Y H +X W", then H
// scanlines top to bottom.  Adaptive-RLE scanlines (2, 2, W>>8, W&255, then
// per channel runs: count > 128 repeats the next byte count-128 times,
// otherwise count literal bytes) decode as decodeRadianceHDR
// (texture.cpp:74-151): channel * 2^(E-136), black when E == 0.  The
// reference refuses flat (uncompressed) scanlines; this reader also accepts
// them, so files written without RLE (for example by simple writers) load.
// PFM: "PF" (RGB) or "Pf" (grey), "W H", scale (negative = little endian),
// rows bottom to top; returned top to bottom like every other image here.
//
// Writers (the CLI's output step, main.cpp:479-485): Radiance RGBE with RLE
// scanlines, PFM, binary PPM, PNG (zlib) and baseline JPEG.  The reference's
// codecs live in its image-module submodule (not in its tree), so the LDR
// formats are written here from their public specifications: PNG (RFC 2083,
// 8-bit RGB, filter 0) and JPEG (ITU-T T.81 baseline sequential DCT with the
// Annex K example quantisation and Huffman tables, quality scaled as the IJG
// library does, 4:4:4 sampling, JFIF header).
#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "rg_host.h"

namespace rg {

namespace {

bool readAll(const std::string& path, std::vector<unsigned char>& out, std::string& err) {
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return true;
}

// one '\n'-terminated line starting at pos (without the newline)
bool nextLine(const std::vector<unsigned char>& b, size_t& pos, std::string& line) {
  if (pos >= b.size()) return false;
  line.clear();
  while (pos < b.size() && b[pos] != '\n') line += (char)b[pos++];
  if (pos < b.size()) pos++;
  if (!line.empty() && line.back() == '\r') line.pop_back();
  return true;
}

}  // namespace

bool readRadianceHdr(const std::string& path, TextureStore& out, std::string& err) {
  std::vector<unsigned char> b;
  if (!readAll(path, b, err)) return false;
  auto bad = [&](const char* why) {
    err = std::string("malformed Radiance HDR file (") + why + "): " + path;
    return false;
  };
  size_t pos = 0;
  std::string line;
  bool magic = false, rgbe = false;
  for (;;) {
    if (!nextLine(b, pos, line)) return bad("header");
    if (line.empty()) break;
    if (line.compare(0, 10, "#?RADIANCE") == 0 || line.compare(0, 6, "#?RGBE") == 0) magic = true;
    if (line.compare(0, 7, "FORMAT=") == 0 && line.compare(7, 15, "32-bit_rle_rgbe") == 0) rgbe = true;
  }
  if (!magic || !rgbe) return bad("not 32-bit_rle_rgbe");
  if (!nextLine(b, pos, line)) return bad("resolution");
  int H = 0, W = 0;
  if (std::sscanf(line.c_str(), "-Y %d +X %d", &H, &W) != 2 || W <= 0 || H <= 0 || W > 65536 || H > 65536)
    return bad("resolution line");
  out.width = W;
  out.height = H;
  out.isHdr = 1;
  out.rgba.assign((size_t)W * H * 4, 0.0f);
  std::vector<unsigned char> sl((size_t)W * 4);
  for (int y = 0; y < H; y++) {
    if (pos + 4 > b.size()) return bad("truncated");
    const unsigned char* h4 = &b[pos];
    if (h4[0] == 2 && h4[1] == 2 && (h4[2] & 0x80) == 0) {
      if (((h4[2] << 8) | h4[3]) != W) return bad("scanline width");
      pos += 4;
      for (int ch = 0; ch < 4; ch++) {
        int p = 0;
        while (p < W) {
          if (pos >= b.size()) return bad("truncated run");
          const int count = b[pos++];
          if (count > 128) {
            const int run = count & 0x7f;
            if (pos >= b.size() || p + run > W) return bad("run overflow");
            const unsigned char v = b[pos++];
            for (int i = 0; i < run; i++) sl[(size_t)(p + i) * 4 + ch] = v;
            p += run;
          } else {
            if (count == 0 || p + count > W || pos + count > b.size()) return bad("literal overflow");
            for (int i = 0; i < count; i++) sl[(size_t)(p + i) * 4 + ch] = b[pos++];
            p += count;
          }
        }
      }
    } else {
      if (pos + (size_t)W * 4 > b.size()) return bad("truncated flat scanline");
      std::memcpy(sl.data(), &b[pos], (size_t)W * 4);
      pos += (size_t)W * 4;
    }
    for (int x = 0; x < W; x++) {
      const unsigned char* q = &sl[(size_t)x * 4];
      const float sc = q[3] == 0 ? 0.0f : std::ldexp(1.0f, (int)q[3] - 128 - 8);
      float* o = &out.rgba[((size_t)y * W + x) * 4];
      o[0] = q[0] * sc;
      o[1] = q[1] * sc;
      o[2] = q[2] * sc;
      o[3] = 1.0f;
    }
  }
  return true;
}

bool readPfm(const std::string& path, TextureStore& out, std::string& err) {
  std::vector<unsigned char> b;
  if (!readAll(path, b, err)) return false;
  auto bad = [&](const char* why) {
    err = std::string("malformed PFM file (") + why + "): " + path;
    return false;
  };
  // three whitespace-separated header tokens after the magic, then one byte
  size_t pos = 0;
  auto token = [&](std::string& t) {
    t.clear();
    while (pos < b.size() && std::isspace(b[pos])) pos++;
    while (pos < b.size() && !std::isspace(b[pos])) t += (char)b[pos++];
    return !t.empty();
  };
  std::string magic, ws, hs, ss;
  if (!token(magic) || (magic != "PF" && magic != "Pf")) return bad("magic");
  if (!token(ws) || !token(hs) || !token(ss)) return bad("header");
  pos++;  // the single whitespace byte before the raster
  const int W = std::atoi(ws.c_str()), H = std::atoi(hs.c_str());
  const double scale = std::atof(ss.c_str());
  const int C = magic == "PF" ? 3 : 1;
  if (W <= 0 || H <= 0 || W > 65536 || H > 65536 || scale == 0.0) return bad("dimensions");
  if (pos > b.size() || b.size() - pos < (size_t)W * H * C * 4) return bad("truncated");
  const bool little = scale < 0.0;
  out.width = W;
  out.height = H;
  out.isHdr = 1;
  out.rgba.assign((size_t)W * H * 4, 1.0f);
  for (int row = 0; row < H; row++) {
    const int y = H - 1 - row;
    for (int x = 0; x < W; x++)
      for (int c = 0; c < C; c++) {
        unsigned char q[4];
        std::memcpy(q, &b[pos + (((size_t)row * W + x) * C + c) * 4], 4);
        if (!little) std::swap(q[0], q[3]), std::swap(q[1], q[2]);
        float v;
        std::memcpy(&v, q, 4);
        float* o = &out.rgba[((size_t)y * W + x) * 4];
        if (C == 3) o[c] = v;
        else o[0] = o[1] = o[2] = v;
      }
  }
  return true;
}

// Texture::loadFromFile (texture.cpp:170-195): '.hdr' by name, everything
// else by content (the reference's loadImage probes the codecs); PFM by name.
bool readImageFile(const std::string& path, TextureStore& out, std::string& err) {
  const size_t dot = path.find_last_of('.');
  std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
  for (char& c : ext) c = (char)std::tolower((unsigned char)c);
  if (ext == "hdr") return readRadianceHdr(path, out, err);
  if (ext == "pfm") return readPfm(path, out, err);
  std::vector<unsigned char> b;
  if (!readAll(path, b, err)) return false;
  if (b.size() >= 2 && b[0] == 0xFF && b[1] == 0xD8) {
    if (decodeJpeg(b, out, err)) return true;
  } else if (b.size() >= 8 && b[0] == 0x89 && b[1] == 'P' && b[2] == 'N' && b[3] == 'G') {
    if (decodePng(b, out, err)) return true;
  } else {
    err = "unsupported image format (Radiance .hdr, PFM, JPEG and PNG are read)";
  }
  err += ": " + path;
  return false;
}

namespace {

// ---- writers -------------------------------------------------------------
inline unsigned char to8(float v) {
  if (!(v > 0.0f)) return 0;
  if (v >= 1.0f) return 255;
  return (unsigned char)(v * 255.0f + 0.5f);
}

bool writeFile(const std::string& path, const std::vector<unsigned char>& data, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot write " + path;
    return false;
  }
  const bool ok = std::fwrite(data.data(), 1, data.size(), f) == data.size();
  if (std::fclose(f) != 0 || !ok) {
    err = "write failed: " + path;
    return false;
  }
  return true;
}

void putStr(std::vector<unsigned char>& o, const std::string& s) { o.insert(o.end(), s.begin(), s.end()); }

bool writeRgbe(const std::string& path, int W, int H, const float* rgba, std::string& err) {
  std::vector<unsigned char> o;
  putStr(o, "#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n-Y " + std::to_string(H) + " +X " + std::to_string(W) + "\n");
  std::vector<unsigned char> q((size_t)W * 4);
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      const float* p = rgba + ((size_t)y * W + x) * 4;
      const float r = std::fmax(p[0], 0.0f), g = std::fmax(p[1], 0.0f), b = std::fmax(p[2], 0.0f);
      const float m = std::fmax(r, std::fmax(g, b));
      unsigned char* e = &q[(size_t)x * 4];
      if (m < 1e-32f || !std::isfinite(m)) {
        e[0] = e[1] = e[2] = e[3] = 0;
      } else {
        int ex;
        const float sc = std::frexp(m, &ex) * 256.0f / m;
        e[0] = (unsigned char)std::fmin(255.0f, r * sc);
        e[1] = (unsigned char)std::fmin(255.0f, g * sc);
        e[2] = (unsigned char)std::fmin(255.0f, b * sc);
        e[3] = (unsigned char)(ex + 128);
      }
    }
    if (W < 8 || W > 32767) {  // RLE scanlines need 8 <= width < 32768
      o.insert(o.end(), q.begin(), q.end());
      continue;
    }
    o.push_back(2);
    o.push_back(2);
    o.push_back((unsigned char)(W >> 8));
    o.push_back((unsigned char)(W & 255));
    for (int ch = 0; ch < 4; ch++) {
      int x = 0;
      auto at = [&](int i) { return q[(size_t)i * 4 + ch]; };
      auto runAt = [&](int i) {
        int r = 1;
        while (i + r < W && r < 127 && at(i + r) == at(i)) r++;
        return r;
      };
      while (x < W) {
        const int run = runAt(x);
        if (run >= 4) {
          o.push_back((unsigned char)(128 + run));
          o.push_back(at(x));
          x += run;
          continue;
        }
        const size_t cntPos = o.size();
        o.push_back(0);
        int n = 0;
        while (x < W && n < 128 && runAt(x) < 4) {
          o.push_back(at(x));
          x++;
          n++;
        }
        o[cntPos] = (unsigned char)n;
      }
    }
  }
  return writeFile(path, o, err);
}

bool writePfmFile(const std::string& path, int W, int H, const float* rgba, std::string& err) {
  std::vector<unsigned char> o;
  putStr(o, "PF\n" + std::to_string(W) + " " + std::to_string(H) + "\n-1.0\n");
  for (int y = H - 1; y >= 0; y--)
    for (int x = 0; x < W; x++) {
      const unsigned char* b = reinterpret_cast<const unsigned char*>(rgba + ((size_t)y * W + x) * 4);
      o.insert(o.end(), b, b + 12);
    }
  return writeFile(path, o, err);
}

bool writePpmFile(const std::string& path, int W, int H, const float* rgba, std::string& err) {
  std::vector<unsigned char> o;
  putStr(o, "P6\n" + std::to_string(W) + " " + std::to_string(H) + "\n255\n");
  for (size_t i = 0; i < (size_t)W * H; i++)
    for (int c = 0; c < 3; c++) o.push_back(to8(rgba[i * 4 + c]));
  return writeFile(path, o, err);
}

void put32be(std::vector<unsigned char>& o, uint32_t v) {
  for (int k = 3; k >= 0; k--) o.push_back((unsigned char)(v >> (8 * k)));
}

void pngChunk(std::vector<unsigned char>& o, const char* type, const std::vector<unsigned char>& data) {
  put32be(o, (uint32_t)data.size());
  const size_t start = o.size();
  o.insert(o.end(), type, type + 4);
  o.insert(o.end(), data.begin(), data.end());
  put32be(o, (uint32_t)crc32(0L, o.data() + start, (uInt)(o.size() - start)));
}

bool writePngFile(const std::string& path, int W, int H, const float* rgba, std::string& err) {
  std::vector<unsigned char> raw;
  raw.reserve(((size_t)W * 3 + 1) * H);
  for (int y = 0; y < H; y++) {
    raw.push_back(0);  // filter: none
    for (int x = 0; x < W; x++)
      for (int c = 0; c < 3; c++) raw.push_back(to8(rgba[((size_t)y * W + x) * 4 + c]));
  }
  uLongf zlen = compressBound((uLong)raw.size());
  std::vector<unsigned char> z(zlen);
  if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) {
    err = "PNG compression failed";
    return false;
  }
  z.resize(zlen);
  std::vector<unsigned char> o = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  std::vector<unsigned char> ihdr;
  put32be(ihdr, (uint32_t)W);
  put32be(ihdr, (uint32_t)H);
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit RGB, deflate, no filter method, no interlace
  pngChunk(o, "IHDR", ihdr);
  pngChunk(o, "IDAT", z);
  pngChunk(o, "IEND", {});
  return writeFile(path, o, err);
}

// ---- baseline JPEG (ITU-T T.81) --------------------------------------------
// Annex K.1 example quantisation tables (row-major) and the zig-zag order.
const unsigned char kQLuma[64] = {16, 11, 10, 16, 24,  40,  51,  61,  12, 12, 14, 19, 26,  58,  60,  55,
                                  14, 13, 16, 24, 40,  57,  69,  56,  14, 17, 22, 29, 51,  87,  80,  62,
                                  18, 22, 37, 56, 68,  109, 103, 77,  24, 35, 55, 64, 81,  104, 113, 92,
                                  49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99};
const unsigned char kQChroma[64] = {17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99,
                                    24, 26, 56, 99, 99, 99, 99, 99, 47, 66, 99, 99, 99, 99, 99, 99,
                                    99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99,
                                    99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99, 99};
const unsigned char kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,
                                   12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6,  7,  14, 21, 28,
                                   35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51,
                                   58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};
// Annex K.3 example Huffman tables: code counts per length 1..16, then symbols.
const unsigned char kDcLumaBits[16] = {0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0};
const unsigned char kDcChromaBits[16] = {0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0};
const unsigned char kDcVals[12] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11};
const unsigned char kAcLumaBits[16] = {0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d};
const unsigned char kAcLumaVals[162] = {
    0x01, 0x02, 0x03, 0x00, 0x04, 0x11, 0x05, 0x12, 0x21, 0x31, 0x41, 0x06, 0x13, 0x51, 0x61, 0x07, 0x22, 0x71,
    0x14, 0x32, 0x81, 0x91, 0xa1, 0x08, 0x23, 0x42, 0xb1, 0xc1, 0x15, 0x52, 0xd1, 0xf0, 0x24, 0x33, 0x62, 0x72,
    0x82, 0x09, 0x0a, 0x16, 0x17, 0x18, 0x19, 0x1a, 0x25, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x34, 0x35, 0x36, 0x37,
    0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58, 0x59,
    0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a, 0x83,
    0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a, 0xa2, 0xa3,
    0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba, 0xc2, 0xc3,
    0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda, 0xe1, 0xe2,
    0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf1, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};
const unsigned char kAcChromaBits[16] = {0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77};
const unsigned char kAcChromaVals[162] = {
    0x00, 0x01, 0x02, 0x03, 0x11, 0x04, 0x05, 0x21, 0x31, 0x06, 0x12, 0x41, 0x51, 0x07, 0x61, 0x71, 0x13, 0x22,
    0x32, 0x81, 0x08, 0x14, 0x42, 0x91, 0xa1, 0xb1, 0xc1, 0x09, 0x23, 0x33, 0x52, 0xf0, 0x15, 0x62, 0x72, 0xd1,
    0x0a, 0x16, 0x24, 0x34, 0xe1, 0x25, 0xf1, 0x17, 0x18, 0x19, 0x1a, 0x26, 0x27, 0x28, 0x29, 0x2a, 0x35, 0x36,
    0x37, 0x38, 0x39, 0x3a, 0x43, 0x44, 0x45, 0x46, 0x47, 0x48, 0x49, 0x4a, 0x53, 0x54, 0x55, 0x56, 0x57, 0x58,
    0x59, 0x5a, 0x63, 0x64, 0x65, 0x66, 0x67, 0x68, 0x69, 0x6a, 0x73, 0x74, 0x75, 0x76, 0x77, 0x78, 0x79, 0x7a,
    0x82, 0x83, 0x84, 0x85, 0x86, 0x87, 0x88, 0x89, 0x8a, 0x92, 0x93, 0x94, 0x95, 0x96, 0x97, 0x98, 0x99, 0x9a,
    0xa2, 0xa3, 0xa4, 0xa5, 0xa6, 0xa7, 0xa8, 0xa9, 0xaa, 0xb2, 0xb3, 0xb4, 0xb5, 0xb6, 0xb7, 0xb8, 0xb9, 0xba,
    0xc2, 0xc3, 0xc4, 0xc5, 0xc6, 0xc7, 0xc8, 0xc9, 0xca, 0xd2, 0xd3, 0xd4, 0xd5, 0xd6, 0xd7, 0xd8, 0xd9, 0xda,
    0xe2, 0xe3, 0xe4, 0xe5, 0xe6, 0xe7, 0xe8, 0xe9, 0xea, 0xf2, 0xf3, 0xf4, 0xf5, 0xf6, 0xf7, 0xf8, 0xf9, 0xfa};

struct HuffTable {
  uint16_t code[256];
  unsigned char len[256];
};

// Code assignment of Annex C: canonical codes in order of length.
HuffTable buildHuff(const unsigned char* bits, const unsigned char* vals) {
  HuffTable t;
  std::memset(&t, 0, sizeof(t));
  int code = 0, k = 0;
  for (int l = 1; l <= 16; l++) {
    for (int i = 0; i < bits[l - 1]; i++) {
      t.code[vals[k]] = (uint16_t)code;
      t.len[vals[k]] = (unsigned char)l;
      k++;
      code++;
    }
    code <<= 1;
  }
  return t;
}

struct BitWriter {
  std::vector<unsigned char>& o;
  uint32_t acc = 0;
  int n = 0;
  explicit BitWriter(std::vector<unsigned char>& out) : o(out) {}
  void put(uint32_t bits, int len) {
    for (int i = len - 1; i >= 0; i--) {
      acc = (acc << 1) | ((bits >> i) & 1u);
      if (++n == 8) {
        o.push_back((unsigned char)acc);
        if (acc == 0xFF) o.push_back(0);  // byte stuffing
        acc = 0;
        n = 0;
      }
    }
  }
  void flush() {
    while (n != 0) put(1, 1);  // pad with 1 bits
  }
};

inline int bitLength(int v) {
  v = v < 0 ? -v : v;
  int n = 0;
  while (v) {
    n++;
    v >>= 1;
  }
  return n;
}

void encodeBlock(BitWriter& bw, const float blk[64], const float qdiv[64], int& prevDc, const HuffTable& dc,
                 const HuffTable& ac) {
  // forward DCT-II: F(u,v) = 1/4 C(u) C(v) sum f(x,y) cos((2x+1)u pi/16) cos((2y+1)v pi/16)
  static float cosT[8][8];
  static bool init = false;
  if (!init) {
    for (int x = 0; x < 8; x++)
      for (int u = 0; u < 8; u++) cosT[x][u] = (float)std::cos((2 * x + 1) * u * 3.14159265358979323846 / 16.0);
    init = true;
  }
  float tmp[64], F[64];
  for (int y = 0; y < 8; y++)
    for (int u = 0; u < 8; u++) {
      float s = 0.0f;
      for (int x = 0; x < 8; x++) s += blk[y * 8 + x] * cosT[x][u];
      tmp[y * 8 + u] = s * (u == 0 ? 0.70710678f : 1.0f);
    }
  for (int v = 0; v < 8; v++)
    for (int u = 0; u < 8; u++) {
      float s = 0.0f;
      for (int y = 0; y < 8; y++) s += tmp[y * 8 + u] * cosT[y][v];
      F[v * 8 + u] = 0.25f * s * (v == 0 ? 0.70710678f : 1.0f);
    }
  int q[64];
  for (int k = 0; k < 64; k++) q[k] = (int)std::lround(F[kZigzag[k]] / qdiv[kZigzag[k]]);
  const int diff = q[0] - prevDc;
  prevDc = q[0];
  const int dcat = bitLength(diff);
  bw.put(dc.code[dcat], dc.len[dcat]);
  if (dcat) bw.put((uint32_t)(diff < 0 ? diff - 1 : diff) & ((1u << dcat) - 1u), dcat);
  int run = 0;
  for (int k = 1; k < 64; k++) {
    if (q[k] == 0) {
      run++;
      continue;
    }
    while (run > 15) {
      bw.put(ac.code[0xF0], ac.len[0xF0]);  // ZRL
      run -= 16;
    }
    const int cat = bitLength(q[k]);
    const int sym = (run << 4) | cat;
    bw.put(ac.code[sym], ac.len[sym]);
    bw.put((uint32_t)(q[k] < 0 ? q[k] - 1 : q[k]) & ((1u << cat) - 1u), cat);
    run = 0;
  }
  if (run > 0) bw.put(ac.code[0x00], ac.len[0x00]);  // EOB
}

bool writeJpegFile(const std::string& path, int W, int H, const float* rgba, int quality, std::string& err) {
  if (W > 65535 || H > 65535) {
    err = "JPEG dimensions above 65535";
    return false;
  }
  quality = std::min(100, std::max(1, quality));
  const int scale = quality < 50 ? 5000 / quality : 200 - 2 * quality;  // IJG quality scaling
  unsigned char ql[64], qc[64];
  float dl[64], dcq[64];
  for (int i = 0; i < 64; i++) {
    ql[i] = (unsigned char)std::min(255, std::max(1, (kQLuma[i] * scale + 50) / 100));
    qc[i] = (unsigned char)std::min(255, std::max(1, (kQChroma[i] * scale + 50) / 100));
    dl[i] = (float)ql[i];
    dcq[i] = (float)qc[i];
  }
  std::vector<unsigned char> o = {0xFF, 0xD8};  // SOI
  // APP0 JFIF 1.01, no density units, no thumbnail
  o.insert(o.end(), {0xFF, 0xE0, 0, 16, 'J', 'F', 'I', 'F', 0, 1, 1, 0, 0, 1, 0, 1, 0, 0});
  // DQT: two 8-bit tables in zig-zag order
  o.insert(o.end(), {0xFF, 0xDB, 0, 132, 0x00});
  for (int k = 0; k < 64; k++) o.push_back(ql[kZigzag[k]]);
  o.push_back(0x01);
  for (int k = 0; k < 64; k++) o.push_back(qc[kZigzag[k]]);
  // SOF0: 8-bit, H x W, three components sampled 1x1
  o.insert(o.end(), {0xFF, 0xC0, 0, 17, 8, (unsigned char)(H >> 8), (unsigned char)(H & 255),
                     (unsigned char)(W >> 8), (unsigned char)(W & 255), 3, 1, 0x11, 0, 2, 0x11, 1, 3, 0x11, 1});
  // DHT: the four example tables
  auto dht = [&](unsigned char tc, const unsigned char* bits, const unsigned char* vals) {
    int nv = 0;
    for (int i = 0; i < 16; i++) nv += bits[i];
    const int len = 2 + 1 + 16 + nv;
    o.insert(o.end(), {0xFF, 0xC4, (unsigned char)(len >> 8), (unsigned char)(len & 255), tc});
    o.insert(o.end(), bits, bits + 16);
    o.insert(o.end(), vals, vals + nv);
  };
  dht(0x00, kDcLumaBits, kDcVals);
  dht(0x10, kAcLumaBits, kAcLumaVals);
  dht(0x01, kDcChromaBits, kDcVals);
  dht(0x11, kAcChromaBits, kAcChromaVals);
  // SOS: three components, full spectral range
  o.insert(o.end(), {0xFF, 0xDA, 0, 12, 3, 1, 0x00, 2, 0x11, 3, 0x11, 0, 63, 0});
  const HuffTable dcL = buildHuff(kDcLumaBits, kDcVals), acL = buildHuff(kAcLumaBits, kAcLumaVals);
  const HuffTable dcC = buildHuff(kDcChromaBits, kDcVals), acC = buildHuff(kAcChromaBits, kAcChromaVals);
  BitWriter bw(o);
  int prev[3] = {0, 0, 0};
  float Y[64], Cb[64], Cr[64];
  for (int by = 0; by < H; by += 8)
    for (int bx = 0; bx < W; bx += 8) {
      for (int j = 0; j < 64; j++) {
        const int x = std::min(bx + (j & 7), W - 1), y = std::min(by + (j >> 3), H - 1);  // replicate edges
        const float* p = rgba + ((size_t)y * W + x) * 4;
        const float r = to8(p[0]), g = to8(p[1]), b = to8(p[2]);
        // JFIF RGB -> YCbCr, level-shifted by -128
        Y[j] = 0.299f * r + 0.587f * g + 0.114f * b - 128.0f;
        Cb[j] = -0.168736f * r - 0.331264f * g + 0.5f * b;
        Cr[j] = 0.5f * r - 0.418688f * g - 0.081312f * b;
      }
      encodeBlock(bw, Y, dl, prev[0], dcL, acL);
      encodeBlock(bw, Cb, dcq, prev[1], dcC, acC);
      encodeBlock(bw, Cr, dcq, prev[2], dcC, acC);
    }
  bw.flush();
  o.insert(o.end(), {0xFF, 0xD9});  // EOI
  return writeFile(path, o, err);
}

}  // namespace

bool writeImageFile(const std::string& path, int W, int H, const float* rgba, std::string& err) {
  if (W <= 0 || H <= 0 || !rgba) {
    err = "empty image";
    return false;
  }
  const size_t dot = path.find_last_of('.');
  std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
  for (char& c : ext) c = (char)std::tolower((unsigned char)c);
  if (ext == "hdr") return writeRgbe(path, W, H, rgba, err);
  if (ext == "pfm") return writePfmFile(path, W, H, rgba, err);
  if (ext == "ppm") return writePpmFile(path, W, H, rgba, err);
  if (ext == "png") return writePngFile(path, W, H, rgba, err);
  if (ext == "jpg" || ext == "jpeg") return writeJpegFile(path, W, H, rgba, 92, err);
  err = "unsupported output format (.hdr .pfm .ppm .png .jpg): " + path;
  return false;
}

}  // namespace rg
