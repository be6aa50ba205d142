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

bool readImageFile(const std::string& path, TextureStore& out, std::string& err) {
  const size_t dot = path.find_last_of('.');
  std::string ext = dot == std::string::npos ? "" : path.substr(dot + 1);
  for (char& c : ext) c = (char)std::tolower((unsigned char)c);
  if (ext == "hdr") return readRadianceHdr(path, out, err);
  if (ext == "pfm") return readPfm(path, out, err);
  err = "unsupported image format (Radiance .hdr and .pfm are read): " + path;
  return false;
}

}  // namespace rg
