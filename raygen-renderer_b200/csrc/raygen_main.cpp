// raygen_main.cpp - the `raygen render <scene.json> [options]` command.
//
// Same command and flags as the reference CLI (src/main.cpp:162-489):
// -o, -r W,H | WxH | N, -s, -c, -d, -enaa, -encs, -enpp, -endn, -dni, -enad,
// --adaptive-base, --adaptive-threshold, -bl*, -cb, -bc, -wc, --dump;
// unknown flags print "unknown argument" and return 1.  Tracer knobs added:
// --seed, --max-depth, --rr-depth, --light-pick-fix, --adaptive-mode pixel|tile,
// --bvh-bins.  A scene path of the form builtin:<kind>[:<seed>] renders one of
// the procedural workloads.  Output (rg_save_image): .hdr (Radiance RGBE) and
// .pfm hold the linear HDR result; .jpg (the default, <scene dir>/<base>.jpg
// as in the reference), .png and .ppm the tonemapped image.
#include <cctype>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "raygen_b200.h"

namespace {

bool parseBool(const char* s) {
  return !(std::strcmp(s, "false") == 0 || std::strcmp(s, "0") == 0 || std::strcmp(s, "no") == 0 ||
           std::strcmp(s, "off") == 0);
}

std::string ext(const std::string& p) {
  const size_t d = p.find_last_of('.');
  if (d == std::string::npos) return "";
  std::string e = p.substr(d + 1);
  for (auto& c : e) c = (char)std::tolower(c);
  return e;
}

void progress(float p, void*) {
  std::printf("\rrendering... %d%% ", (int)(p * 100.0f));
  std::fflush(stdout);
}

}  // namespace

int main(int argc, const char* argv[]) {
  if (argc < 2) {
    std::printf("usage: raygen <command> [scene.json|arguments...]\n");
    return 0;
  }
  rg_settings rs;
  rg_settings_default(&rs);
  std::string cmd, scene, out;
  bool dump = false;
  for (int i = 1; i < argc; i++) {
    const char* a = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) {
        std::printf("missing value for %s\n", a);
        std::exit(1);
      }
      return argv[++i];
    };
    auto is = [&](const char* s) { return std::strcmp(a, s) == 0; };
    if (a[0] == '-') {
      if (is("-o")) out = next();
      else if (is("-r") || is("--resolution")) {
        const char* v = next();
        int w = rs.resolution_width, h = rs.resolution_height;
        int n = std::sscanf(v, "%d,%d", &w, &h);
        if (n < 2) n = std::sscanf(v, "%dx%d", &w, &h);
        if (n == 1) { rs.resolution_width = w; rs.resolution_height = w; }
        else if (n == 2) { rs.resolution_width = w; rs.resolution_height = h; }
      } else if (is("--dump")) dump = true;
      else if (is("-ver") || is("--ver") || is("--version")) { std::printf("%s\n", rg_version()); return 0; }
      else if (is("-h") || is("--help")) {
        std::printf("%s\nusage: ./raygen render <scene.json> [parameters...]\n", rg_version());
        return 0;
      }
      else if (is("-s") || is("--samples")) rs.samples = std::atoi(next());
      else if (is("-c") || is("--threads") || is("--cores")) rs.threads = std::atoi(next());
      else if (is("-enaa") || is("--enable-antialias")) rs.enable_antialias = parseBool(next());
      else if (is("-encs") || is("--enable-color-sampling")) rs.enable_color_sampling = parseBool(next());
      else if (is("-enpp") || is("--enable-postprocess")) rs.enable_rendering_postprocess = parseBool(next());
      else if (is("-endn") || is("--enable-denoise")) rs.enable_denoise = parseBool(next());
      else if (is("-dni") || is("--denoise-intensity")) rs.denoise_intensity = (float)std::atof(next());
      else if (is("-enad") || is("--enable-adaptive")) rs.enable_adaptive_sampling = parseBool(next());
      else if (is("--adaptive-base")) rs.adaptive_base_samples = std::atoi(next());
      else if (is("--adaptive-threshold")) rs.adaptive_threshold = (float)std::atof(next());
      else if (is("-blth") || is("--bloom-threshold")) rs.bloom_threshold = (float)std::atof(next());
      else if (is("-blst") || is("--bloom-strength")) rs.bloom_strength = (float)std::atof(next());
      else if (is("-blcv") || is("--bloom-curve")) rs.bloom_curve = (float)std::atof(next());
      else if (is("-blrd") || is("--bloom-radius")) rs.bloom_radius = (float)std::atof(next());
      else if (is("-d") || is("--shader")) rs.shader_provider = std::atoi(next());
      else if (is("-cb") || is("--cullback")) rs.cull_back_face = parseBool(next());
      else if (is("-bc") || is("--backcolor")) {
        float c[4] = {rs.back_color[0], rs.back_color[1], rs.back_color[2], rs.back_color[3]};
        if (std::sscanf(next(), "%f,%f,%f,%f", &c[0], &c[1], &c[2], &c[3]) == 3) c[3] = 1.0f;
        for (int k = 0; k < 4; k++) rs.back_color[k] = c[k];
      } else if (is("-wc") || is("--worldcolor")) {
        float c[4] = {rs.world_color[0], rs.world_color[1], rs.world_color[2], 1.0f};
        std::sscanf(next(), "%f,%f,%f,%f", &c[0], &c[1], &c[2], &c[3]);
        for (int k = 0; k < 3; k++) rs.world_color[k] = c[k];
      } else if (is("--seed")) rs.seed = (uint32_t)std::strtoul(next(), nullptr, 10);
      else if (is("--max-depth")) rs.max_depth = std::atoi(next());
      else if (is("--rr-depth")) rs.rr_depth = std::atoi(next());
      else if (is("--light-pick-fix")) rs.light_pick_fix = parseBool(next());
      else if (is("--bvh-bins")) rs.bvh_bins = std::atoi(next());
      else if (is("--adaptive-mode")) rs.adaptive_mode = std::strcmp(next(), "pixel") == 0 ? RG_ADAPTIVE_PIXEL : RG_ADAPTIVE_TILE;
      else {
        std::printf("unknown argument: %s\n", a);
        return 1;
      }
    } else if (cmd.empty()) {
      cmd = a;
    } else if (scene.empty()) {
      scene = a;
    } else {
      std::printf("unknown argument: %s\n", a);
      return 1;
    }
  }
  if (cmd.empty()) { std::printf("raygen: no command specified.\n"); return 1; }
  if (cmd != "render") { std::printf("raygen: only the render command is supported\n"); return 1; }
  if (scene.empty()) { std::printf("raygen: no input file specified.\n"); return 1; }
  rg_scene_desc* desc = nullptr;
  rg_status st;
  if (scene.rfind("builtin:", 0) == 0) {
    int kind = 1;
    unsigned seed = 1;
    std::sscanf(scene.c_str() + 8, "%d:%u", &kind, &seed);
    st = rg_scene_builtin(kind, seed, nullptr, 0, &desc);
  } else {
    st = rg_load_scene_json(scene.c_str(), &desc);
  }
  if (st != RG_OK) {
    std::printf("raygen: cannot load scene %s: %s\n", scene.c_str(), rg_last_error());
    return 1;
  }
  if (out.empty()) {
    std::string base = scene;
    const size_t d = base.find_last_of('.');
    if (d != std::string::npos && base.find('/', d) == std::string::npos) base = base.substr(0, d);
    for (auto& c : base) if (c == ':') c = '_';
    out = base + ".jpg";
  }
  std::printf("%s\n\n  input : %s\n  output: %s\n\n", rg_version(), scene.c_str(), out.c_str());
  std::printf("  resolution     : %d x %d\n  shader system  : %d\n  samples        : %d\n  denoise        : %s\n\n",
              rs.resolution_width, rs.resolution_height, rs.shader_provider, rs.samples, rs.enable_denoise ? "yes" : "no");
  if (dump) std::printf("  triangles: %d  objects: %d  materials: %d\n", desc->num_triangles, desc->num_objects, desc->num_materials);
  rg_handle* h = nullptr;
  if ((st = rg_create(&rs, &h)) != RG_OK) {
    std::printf("raygen: %s\n", rg_last_error());
    return 1;
  }
  const auto t0 = std::chrono::steady_clock::now();
  if ((st = rg_set_scene(h, desc)) != RG_OK || (rg_set_progress_cb(h, progress, nullptr), (st = rg_render(h)) != RG_OK)) {
    std::printf("raygen: render failed (%d): %s\n", st, rg_last_error());
    rg_destroy(h);
    rg_scene_free(desc);
    return 1;
  }
  const auto t1 = std::chrono::steady_clock::now();
  std::vector<float> img((size_t)rs.resolution_width * rs.resolution_height * 4);
  // .hdr / .pfm: the linear HDR buffer, no tonemap (main.cpp:479-485); otherwise the LDR result
  const std::string e = ext(out);
  const bool linear = e == "hdr" || e == "pfm";
  const bool ok = (linear ? rg_get_hdr(h, img.data(), img.size()) : rg_get_ldr(h, img.data(), img.size())) == RG_OK &&
                  rg_save_image(out.c_str(), rs.resolution_width, rs.resolution_height, img.data()) == RG_OK;
  rg_stats stats;
  rg_get_stats(h, &stats);
  std::printf("\rdone. (%.3f s; trace %.1f ms, %.1f Msamples/s)\n", std::chrono::duration<double>(t1 - t0).count(),
              stats.trace_ms, stats.trace_ms > 0 ? stats.samples / (stats.trace_ms * 1e3) : 0.0);
  rg_destroy(h);
  rg_scene_free(desc);
  if (!ok) {
    std::printf("raygen: cannot write %s: %s\n", out.c_str(), rg_last_error());
    return 1;
  }
  return 0;
}
