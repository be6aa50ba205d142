// scene_gen.cpp - the seeded procedural scenes (cube room, heavy-geometry
// spheres, batch jobs) built on the CPU for the CPU-side timing and checking
// paths, so that those paths map no library of the tracer itself.
//
// Test and baseline infrastructure only: it links the same scene generator
// source as the tracer library (raygen-renderer_b200/csrc/rg_scene.cpp),
// compiled here by the host compiler with the same floating-point flags, so
// the arrays are identical to rg_scene_builtin's (a CPU test compares them).
#include <mutex>
#include <unordered_map>

#include "rg_host.h"

namespace {
std::mutex g_mu;
std::unordered_map<const rg_scene_desc*, rg::SceneStore*> g_stores;
}  // namespace

extern "C" int32_t og_scene_builtin(int32_t kind, uint32_t seed, const int32_t* iparams, int32_t n_iparams,
                                    rg_scene_desc** out) {
  if (!out) return RG_ERR_INVALID_ARGUMENT;
  rg::SceneStore* st = nullptr;
  const rg_status rs = rg::buildBuiltinScene(kind, seed, iparams, n_iparams, &st);
  if (rs != RG_OK) return rs;
  std::lock_guard<std::mutex> lk(g_mu);
  g_stores[&st->desc] = st;
  *out = &st->desc;
  return RG_OK;
}

extern "C" int32_t og_scene_free(rg_scene_desc* scene) {
  rg::SceneStore* st = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_stores.find(scene);
    if (it == g_stores.end()) return RG_ERR_INVALID_ARGUMENT;
    st = it->second;
    g_stores.erase(it);
  }
  delete st;
  return RG_OK;
}
