// rg_json.cpp - reference scene JSON loader (placeholder until the loader lands).
#include "rg_host.h"

namespace rg {

rg_status loadSceneJson(const char* path, SceneStore** out, std::string& err) {
  (void)path;
  *out = nullptr;
  err = "scene JSON loading is not built yet";
  return RG_ERR_UNSUPPORTED;
}

}  // namespace rg
