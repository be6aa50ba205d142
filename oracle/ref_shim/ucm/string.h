// Clean-room stand-in for the reference's common-class submodule ("ucm"):
// the string class is used only as a member and parameter type by the
// headers the harness compiles.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <functional>
#include <string>
#include "types.h"
namespace ucm {
class string : public std::string {
 public:
  using std::string::string;
  string() = default;
  string(const std::string& s) : std::string(s) {}
};
}  // namespace ucm
using namespace ucm;
