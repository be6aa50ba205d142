// Clean-room stand-in for the reference's common-class submodule ("ucm"):
// integer type names.  TEST INFRASTRUCTURE ONLY.
#pragma once
#include <cstdint>
namespace ucm {
typedef unsigned int uint;
typedef unsigned short ushort;
typedef unsigned long ulong;
typedef unsigned char byte;
}  // namespace ucm
using namespace ucm;
