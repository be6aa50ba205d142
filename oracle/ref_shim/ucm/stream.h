// Clean-room stand-in for the reference's common-class submodule ("ucm").
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "types.h"
namespace ucm {
class Stream {};
class FileStream : public Stream {};
class MemoryStream : public Stream {};
}  // namespace ucm
using namespace ucm;
