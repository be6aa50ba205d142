// Clean-room stand-in for the reference's common-class submodule ("ucm").
// TEST INFRASTRUCTURE ONLY.
#pragma once
namespace ucm {
class Stopwatch {};
}  // namespace ucm
using namespace ucm;
