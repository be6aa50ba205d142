// Clean-room stand-in for the reference's graphics-math submodule ("ugm").
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "types2d.h"
#include "types3d.h"
