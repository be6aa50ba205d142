// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// the umbrella header (it makes the ugm names visible unqualified, as the
// reference's headers expect).  TEST INFRASTRUCTURE ONLY.
#pragma once
#include "color.h"
#include "functions.h"
#include "image.h"
#include "matrix.h"
#include "types2d.h"
#include "types3d.h"
