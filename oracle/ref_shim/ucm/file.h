// Clean-room stand-in for the reference's common-class submodule ("ucm").
// TEST INFRASTRUCTURE ONLY.
#pragma once
#include "stream.h"
#include "string.h"
