// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// the space-tree templates appear only as members of the renderer class in
// the headers the harness compiles.  TEST INFRASTRUCTURE ONLY.
#pragma once

#include <vector>

#include "types3d.h"

namespace ugm {

template <class T>
struct SpaceTreeNode {
  BoundingBox bbox;
  std::vector<T> list;
  std::vector<SpaceTreeNode*> children;
};

template <class T>
struct SpaceTree {
  SpaceTreeNode<T> root;
};

}  // namespace ugm

using namespace ugm;
