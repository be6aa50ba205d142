// Clean-room stand-in for the reference's graphics-math submodule ("ugm"):
// the image classes only appear as members and parameters in the headers the
// harness compiles; none of their pixels is read.  TEST INFRASTRUCTURE ONLY.
#pragma once

#include <vector>

#include "color.h"
#include "types2d.h"

namespace ugm {

class Image {
 public:
  int width() const { return w_; }
  int height() const { return h_; }
  void createEmpty(int w, int h) {
    w_ = w;
    h_ = h;
    px_.assign((size_t)w * h * 4, 0.0f);
  }

 private:
  int w_ = 0, h_ = 0;
  std::vector<float> px_;
};
typedef Image Image4f;
typedef Image Image3f;

}  // namespace ugm

using namespace ugm;
