// Reference kernel `makeSquare` (CopyToSquare.cu), host-compiled.
#include "ref_launch.h"
namespace ref_sq {
ESB_REF_USING
#include "CopyToSquare.cu"
}

extern "C" int ref_make_square(int W, int H, int maxsize, const float* in, float* out, int bx, int by, int mirrorY,
                               int fillZero) {
  esb_grid(dim3((maxsize + 15) / 16, (maxsize + 15) / 16), dim3(16, 16), 1, [&]() {
    ref_sq::makeSquare(W, H, maxsize, W, (float*)in, out, bx, by, mirrorY != 0, fillZero != 0);
  });
  return 0;
}
