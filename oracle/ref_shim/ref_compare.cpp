// Reference kernels `compare` and `cropBorder` (Compare.cu), host-compiled.
#include "ref_launch.h"
namespace ref_cmp {
ESB_REF_USING
#include "Compare.cu"
}

extern "C" int ref_compare(int W, int H, float* real, float* virt, float* dist, float realLength, const float* cut4,
                           const float* dim4, float scale) {
  const size_t stride = (size_t)W * sizeof(float);
  const float4 c = make_float4(cut4[0], cut4[1], cut4[2], cut4[3]), d = make_float4(dim4[0], dim4[1], dim4[2], dim4[3]);
  esb_grid(dim3((W + 15) / 16, (H + 15) / 16), dim3(16, 16), 1, [&]() {
    ref_cmp::compare(W, H, stride, real, virt, dist, realLength, c, d, scale);
  });
  return 0;
}

extern "C" int ref_crop_border(int W, int H, float* img, const float* cut2, const float* dim2, const int* p) {
  const size_t stride = (size_t)W * sizeof(float);
  esb_grid(dim3((W + 15) / 16, (H + 15) / 16), dim3(16, 16), 1, [&]() {
    ref_cmp::cropBorder(W, H, stride, img, make_float2(cut2[0], cut2[1]), make_float2(dim2[0], dim2[1]),
                        make_int2(p[0], p[1]), make_int2(p[2], p[3]), make_int2(p[4], p[5]), make_int2(p[6], p[7]));
  });
  return 0;
}
