// Reference kernels `backProjection` / `backProjectionFP16`
// (BackProjectionSquareOS.cu), host-compiled. The surface reference is bound
// to the volume and the texture reference to the image, as
// Reconstructor.cpp:318-327 and EmSart.cpp:420-425 bind them.
#include "ref_launch.h"
namespace kbp {
ESB_REF_USING
#include "BackProjectionSquareOS.cu"
volatile thread_local unsigned char sBuffer[2 * 8 * 16 * 4 * 16];
}

extern "C" int ref_bp(const RefGeom* g, void* vol, int fp16, const float* img, int W, int H, float lambda, int os,
                      float distMin, float distMax, int linear, int weight8, int nthreads) {
  ESB_REF_SET_CONSTANTS(kbp, *g, true);
  EsbSoftTexture t;
  t.data = img;
  t.dims = 2;
  t.nx = W;
  t.ny = H;
  t.pitch_elems = (size_t)W;
  t.linear = linear;
  t.weight8 = weight8;
  kbp::tex.bound = &t;
  kbp::surfref.data = vol;
  kbp::surfref.nx_bytes = (int)g->dim[0] * (fp16 ? 2 : 4);
  kbp::surfref.ny = (int)g->dim[1];
  kbp::surfref.nz = (int)g->dim[2];
  const int nq = g->dimXQuarter;
  dim3 block(8, 16, 4), grid((nq + 7) / 8, ((int)g->dim[1] + 15) / 16, ((int)g->dim[2] + 3) / 4);
  const float inv = 1.0f / (float)os;
  esb_grid(grid, block, nthreads, [&]() {
    if (fp16)
      kbp::backProjectionFP16(W, H, lambda, os, inv, (float*)img, W * 4, distMin, distMax);
    else
      kbp::backProjection(W, H, lambda, os, inv, (float*)img, W * 4, distMin, distMax);
  });
  return 0;
}
