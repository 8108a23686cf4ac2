// Reference kernel `march` (ForwardProjectionRayMarcher_TL.cu), host-compiled.
#include "ref_launch.h"
namespace ref_fp {
ESB_REF_USING
#include "ForwardProjectionRayMarcher_TL.cu"
}

extern "C" int ref_march(const RefGeom* g, const float* vol, int W, int H, float* proj, float* dist, int weight8,
                         int nthreads) {
  ESB_REF_SET_CONSTANTS(ref_fp, *g, false);
  EsbSoftTexture t;
  t.data = vol;
  t.dims = 3;
  t.nx = (int)g->dim[0];
  t.ny = (int)g->dim[1];
  t.nz = (int)g->dim[2];
  t.weight8 = weight8;
  const CUtexObject obj = (CUtexObject)(uintptr_t)&t;
  const size_t stride = (size_t)W * sizeof(float);
  esb_grid(dim3((W + 31) / 32, (H + 7) / 8), dim3(32, 8), nthreads, [&]() {
    ref_fp::march(W, H, stride, proj, dist, obj, make_int2(0, 0), make_int2(W, H));
  });
  return 0;
}
