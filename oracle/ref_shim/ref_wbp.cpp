// Reference kernels `wbpWeighting`, `fourierFilter`, `doseWeighting`
// (wbpWeighting.cu), host-compiled.
#include "ref_launch.h"
namespace ref_wbp {
ESB_REF_USING
#include "wbpWeighting.cu"
}

extern "C" int ref_wbp_weighting(float* spec, int n, float psi_deg, int fm) {
  // WbpWeightingKernel::operator(): angle = -psi / 180 * pi (Kernels.cpp:456)
  const float ang = -psi_deg / 180.0f * (float)3.14159265358979323846;
  const size_t stride = (size_t)(n / 2 + 1) * sizeof(cuComplex);
  esb_grid(dim3((n / 2 + 1 + 15) / 16, (n + 15) / 16), dim3(16, 16), 1, [&]() {
    ref_wbp::wbpWeighting((cuComplex*)spec, stride, (unsigned)n, ang, (ref_wbp::FilterMethod)fm);
  });
  return 0;
}

extern "C" int ref_fourier_filter(float* spec, int n, float lp, float hp, float lps, float hps) {
  const size_t stride = (size_t)(n / 2 + 1) * sizeof(float2);
  esb_grid(dim3((n / 2 + 1 + 15) / 16, (n + 15) / 16), dim3(16, 16), 1, [&]() {
    ref_wbp::fourierFilter((float2*)spec, stride, n, lp, hp, lps, hps);
  });
  return 0;
}

extern "C" int ref_dose_weighting(float* spec, int n, float dose, float pixelsize) {
  const size_t stride = (size_t)(n / 2 + 1) * sizeof(float2);
  esb_grid(dim3((n / 2 + 1 + 15) / 16, (n + 15) / 16), dim3(16, 16), 1, [&]() {
    ref_wbp::doseWeighting((float2*)spec, stride, n, dose, pixelsize);
  });
  return 0;
}
