// Reference kernels `wbpWeighting`, `fourierFilter`, `doseWeighting` and
// `rot3d` (wbpWeighting.cu), host-compiled.
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

// Kernel `rot3d` as RotKernel::operator() launches it (Kernels.cpp:1338-1381):
// 8^3 blocks over the size^3 output, the input bound to `texVol` (linear
// filtering, clamp addressing). The kernel has no bounds check: size must be
// a multiple of 8.
extern "C" int ref_rot3d(const float* in, float* out, int size, const float* rot, int weight8, int nthreads) {
  if (size <= 0 || size % 8) return 1;
  EsbSoftTexture t;
  t.data = in;
  t.dims = 3;
  t.nx = t.ny = t.nz = size;
  t.linear = 1;
  t.weight8 = weight8;
  ref_wbp::texVol.bound = &t;
  const float3 r0 = make_float3(rot[0], rot[1], rot[2]), r1 = make_float3(rot[3], rot[4], rot[5]),
               r2 = make_float3(rot[6], rot[7], rot[8]);
  esb_grid(dim3(size / 8, size / 8, size / 8), dim3(8, 8, 8), nthreads,
           [&]() { ref_wbp::rot3d(size, r0, r1, r2, out); });
  return 0;
}

// Kernels of GetDisplacement (Reconstructor.cpp:1746-1960), launched as
// ConjKernel, MaxShiftKernel, MaxShiftWeightedKernel and FindPeakKernel do
// (16 x 16 blocks; Reconstructor.cpp:252-266): conjMul over the N/2+1 x N
// half spectra, the others over the N x N correlation.
extern "C" int ref_conj_mul(float* a, const float* b, int n) {
  const size_t stride = (size_t)(n / 2 + 1) * sizeof(float2);
  esb_grid(dim3((n / 2 + 1 + 15) / 16, (n + 15) / 16), dim3(16, 16), 1,
           [&]() { ref_wbp::conjMul((float2*)a, (float2*)b, stride, n); });
  return 0;
}

extern "C" int ref_max_shift(float* img, int n, int max_shift, int weighted) {
  const size_t stride = (size_t)n * sizeof(float);
  esb_grid(dim3((n + 15) / 16, (n + 15) / 16), dim3(16, 16), 1, [&]() {
    if (weighted) ref_wbp::maxShiftWeighted(img, stride, n, max_shift);
    else ref_wbp::maxShift(img, stride, n, max_shift);
  });
  return 0;
}

extern "C" int ref_find_peak(float* img, unsigned char* mask, int n, float threshold) {
  const size_t stride = (size_t)n * sizeof(float);
  esb_grid(dim3((n + 15) / 16, (n + 15) / 16), dim3(16, 16), 1,
           [&]() { ref_wbp::findPeak(img, stride, (char*)mask, (size_t)n, n, threshold); });
  return 0;
}
