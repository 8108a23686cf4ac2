// Reference kernel `ctf` (ctf.cu), host-compiled, with the constants of
// SetConstantValues(CTFKernel, ...) (Kernels.cpp:1104-1131) and the unit
// conversions of CTFKernel::operator() (Kernels.cpp:395-436).
#include "ref_launch.h"
namespace kctf {
ESB_REF_USING
#include "ctf.cu"
}
#undef h
#undef c
#undef Cs
#undef Cc
#undef PhaseShift
#undef EnergySpread
#undef E0
#undef RelativisticCorrectionFactor
#undef H
#undef a1
#undef a2
#undef b1
#undef b2
#undef lambda

extern "C" int ref_ctf(float* spec, int n, float defocusMin_nm, float defocusMax_nm, float angle_deg, int applyForFP,
                       int phaseFlipOnly, float wiener, const float* beta, float cs_mm, float voltage_kv,
                       float ampContrast, float pixelsize_nm) {
  using namespace kctf;
  c_cs = cs_mm;
  c_voltage = voltage_kv;
  c_openingAngle = 0.01f;
  c_ampContrast = ampContrast;
  c_phaseContrast = sqrtf(1 - ampContrast * ampContrast);
  float ps = pixelsize_nm * powf(10, -9);
  c_pixelsize = ps;
  c_pixelcount = (float)n;
  float maxFreq = 1.0 / (ps * 2.0f);
  c_maxFreq = maxFreq;
  c_freqStepSize = maxFreq / ((float)n / 2.0f);
  c_applyScatteringProfile = 0;
  c_applyEnvelopeFunction = 0;
  const float d0 = defocusMin_nm * 0.000000001f, d1 = defocusMax_nm * 0.000000001f;
  const float ang = angle_deg / 180.0f * (float)3.14159265358979323846;
  const size_t stride = (size_t)(n / 2 + 1) * sizeof(cuComplex);
  const float4 b = make_float4(beta[0], beta[1], beta[2], beta[3]);
  esb_grid(dim3((n / 2 + 1 + 15) / 16, (n + 15) / 16), dim3(16, 16), 1, [&]() {
    kctf::ctf((cuComplex*)spec, stride, d0, d1, ang, applyForFP != 0, phaseFlipOnly != 0, wiener, b);
  });
  return 0;
}
