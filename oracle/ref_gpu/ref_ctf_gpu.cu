// The reference's kernel `ctf` (src/EmSART/cuda_kernels/ctf.cu, included
// unmodified from the reference tree) built for the GPU, with a C launcher
// that sets its constants as SetConstantValues(CTFKernel, ...) does
// (Kernels.cpp:1104-1131) and converts units as CTFKernel::operator() does
// (Kernels.cpp:395-436), on 16 x 16 blocks (CTFKernel(CUmodule),
// Kernels.cpp:388-392). TEST INFRASTRUCTURE: the only kernel of the
// reference's EmSART path that compiles with CUDA 12; the GPU tests compare
// the library's CTF filter with it, result and time.
#include "ctf.cu"

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

#include <cuda_runtime.h>

// spec: device, n x (n/2 + 1) complex; set_constants: upload the kernel's
// constants first (the reference sets them once per projection); returns a
// cudaError_t.
extern "C" int ref_ctf_gpu(float* spec, int n, float defocusMin_nm, float defocusMax_nm, float angle_deg,
                           int applyForFP, int phaseFlipOnly, float wiener, const float* beta, float cs_mm,
                           float voltage_kv, float ampContrast, float pixelsize_nm, int set_constants,
                           void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  const float openingAngle = 0.01f;
  const float phaseContrast = sqrtf(1 - ampContrast * ampContrast);
  const float ps = pixelsize_nm * powf(10, -9);
  const float count = (float)n;
  const float maxFreq = 1.0 / (ps * 2.0f);
  const float step = maxFreq / (count / 2.0f);
  const float zero = 0.0f;
  cudaError_t e = cudaSuccess;
#define ESB_SET(sym, val)                                                                        \
  if (set_constants && e == cudaSuccess)                                                               \
    e = cudaMemcpyToSymbolAsync(sym, &(val), sizeof(float), 0, cudaMemcpyHostToDevice, st)
  ESB_SET(c_cs, cs_mm);
  ESB_SET(c_voltage, voltage_kv);
  ESB_SET(c_openingAngle, openingAngle);
  ESB_SET(c_ampContrast, ampContrast);
  ESB_SET(c_phaseContrast, phaseContrast);
  ESB_SET(c_pixelsize, ps);
  ESB_SET(c_pixelcount, count);
  ESB_SET(c_maxFreq, maxFreq);
  ESB_SET(c_freqStepSize, step);
  ESB_SET(c_applyScatteringProfile, zero);
  ESB_SET(c_applyEnvelopeFunction, zero);
#undef ESB_SET
  if (e != cudaSuccess) return (int)e;
  const float d0 = defocusMin_nm * 0.000000001f, d1 = defocusMax_nm * 0.000000001f;
  const float ang = angle_deg / 180.0f * (float)3.14159265358979323846;
  const size_t stride = (size_t)(n / 2 + 1) * sizeof(cuComplex);
  const float4 b = make_float4(beta[0], beta[1], beta[2], beta[3]);
  dim3 blk(16, 16), grd((n / 2 + 1 + 15) / 16, (n + 15) / 16);
  ctf<<<grd, blk, 0, st>>>((cuComplex*)spec, stride, d0, d1, ang, applyForFP != 0, phaseFlipOnly != 0, wiener, b);
  return (int)cudaGetLastError();
}
