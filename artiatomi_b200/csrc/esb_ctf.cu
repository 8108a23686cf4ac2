// The Fourier-space CTF filters of the reconstruction path: kernel `ctf`
// (ctf.cu:82-240) on one spectrum, on a stack of slab spectra in place, and
// on one spectrum for several defocus ranges. Built with the compiler's
// default contraction of multiply-adds, as nvcc builds the reference's
// kernel (the other image kernels keep the reference's uncontracted order);
// the results agree with the reference's kernel to float rounding.
#include <math.h>

#include "esb_device.cuh"

namespace esb {

namespace {
inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }
}  // namespace

// The `ctf` kernel on `count` spectra in place, spectrum k with the defocus
// range of slab k (same expressions as k_ctf).
__global__ void k_ctf_batch(float2* __restrict__ spec, size_t spec_stride, int n, CtfConst k, CtfSlabs slabs,
                            float angle, int applyForFP, int phaseFlipOnly, float wiener, float4 beta) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= (unsigned)(n / 2 + 1) || y >= (unsigned)n) return;
  const float PI = 3.14159265358979323846f;
  float xpos = (float)x, ypos = (float)y;
  if (ypos > k.pixelcount * 0.5f) ypos = (k.pixelcount - ypos) * -1.0f;
  float alpha = (xpos == 0.f) ? (PI * 0.5f) : atan2f(ypos, xpos);
  float beta_ = alpha - angle;
  const float c2 = (1.f - cosf(2.f * beta_));
  float radius = sqrtf(xpos * xpos + ypos * ypos);
  float length = radius * k.freqStep;
  float L = k.lambda;
  const float l = length / 100000000.0f;
  const float e0 = expf(-beta.y * l - beta.z * l * l - beta.w * l * l * l);
  const size_t i = (size_t)y * (n / 2 + 1) + x;
  for (int s = 0; s < slabs.count; ++s) {
    const float d0 = slabs.d0[s], d1 = slabs.d1[s];
    float defocus = d0 + c2 * (d1 - d0);
    float m = (PI / 2.0f) * (k.cs * L * L * L * length * length * length * length - 2.f * defocus * L * length * length);
    float nn = k.phaseC * sinf(m) + k.ampC * cosf(m);
    float2 res = spec[(size_t)s * spec_stride + i];
    if (applyForFP && radius > beta.x && !phaseFlipOnly) {
      float e = fmaxf(e0, 0.01f);
      float val = nn * e;
      if (fabsf(val) < 0.0001f && val >= 0.f) val = 0.0001f;
      if (fabsf(val) < 0.0001f && val < 0.f) val = -0.0001f;
      res.x = res.x * -val;
      res.y = res.y * -val;
    }
    if (!applyForFP && radius > beta.x && !phaseFlipOnly) {
      float e = fmaxf(e0, wiener);
      float val = nn * e;
      float f = -val / (val * val + wiener);
      res.x = res.x * f;
      res.y = res.y * f;
    }
    if (phaseFlipOnly && nn >= 0.f) {
      res.x = -res.x;
      res.y = -res.y;
    }
    spec[(size_t)s * spec_stride + i] = res;
  }
}

// Kernel `ctf` (ctf.cu:82-240).
__global__ void k_ctf(float2* __restrict__ spec, int n, CtfConst k, float d0, float d1, float angle, int applyForFP,
                      int phaseFlipOnly, float wiener, float4 beta) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= (unsigned)(n / 2 + 1) || y >= (unsigned)n) return;
  const float PI = 3.14159265358979323846f;
  float xpos = (float)x, ypos = (float)y;
  if (ypos > k.pixelcount * 0.5f) ypos = (k.pixelcount - ypos) * -1.0f;
  float alpha = (xpos == 0.f) ? (PI * 0.5f) : atan2f(ypos, xpos);
  float beta_ = alpha - angle;
  float defocus = d0 + (1.f - cosf(2.f * beta_)) * (d1 - d0);
  float radius = sqrtf(xpos * xpos + ypos * ypos);
  float length = radius * k.freqStep;
  float L = k.lambda;
  float m = (PI / 2.0f) * (k.cs * L * L * L * length * length * length * length - 2.f * defocus * L * length * length);
  float nn = k.phaseC * sinf(m) + k.ampC * cosf(m);
  const size_t i = (size_t)y * (n / 2 + 1) + x;
  float2 res = spec[i];
  if (applyForFP && radius > beta.x && !phaseFlipOnly) {
    float l = length / 100000000.0f;
    float e = expf(-beta.y * l - beta.z * l * l - beta.w * l * l * l);
    e = fmaxf(e, 0.01f);
    float val = nn * e;
    if (fabsf(val) < 0.0001f && val >= 0.f) val = 0.0001f;
    if (fabsf(val) < 0.0001f && val < 0.f) val = -0.0001f;
    res.x = res.x * -val;
    res.y = res.y * -val;
  }
  if (!applyForFP && radius > beta.x && !phaseFlipOnly) {
    float l = length / 100000000.0f;
    float e = expf(-beta.y * l - beta.z * l * l - beta.w * l * l * l);
    e = fmaxf(e, wiener);
    float val = nn * e;
    float f = -val / (val * val + wiener);
    res.x = res.x * f;
    res.y = res.y * f;
  }
  if (phaseFlipOnly && nn >= 0.f) {
    res.x = -res.x;
    res.y = -res.y;
  }
  spec[i] = res;
}

// The `ctf` kernel applied to one spectrum for several defocus ranges at
// once: out + k * out_stride = ctf(in, d0[k], d1[k]). The per-frequency
// terms that do not depend on defocus are computed once; each output equals
// what k_ctf would make of a copy of `in` (same expressions, same order).
__global__ void k_ctf_slabs(const float2* __restrict__ in, float2* __restrict__ out, size_t out_stride, int n,
                            CtfConst k, CtfSlabs slabs, float angle, int applyForFP, int phaseFlipOnly, float wiener,
                            float4 beta) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= (unsigned)(n / 2 + 1) || y >= (unsigned)n) return;
  const float PI = 3.14159265358979323846f;
  float xpos = (float)x, ypos = (float)y;
  if (ypos > k.pixelcount * 0.5f) ypos = (k.pixelcount - ypos) * -1.0f;
  float alpha = (xpos == 0.f) ? (PI * 0.5f) : atan2f(ypos, xpos);
  float beta_ = alpha - angle;
  const float c2 = (1.f - cosf(2.f * beta_));
  float radius = sqrtf(xpos * xpos + ypos * ypos);
  float length = radius * k.freqStep;
  float L = k.lambda;
  const float l = length / 100000000.0f;
  const float e0 = expf(-beta.y * l - beta.z * l * l - beta.w * l * l * l);
  const size_t i = (size_t)y * (n / 2 + 1) + x;
  const float2 src = in[i];
  for (int s = 0; s < slabs.count; ++s) {
    const float d0 = slabs.d0[s], d1 = slabs.d1[s];
    float defocus = d0 + c2 * (d1 - d0);
    float m = (PI / 2.0f) * (k.cs * L * L * L * length * length * length * length - 2.f * defocus * L * length * length);
    float nn = k.phaseC * sinf(m) + k.ampC * cosf(m);
    float2 res = src;
    if (applyForFP && radius > beta.x && !phaseFlipOnly) {
      float e = fmaxf(e0, 0.01f);
      float val = nn * e;
      if (fabsf(val) < 0.0001f && val >= 0.f) val = 0.0001f;
      if (fabsf(val) < 0.0001f && val < 0.f) val = -0.0001f;
      res.x = res.x * -val;
      res.y = res.y * -val;
    }
    if (!applyForFP && radius > beta.x && !phaseFlipOnly) {
      float e = fmaxf(e0, wiener);
      float val = nn * e;
      float f = -val / (val * val + wiener);
      res.x = res.x * f;
      res.y = res.y * f;
    }
    if (phaseFlipOnly && nn >= 0.f) {
      res.x = -res.x;
      res.y = -res.y;
    }
    out[(size_t)s * out_stride + i] = res;
  }
}

cudaError_t launch_ctf_batch(float* spec, size_t spec_stride, int n, const CtfConst& k, const CtfSlabs& slabs_nm,
                             float angle_deg, int applyForFP, int phaseFlip, float wiener, float4 beta,
                             cudaStream_t st) {
  dim3 b(32, 8);
  CtfSlabs sl = slabs_nm;
  for (int i = 0; i < sl.count; ++i) {
    sl.d0[i] = slabs_nm.d0[i] * 0.000000001f;
    sl.d1[i] = slabs_nm.d1[i] * 0.000000001f;
  }
  float ang = angle_deg / 180.0f * 3.14159265358979323846f;
  k_ctf_batch<<<grid2(n / 2 + 1, n, b), b, 0, st>>>((float2*)spec, spec_stride / 2, n, k, sl, ang, applyForFP,
                                                    phaseFlip, wiener, beta);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

CtfConst make_ctf_const(int n, float cs_mm, float voltage_kv, float amp_contrast, float pixel_size_nm) {
  // SetConstantValues(CTFKernel, ...) (Kernels.cpp:1104-1131) and the
  // wavelength macro of ctf.cu:62.
  CtfConst k;
  float pixelsize = pixel_size_nm * powf(10.0f, -9.0f);
  k.pixelcount = (float)n;
  float maxFreq = (float)(1.0 / (pixelsize * 2.0f));
  k.freqStep = maxFreq / (k.pixelcount / 2.0f);
  k.ampC = amp_contrast;
  k.phaseC = sqrtf(1.0f - amp_contrast * amp_contrast);
  float hc = ((float)6.63E-34) * ((float)3.00E+08);
  double X = (double)(2 * 511 * voltage_kv * 1000.0f * 1000.0f) + (double)(voltage_kv * voltage_kv * 1000.0f * 1000.0f);
  k.lambda = hc / (float)sqrt((float)(X * 1.602E-19 * 1.602E-19));
  k.cs = cs_mm * 0.001f;
  return k;
}

cudaError_t launch_ctf(float* spec, int n, const CtfConst& k, float d0_nm, float d1_nm, float angle_deg,
                       int applyForFP, int phaseFlip, float wiener, float4 beta, cudaStream_t st) {
  dim3 b(32, 8);
  float d0 = d0_nm * 0.000000001f, d1 = d1_nm * 0.000000001f;
  float ang = angle_deg / 180.0f * 3.14159265358979323846f;
  k_ctf<<<grid2(n / 2 + 1, n, b), b, 0, st>>>((float2*)spec, n, k, d0, d1, ang, applyForFP, phaseFlip, wiener, beta); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

// out_stride: floats between output spectra (even: whole complex values).
cudaError_t launch_ctf_slabs(const float* in, float* out, size_t out_stride, int n, const CtfConst& k,
                             const CtfSlabs& slabs_nm, float angle_deg, int applyForFP, int phaseFlip, float wiener,
                             float4 beta, cudaStream_t st) {
  dim3 b(32, 8);
  CtfSlabs sl = slabs_nm;
  for (int i = 0; i < sl.count; ++i) {
    sl.d0[i] = slabs_nm.d0[i] * 0.000000001f;
    sl.d1[i] = slabs_nm.d1[i] * 0.000000001f;
  }
  float ang = angle_deg / 180.0f * 3.14159265358979323846f;
  k_ctf_slabs<<<grid2(n / 2 + 1, n, b), b, 0, st>>>((const float2*)in, (float2*)out, out_stride / 2, n, k, sl, ang,
                                                    applyForFP, phaseFlip, wiener, beta); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace esb
