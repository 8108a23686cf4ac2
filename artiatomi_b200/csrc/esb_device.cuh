// Shared device-side definitions of the EmSART B200 kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/esb.h"

namespace esb {

// Kernel-side copy of esb_constants, passed by value as a launch parameter
// (252 bytes) instead of the reference's per-symbol __constant__ writes.
struct KConst {
  float3 n, det, u, v;
  float3 bbMin, bbMax, bbRcp, dim, vs;
  float zShift;
  int dimXQuarter;
  float4 detMat[4];
  float aniso[9];
  float anisoInv[9];
};

inline KConst to_kconst(const esb_constants& c) {
  KConst k;
  k.n = make_float3(c.proj_norm[0], c.proj_norm[1], c.proj_norm[2]);
  k.det = make_float3(c.detektor[0], c.detektor[1], c.detektor[2]);
  k.u = make_float3(c.u_pitch[0], c.u_pitch[1], c.u_pitch[2]);
  k.v = make_float3(c.v_pitch[0], c.v_pitch[1], c.v_pitch[2]);
  k.bbMin = make_float3(c.bbox_min[0], c.bbox_min[1], c.bbox_min[2]);
  k.bbMax = make_float3(c.bbox_max[0], c.bbox_max[1], c.bbox_max[2]);
  k.bbRcp = make_float3(c.bbox_rcp[0], c.bbox_rcp[1], c.bbox_rcp[2]);
  k.dim = make_float3(c.volume_dim[0], c.volume_dim[1], c.volume_dim[2]);
  k.vs = make_float3(c.voxel_size[0], c.voxel_size[1], c.voxel_size[2]);
  k.zShift = c.z_shift;
  k.dimXQuarter = c.volume_dim_x_quarter;
  for (int r = 0; r < 4; ++r)
    k.detMat[r] = make_float4(c.detector_matrix[4 * r + 0], c.detector_matrix[4 * r + 1], c.detector_matrix[4 * r + 2],
                              c.detector_matrix[4 * r + 3]);
  for (int i = 0; i < 9; ++i) {
    k.aniso[i] = c.mag_aniso[i];
    k.anisoInv[i] = c.mag_aniso_inv[i];
  }
  return k;
}

// Defocus slabs of one projection (the reference's loop
// for (ray = t_in; ray < t_out; ray += thickness), Reconstructor.cpp:515,
// 935): slab k spans bound[k] <= t < bound[k+1] with the float recurrence
// bound[k+1] = bound[k] + thickness. Slab images are k * stride apart.
#define ESB_MAX_SLABS 256
struct SlabTable {
  int count;
  float bound[ESB_MAX_SLABS + 1];
};

// The subset back-projection (launch_bp_axis_set): up to ESB_BP_SET_MAX
// projections in one launch, each with up to ESB_BP_SET_MAX_SLABS CTF slabs.
#define ESB_BP_SET_MAX 8
#define ESB_BP_SET_MAX_SLABS 64

// Constants of kernel `ctf` (SetConstantValues(CTFKernel...), Kernels.cpp:1104-1131).
struct CtfConst {
  float cs, lambda, ampC, phaseC, freqStep, pixelcount;
};

// Launch shape of the single-axis back-projection: blocks of bx quads x by
// rows (bx * by <= 128), over volume planes [z0, z0 + nz) (nz = 0: to the
// end) written from plane 0 of the buffer passed.
struct BpShape {
  int bx, by, z0, nz;
};

// Every kernel launch of the library is counted (esb_kernel_launches).
void count_launch();
#define ESB_COUNT_LAUNCH() ::esb::count_launch()

// Defocus ranges of up to ESB_CTF_SLAB_BATCH slabs filtered in one launch.
#define ESB_CTF_SLAB_BATCH 16
struct CtfSlabs {
  int count;
  float d0[ESB_CTF_SLAB_BATCH], d1[ESB_CTF_SLAB_BATCH];
};

template <int VT>
struct Voxel;
template <>
struct Voxel<ESB_VOXEL_F32> {
  typedef float T;
  static __device__ __forceinline__ float load(const void* p, long i) { return __ldg((const float*)p + i); }
  static __device__ __forceinline__ float loadrw(const void* p, long i) { return ((const float*)p)[i]; }
  static __device__ __forceinline__ void store(void* p, long i, float v) { ((float*)p)[i] = v; }
};
template <>
struct Voxel<ESB_VOXEL_F16> {
  typedef __half T;
  static __device__ __forceinline__ float load(const void* p, long i) {
    return __half2float(__ldg((const __half*)p + i));
  }
  static __device__ __forceinline__ float loadrw(const void* p, long i) { return __half2float(((const __half*)p)[i]); }
  static __device__ __forceinline__ void store(void* p, long i, float v) { ((__half*)p)[i] = __float2half_rn(v); }
};
template <>
struct Voxel<ESB_VOXEL_BF16> {
  typedef __nv_bfloat16 T;
  static __device__ __forceinline__ float load(const void* p, long i) {
    return __bfloat162float(__ldg((const __nv_bfloat16*)p + i));
  }
  static __device__ __forceinline__ float loadrw(const void* p, long i) {
    return __bfloat162float(((const __nv_bfloat16*)p)[i]);
  }
  static __device__ __forceinline__ void store(void* p, long i, float v) {
    ((__nv_bfloat16*)p)[i] = __float2bfloat16_rn(v);
  }
};

// Texel index for a filtered coordinate with clamp addressing.
__device__ __forceinline__ int clamp_texel(float f, int n) {
  if (!(f > 0.0f)) return 0;
  if (f > (float)(n - 1)) return n - 1;
  return (int)f;
}

}  // namespace esb
