// Ray geometry and trilinear sampling shared by the fast forward projector
// (esb_projector_fast.cu) and its adjoint and gradients (esb_adjoint.cu).
#pragma once

#include <float.h>

#include "esb_device.cuh"

namespace esb {
namespace raycore {

// Number of samples J of the float recurrence t_{j+1} = fl(t_j + h) from t0
// with t_j <= tout, and its constant step; ok = false when the recurrence is
// not an arithmetic progression over [t0, tout].
__device__ __forceinline__ int progression(float t0, float tout, float h, float& step, bool& ok) {
  ok = true;
  step = h;
  if (!(t0 <= tout)) return 0;
  float t1 = __fadd_rn(t0, h);
  step = __fsub_rn(t1, t0);
  float t2 = __fadd_rn(t1, h);
  if (!(t0 > 0.0f) || __fsub_rn(t2, t1) != step || !(step > 0.0f)) {
    ok = false;
    return 0;
  }
  int J = (int)__fdiv_rn(__fsub_rn(tout, t0), step) + 1;
  if (J < 1) J = 1;
  while (J > 1 && __fadd_rn(t0, __fmul_rn((float)(J - 1), step)) > tout) --J;
  while (__fadd_rn(t0, __fmul_rn((float)J, step)) <= tout) ++J;
  // the last sample must stay in the binade of t0 (exact arithmetic there)
  const float tl = __fadd_rn(t0, __fmul_rn((float)(J - 1), step));
  int e0, e1;
  frexpf(t0, &e0);
  frexpf(tl, &e1);
  if (e0 != e1) ok = false;
  return J;
}

template <int VT>
struct Cell {
  const void* __restrict__ vol;
  int nx, ny, nz;
  long sy, sz;
  __device__ __forceinline__ float at(int x, int y, int z) const {
    x = x < 0 ? 0 : (x > nx - 1 ? nx - 1 : x);
    y = y < 0 ? 0 : (y > ny - 1 ? ny - 1 : y);
    z = z < 0 ? 0 : (z > nz - 1 ? nz - 1 : z);
    return Voxel<VT>::load(vol, (long)z * sz + (long)y * sy + x);
  }
};

// Trilinear sample at interpolation coordinates (x, y, z) (texel centres at
// integers), clamp addressing.
template <int VT>
__device__ __forceinline__ float trilinear(const Cell<VT>& C, float x, float y, float z) {
  float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  float a = x - fx, b = y - fy, c = z - fz;
  int ix = (int)fmaxf(fminf(fx, 1.0e9f), -1.0e9f), iy = (int)fmaxf(fminf(fy, 1.0e9f), -1.0e9f),
      iz = (int)fmaxf(fminf(fz, 1.0e9f), -1.0e9f);
  float c000 = C.at(ix, iy, iz), c100 = C.at(ix + 1, iy, iz), c010 = C.at(ix, iy + 1, iz),
        c110 = C.at(ix + 1, iy + 1, iz);
  float c001 = C.at(ix, iy, iz + 1), c101 = C.at(ix + 1, iy, iz + 1), c011 = C.at(ix, iy + 1, iz + 1),
        c111 = C.at(ix + 1, iy + 1, iz + 1);
  float ia = 1.f - a, ib = 1.f - b, ic = 1.f - c;
  return ic * (ib * (ia * c000 + a * c100) + b * (ia * c010 + a * c110)) +
         c * (ib * (ia * c001 + a * c101) + b * (ia * c011 + a * c111));
}

// Ray start and box entry/exit: the reference's expressions, operation by
// operation without contraction, so t_in/t_out (|t| ~ 1e4) and hence the
// sample positions and ray lengths equal the reference's FP32 values.
__device__ __forceinline__ float mul_add_rn(float a, float b, float c) { return __fadd_rn(__fmul_rn(a, b), c); }

__device__ __forceinline__ float3 ray_src(const KConst& c, float px, float py) {
  float xA = __fadd_rn(__fadd_rn(__fmul_rn(c.aniso[0], px), __fmul_rn(c.aniso[1], py)), __fmul_rn(c.aniso[2], 1.0f));
  float yA = __fadd_rn(__fadd_rn(__fmul_rn(c.aniso[3], px), __fmul_rn(c.aniso[4], py)), __fmul_rn(c.aniso[5], 1.0f));
  float3 s;
  s.x = mul_add_rn(yA, c.v.x, mul_add_rn(xA, c.u.x, c.det.x));
  s.y = mul_add_rn(yA, c.v.y, mul_add_rn(xA, c.u.y, c.det.y));
  s.z = mul_add_rn(yA, c.v.z, mul_add_rn(xA, c.u.z, c.det.z));
  return s;
}

__device__ __forceinline__ void hit(float3 s, float3 d, float3 lo, float3 hi, float& tin, float& tout) {
  float ex = __fdiv_rn(__fsub_rn(lo.x, s.x), d.x), ey = __fdiv_rn(__fsub_rn(lo.y, s.y), d.y),
        ez = __fdiv_rn(__fsub_rn(lo.z, s.z), d.z);
  float xx = __fdiv_rn(__fsub_rn(hi.x, s.x), d.x), xy = __fdiv_rn(__fsub_rn(hi.y, s.y), d.y),
        xz = __fdiv_rn(__fsub_rn(hi.z, s.z), d.z);
  tin = fmaxf(fmaxf(fminf(ex, xx), fminf(ey, xy)), fminf(ez, xz));
  tout = fminf(fminf(fmaxf(ex, xx), fmaxf(ey, xy)), fmaxf(ez, xz));
}

// Sum of the 4 sub-ray values of a pixel (adjacent lanes) in the reference's
// order ((v0 + v1) + v2) + v3, valid in the group's first lane.
__device__ __forceinline__ float quad_sum_ordered(float v) {
  const float v1 = __shfl_down_sync(0xffffffffu, v, 1);
  const float v2 = __shfl_down_sync(0xffffffffu, v, 2);
  const float v3 = __shfl_down_sync(0xffffffffu, v, 3);
  return __fadd_rn(__fadd_rn(__fadd_rn(v, v1), v2), v3);
}

// Interpolation coordinates (texel centres at integers) of world point p.
// Sample positions are computed with explicit roundings (no contraction left
// to the compiler), so the forward projector, its adjoint and the CPU
// oracle place every sample at the same float coordinates.
__device__ __forceinline__ float3 interp_coord(const KConst& c, float3 p) {
  return make_float3(__fsub_rn(__fmul_rn(__fmul_rn(__fsub_rn(p.x, c.bbMin.x), c.bbRcp.x), c.dim.x), 0.5f),
                     __fsub_rn(__fmul_rn(__fmul_rn(__fsub_rn(p.y, c.bbMin.y), c.bbRcp.y), c.dim.y), 0.5f),
                     __fsub_rn(__fsub_rn(__fmul_rn(__fmul_rn(__fsub_rn(p.z, c.bbMin.z), c.bbRcp.z), c.dim.z), c.zShift),
                               0.5f));
}

// World point s + t * n of a ray.
__device__ __forceinline__ float3 ray_point(const KConst& c, float3 s, float t) {
  return make_float3(__fmaf_rn(t, c.n.x, s.x), __fmaf_rn(t, c.n.y, s.y), __fmaf_rn(t, c.n.z, s.z));
}

// Per-sample step of the interpolation coordinates for a ray step `step`.
__device__ __forceinline__ float3 interp_step(const KConst& c, float step) {
  return make_float3(__fmul_rn(__fmul_rn(__fmul_rn(step, c.n.x), c.bbRcp.x), c.dim.x),
                     __fmul_rn(__fmul_rn(__fmul_rn(step, c.n.y), c.bbRcp.y), c.dim.y),
                     __fmul_rn(__fmul_rn(__fmul_rn(step, c.n.z), c.bbRcp.z), c.dim.z));
}

// Coordinate of sample j along one axis: q + j * dq, rounded once.
__device__ __forceinline__ float qpos(float q, int j, float dq) { return __fmaf_rn((float)j, dq, q); }

}  // namespace raycore
}  // namespace esb
