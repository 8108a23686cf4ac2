// Forward projection (ray marcher, slab slicer, traversal length) and the
// ray-length-normalised back-projection, "faithful" variants.
//
// These kernels evaluate the reference's arithmetic in the reference's order
// with IEEE single precision. This file is compiled with --fmad=false, so no
// multiply-add is fused. The FP32 oracle evaluates the same expressions the
// same way, which makes the two agree to the last bit apart from summation
// order. The projection geometry and the float ray parameter t (advanced by
// t += 0.15 * voxelSize, whose rounding on the float grid of t ~ 1e4 sets the
// reference's effective step) are reproduced exactly. The texture unit is
// replaced by software trilinear/bilinear filtering in FP32 (texel centres at
// +0.5, clamp addressing).
#include <float.h>

#include "esb_device.cuh"

namespace esb {

// tex3D<float>(texObj, x, y, z) with LINEAR filter and CLAMP addressing
// (texture object created at EmSart.cpp:421).
template <int VT>
__device__ __forceinline__ float tex3d_sw(const void* __restrict__ vol, int nx, int ny, int nz, float x, float y,
                                          float z) {
  float xb = x - 0.5f, yb = y - 0.5f, zb = z - 0.5f;
  float fx = floorf(xb), fy = floorf(yb), fz = floorf(zb);
  float a = xb - fx, b = yb - fy, c = zb - fz;
  int x0 = clamp_texel(fx, nx), x1 = clamp_texel(fx + 1.0f, nx);
  int y0 = clamp_texel(fy, ny), y1 = clamp_texel(fy + 1.0f, ny);
  int z0 = clamp_texel(fz, nz), z1 = clamp_texel(fz + 1.0f, nz);
  const long sy = nx, sz = (long)nx * ny;
  const long r00 = z0 * sz + y0 * sy, r10 = z0 * sz + y1 * sy, r01 = z1 * sz + y0 * sy, r11 = z1 * sz + y1 * sy;
  float t000 = Voxel<VT>::load(vol, r00 + x0), t100 = Voxel<VT>::load(vol, r00 + x1);
  float t010 = Voxel<VT>::load(vol, r10 + x0), t110 = Voxel<VT>::load(vol, r10 + x1);
  float t001 = Voxel<VT>::load(vol, r01 + x0), t101 = Voxel<VT>::load(vol, r01 + x1);
  float t011 = Voxel<VT>::load(vol, r11 + x0), t111 = Voxel<VT>::load(vol, r11 + x1);
  float ia = 1.0f - a, ib = 1.0f - b, ic = 1.0f - c;
  return ic * (ib * (ia * t000 + a * t100) + b * (ia * t010 + a * t110)) +
         c * (ib * (ia * t001 + a * t101) + b * (ia * t011 + a * t111));
}

// tex2D(tex, x, y) on a pitched float image, CLAMP addressing; POINT filter
// without CTF, LINEAR with CTF (Reconstructor.cpp:318-327).
__device__ __forceinline__ float tex2d_sw(const float* __restrict__ img, int w, int h, size_t pitchE, float x, float y,
                                          bool linear) {
  if (!linear) {
    int ix = clamp_texel(floorf(x), w), iy = clamp_texel(floorf(y), h);
    return __ldg(img + (size_t)iy * pitchE + ix);
  }
  float xb = x - 0.5f, yb = y - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  float a = xb - fx, b = yb - fy;
  int x0 = clamp_texel(fx, w), x1 = clamp_texel(fx + 1.0f, w);
  int y0 = clamp_texel(fy, h), y1 = clamp_texel(fy + 1.0f, h);
  float t00 = __ldg(img + (size_t)y0 * pitchE + x0), t10 = __ldg(img + (size_t)y0 * pitchE + x1);
  float t01 = __ldg(img + (size_t)y1 * pitchE + x0), t11 = __ldg(img + (size_t)y1 * pitchE + x1);
  return (1.0f - b) * ((1.0f - a) * t00 + a * t10) + b * ((1.0f - a) * t01 + a * t11);
}

// Ray start of detector sub-pixel (px, py) through the mag-anisotropy matrix
// (ForwardProjectionRayMarcher_TL.cu:84-90; DeviceVariables.cuh:42-47).
__device__ __forceinline__ float3 ray_source(const KConst& c, float px, float py) {
  float xA = c.aniso[0] * px + c.aniso[1] * py + c.aniso[2] * 1.0f;
  float yA = c.aniso[3] * px + c.aniso[4] * py + c.aniso[5] * 1.0f;
  float3 s = c.det;
  s.x = s.x + xA * c.u.x;
  s.y = s.y + xA * c.u.y;
  s.z = s.z + xA * c.u.z;
  s.x = s.x + yA * c.v.x;
  s.y = s.y + yA * c.v.y;
  s.z = s.z + yA * c.v.z;
  return s;
}

// Slab test of src + t*dir against [lo, hi] (ForwardProjectionRayMarcher_TL.cu:92-107).
__device__ __forceinline__ void box_hit(float3 s, float3 d, float3 lo, float3 hi, float& tin, float& tout) {
  float ex = (lo.x - s.x) / d.x, ey = (lo.y - s.y) / d.y, ez = (lo.z - s.z) / d.z;
  float xx = (hi.x - s.x) / d.x, xy = (hi.y - s.y) / d.y, xz = (hi.z - s.z) / d.z;
  tin = fmaxf(fmaxf(fminf(ex, xx), fminf(ey, xy)), fminf(ez, xz));
  tout = fminf(fminf(fmaxf(ex, xx), fmaxf(ey, xy)), fmaxf(ez, xz));
}

// Kernel `march` (ForwardProjectionRayMarcher_TL.cu:58-160): one thread per
// detector pixel, 2x2 sub-rays at 0.25/0.75, samples every 0.15 voxel while
// t <= t_out. proj += sum/4, dist = mean chord of the sub-rays that hit.
template <int VT>
__global__ void __launch_bounds__(256) k_march(KConst c, const void* __restrict__ vol, float* __restrict__ proj,
                                               float* __restrict__ dist, size_t pitchE, int x0, int y0, int x1, int y1) {
  const int x = x0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = y0 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= x1 || y >= y1) return;
  const int nx = (int)c.dim.x, ny = (int)c.dim.y, nz = (int)c.dim.z;
  const float h = c.vs.x * 0.15f;
  float temp = 0.0f, gx = 0.0f, gz = 0.0f;
#pragma unroll 1
  for (int o = 0; o < 4; ++o) {
    const float osx = (o & 2) ? 0.75f : 0.25f, osy = (o & 1) ? 0.75f : 0.25f;
    float3 s = ray_source(c, (float)x + osx, (float)y + osy);
    float tin, tout;
    box_hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    if (tout - tin > 0.0f) {
      gx += 1.0f;
      gz += tout - tin;
      float fx = s.x + tin * c.n.x, fy = s.y + tin * c.n.y, fz = s.z + tin * c.n.z;
#pragma unroll 1
      while (tin <= tout) {
        float cx = (fx - c.bbMin.x) * c.bbRcp.x * c.dim.x;
        float cy = (fy - c.bbMin.y) * c.bbRcp.y * c.dim.y;
        float cz = (fz - c.bbMin.z) * c.bbRcp.z * c.dim.z - c.zShift;
        float smp = tex3d_sw<VT>(vol, nx, ny, nz, cx, cy, cz);
        temp += smp * c.vs.x * 0.15f;
        tin += h;
        fx = s.x + tin * c.n.x;
        fy = s.y + tin * c.n.y;
        fz = s.z + tin * c.n.z;
      }
    }
  }
  const size_t i = (size_t)y * pitchE + x;
  proj[i] += temp * 0.25f;
  dist[i] = fmaxf(0.0f, gz / gx);
}

// Kernel `slicer` (ForwardProjectionSlicer.cu:57-220). The reference takes
// the first sample of every ray at the un-advanced ray start (f = c_source,
// :126-141), which lands outside the volume and reads the clamped border.
// That behaviour is kept.
template <int VT>
__global__ void __launch_bounds__(256) k_slicer(KConst c, const void* __restrict__ vol, float* __restrict__ proj,
                                                size_t pitchE, float tminDef, float tmaxDef, int x0, int y0, int x1,
                                                int y1) {
  const int x = x0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = y0 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= x1 || y >= y1) return;
  const int nx = (int)c.dim.x, ny = (int)c.dim.y, nz = (int)c.dim.z;
  const float h = c.vs.x * 0.15f;
  float temp = 0.0f;
#pragma unroll 1
  for (int o = 0; o < 4; ++o) {
    const float osx = (o & 2) ? 0.75f : 0.25f, osy = (o & 1) ? 0.75f : 0.25f;
    float3 s = ray_source(c, (float)x + osx, (float)y + osy);
    float tin, tout;
    box_hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    if (tout - tin > 0.0f) {
      tin = fmaxf(tin, tminDef);
      tout = fminf(tout, tmaxDef);
      float fx = s.x, fy = s.y, fz = s.z;
#pragma unroll 1
      while (tin <= tout) {
        float cx = (fx - c.bbMin.x) * c.bbRcp.x * c.dim.x;
        float cy = (fy - c.bbMin.y) * c.bbRcp.y * c.dim.y;
        float cz = (fz - c.bbMin.z) * c.bbRcp.z * c.dim.z - c.zShift;
        float smp = tex3d_sw<VT>(vol, nx, ny, nz, cx, cy, cz);
        temp += smp * c.vs.x * 0.15f;
        tin += h;
        fx = s.x + tin * c.n.x;
        fy = s.y + tin * c.n.y;
        fz = s.z + tin * c.n.z;
      }
    }
  }
  proj[(size_t)y * pitchE + x] += temp * 0.25f;
}

// Kernel `volTraversalLength` (ForwardProjectionSlicer.cu:224-288).
__global__ void __launch_bounds__(256) k_travlen(KConst c, float* __restrict__ dist, size_t pitchE, int x0, int y0,
                                                 int x1, int y1) {
  const int x = x0 + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = y0 + (int)(blockIdx.y * blockDim.y + threadIdx.y);
  if (x >= x1 || y >= y1) return;
  float3 s = ray_source(c, (float)x + 0.5f, (float)y + 0.5f);
  float tin, tout, val = 0.0f;
  box_hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
  if (tout > tin) val = tout - tin;
  dist[(size_t)y * pitchE + x] += val;
}

// One 4-voxel quad of kernel `backProjection` / `backProjectionFP16`
// (BackProjectionSquareOS.cu:263-782 / 786-1291): bound the quad's 5x1x1
// macro cell on the detector, walk the OS x OS sub-pixel grid inside it,
// intersect each sub-pixel ray with the 4 voxels and accumulate
// sample*chord and chord; then voxel += lambda * sum / chord_sum.
template <int VT>
__global__ void __launch_bounds__(128) k_bp(KConst c, void* __restrict__ vol, const float* __restrict__ img, int pw,
                                            int ph, size_t pitchE, float lambda, int os, float inv, float distMin,
                                            float distMax, int linear) {
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int z = (int)blockIdx.z;
  const int ny = (int)c.dim.y, nz = (int)c.dim.z;
  if (q >= c.dimXQuarter || y >= ny || z >= nz) return;
  const int x = 4 * q;
  const long nx = (long)c.dim.x;
  const long base = ((long)z * ny + y) * nx + x;

  float3 mcMin = make_float3(c.bbMin.x + (float)x * c.vs.x, c.bbMin.y + (float)y * c.vs.y, c.bbMin.z + (float)z * c.vs.z);
  float3 mcMax = make_float3(c.bbMin.x + (float)(x + 5) * c.vs.x, c.bbMin.y + (float)(y + 1) * c.vs.y,
                             c.bbMin.z + (float)(z + 1) * c.vs.z);
  const float ndet = -c.n.x * c.det.x - c.n.y * c.det.y - c.n.z * c.det.z;
  float3 bmin = make_float3(FLT_MAX, FLT_MAX, FLT_MAX);
  float3 bmax = make_float3(-200000.f, -200000.f, -200000.f);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    float px = (k & 4) ? mcMin.x + (mcMax.x - mcMin.x) : mcMin.x;
    float py = (k & 2) ? mcMin.y + (mcMax.y - mcMin.y) : mcMin.y;
    float pz = (k & 1) ? mcMin.z + (mcMax.z - mcMin.z) : mcMin.z;
    float t = (c.n.x * px + c.n.y * py + c.n.z * pz);
    t += ndet;
    t = fabsf(t);
    if (k == 0 && !(t >= distMin && t < distMax)) return;
    float hx = t * (-c.n.x) + px, hy = t * (-c.n.y) + py, hz = t * (-c.n.z) + pz;
    bmin.x = fminf(hx, bmin.x);
    bmin.y = fminf(hy, bmin.y);
    bmin.z = fminf(hz, bmin.z);
    bmax.x = fmaxf(hx, bmax.x);
    bmax.y = fmaxf(hy, bmax.y);
    bmax.z = fmaxf(hz, bmax.z);
  }
  float3 lo = make_float3(fminf(bmin.x, bmax.x), fminf(bmin.y, bmax.y), fminf(bmin.z, bmax.z));
  float3 hi = make_float3(fmaxf(bmin.x, bmax.x), fmaxf(bmin.y, bmax.y), fmaxf(bmin.z, bmax.z));
  if (c.n.x <= 0.0f) {
    float tmp = lo.x;
    lo.x = hi.x;
    hi.x = tmp;
  }
  float plx = c.detMat[0].x * lo.x + c.detMat[0].y * lo.y + c.detMat[0].z * lo.z + 1.0f * c.detMat[0].w;
  float ply = c.detMat[1].x * lo.x + c.detMat[1].y * lo.y + c.detMat[1].z * lo.z + 1.0f * c.detMat[1].w;
  float phx = c.detMat[0].x * hi.x + c.detMat[0].y * hi.y + c.detMat[0].z * hi.z + 1.0f * c.detMat[0].w;
  float phy = c.detMat[1].x * hi.x + c.detMat[1].y * hi.y + c.detMat[1].z * hi.z + 1.0f * c.detMat[1].w;
  int pbx = (int)floorf(fminf(plx, phx));
  int pbz = (int)floorf(fminf(ply, phy));
  int pby = (int)ceilf(fmaxf(plx, phx));
  int pbw = (int)ceilf(fmaxf(ply, phy));
  pbx = (int)fminf(fmaxf((float)pbx, 0.0f), (float)(pw - 1));
  pby = (int)fminf(fmaxf((float)pby, 0.0f), (float)(pw - 1));
  pbz = (int)fminf(fmaxf((float)pbz, 0.0f), (float)(ph - 1));
  pbw = (int)fminf(fmaxf((float)pbw, 0.0f), (float)(ph - 1));

  float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, acc3 = 0.f;
  float d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
  const float by0 = c.bbMin.y + (float)y * c.vs.y, by1 = c.bbMin.y + (float)(y + 1) * c.vs.y;
  const float bz0 = c.bbMin.z + (float)z * c.vs.z, bz1 = c.bbMin.z + (float)(z + 1) * c.vs.z;
  float bx[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) bx[k] = c.bbMin.x + (float)(x + k) * c.vs.x;

#pragma unroll 1
  for (float pyf = (float)pbz + inv * 0.5f; pyf < (float)pbw; pyf += inv) {
#pragma unroll 1
    for (float pxf = (float)pbx + inv * 0.5f; pxf < (float)pby; pxf += inv) {
      float xA = c.anisoInv[0] * pxf + c.anisoInv[1] * pyf + c.anisoInv[2] * 1.0f;
      float yA = c.anisoInv[3] * pxf + c.anisoInv[4] * pyf + c.anisoInv[5] * 1.0f;
      float rx = c.det.x, ry = c.det.y, rz = c.det.z;
      rx = rx + pxf * c.u.x;
      ry = ry + pxf * c.u.y;
      rz = rz + pxf * c.u.z;
      rx = rx + pyf * c.v.x;
      ry = ry + pyf * c.v.y;
      rz = rz + pyf * c.v.z;
      // c_source = ray + 100000.0 * n, evaluated in double (:534-536)
      float sx = (float)((double)rx + 100000.0 * (double)c.n.x);
      float sy = (float)((double)ry + 100000.0 * (double)c.n.y);
      float sz = (float)((double)rz + 100000.0 * (double)c.n.z);
      rx = rx - sx;
      ry = ry - sy;
      rz = rz - sz;
      float il = 1.0f / sqrtf(rx * rx + ry * ry + rz * rz);
      rx = rx * il;
      ry = ry * il;
      rz = rz * il;
      // y and z slabs are shared by the 4 voxels of the quad
      float ey = (by0 - sy) / ry, xy = (by1 - sy) / ry;
      float ez = (bz0 - sz) / rz, xz = (bz1 - sz) / rz;
      float tyz_in = fmaxf(fminf(ey, xy), fminf(ez, xz));
      float tyz_out = fminf(fmaxf(ey, xy), fmaxf(ez, xz));
      float tx[5];
#pragma unroll
      for (int k = 0; k < 5; ++k) tx[k] = (bx[k] - sx) / rx;
      bool sampled = false;
      float smp = 0.0f;
#define ESB_BP_VOXEL(K, ACC, DACC)                                                     \
  {                                                                                    \
    float tin = fmaxf(fminf(tx[K], tx[K + 1]), tyz_in);                                \
    float tout = fminf(fmaxf(tx[K], tx[K + 1]), tyz_out);                              \
    if (tout - tin > 0.0f) {                                                           \
      if (!sampled) {                                                                  \
        smp = tex2d_sw(img, pw, ph, pitchE, xA, yA, linear != 0);                      \
        sampled = true;                                                                \
      }                                                                                \
      ACC += smp * (tout - tin);                                                       \
      DACC += (tout - tin);                                                            \
    }                                                                                  \
  }
      ESB_BP_VOXEL(0, acc0, d0)
      ESB_BP_VOXEL(1, acc1, d1)
      ESB_BP_VOXEL(2, acc2, d2)
      ESB_BP_VOXEL(3, acc3, d3)
#undef ESB_BP_VOXEL
    }
  }
  d0 = fmaxf(0.f, d0);
  d1 = fmaxf(0.f, d1);
  d2 = fmaxf(0.f, d2);
  d3 = fmaxf(0.f, d3);
  float v0 = Voxel<VT>::loadrw(vol, base + 0), v1 = Voxel<VT>::loadrw(vol, base + 1);
  float v2 = Voxel<VT>::loadrw(vol, base + 2), v3 = Voxel<VT>::loadrw(vol, base + 3);
  if (d0 != 0.0f) v0 += (lambda * acc0 / d0);
  if (d1 != 0.0f) v1 += (lambda * acc1 / d1);
  if (d2 != 0.0f) v2 += (lambda * acc2 / d2);
  if (d3 != 0.0f) v3 += (lambda * acc3 / d3);
  Voxel<VT>::store(vol, base + 0, v0);
  Voxel<VT>::store(vol, base + 1, v1);
  Voxel<VT>::store(vol, base + 2, v2);
  Voxel<VT>::store(vol, base + 3, v3);
}

// ----------------------------------------------------------------- launchers
cudaError_t launch_march(const KConst& c, const void* vol, int vt, float* proj, float* dist, size_t pitchE, int x0,
                         int y0, int x1, int y1, cudaStream_t st) {
  if (x1 <= x0 || y1 <= y0) return cudaSuccess;
  dim3 blk(32, 8), grd((x1 - x0 + 31) / 32, (y1 - y0 + 7) / 8);
  switch (vt) {
    case ESB_VOXEL_F32: k_march<ESB_VOXEL_F32><<<grd, blk, 0, st>>>(c, vol, proj, dist, pitchE, x0, y0, x1, y1); ESB_COUNT_LAUNCH(); break;
    case ESB_VOXEL_F16: k_march<ESB_VOXEL_F16><<<grd, blk, 0, st>>>(c, vol, proj, dist, pitchE, x0, y0, x1, y1); ESB_COUNT_LAUNCH(); break;
    default: k_march<ESB_VOXEL_BF16><<<grd, blk, 0, st>>>(c, vol, proj, dist, pitchE, x0, y0, x1, y1); ESB_COUNT_LAUNCH(); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_slicer(const KConst& c, const void* vol, int vt, float* proj, size_t pitchE, float tmin, float tmax,
                          int x0, int y0, int x1, int y1, cudaStream_t st) {
  if (x1 <= x0 || y1 <= y0) return cudaSuccess;
  dim3 blk(32, 8), grd((x1 - x0 + 31) / 32, (y1 - y0 + 7) / 8);
  switch (vt) {
    case ESB_VOXEL_F32: k_slicer<ESB_VOXEL_F32><<<grd, blk, 0, st>>>(c, vol, proj, pitchE, tmin, tmax, x0, y0, x1, y1); ESB_COUNT_LAUNCH(); break;
    case ESB_VOXEL_F16: k_slicer<ESB_VOXEL_F16><<<grd, blk, 0, st>>>(c, vol, proj, pitchE, tmin, tmax, x0, y0, x1, y1); ESB_COUNT_LAUNCH(); break;
    default: k_slicer<ESB_VOXEL_BF16><<<grd, blk, 0, st>>>(c, vol, proj, pitchE, tmin, tmax, x0, y0, x1, y1); ESB_COUNT_LAUNCH(); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_travlen(const KConst& c, float* dist, size_t pitchE, int x0, int y0, int x1, int y1,
                           cudaStream_t st) {
  if (x1 <= x0 || y1 <= y0) return cudaSuccess;
  dim3 blk(32, 8), grd((x1 - x0 + 31) / 32, (y1 - y0 + 7) / 8);
  k_travlen<<<grd, blk, 0, st>>>(c, dist, pitchE, x0, y0, x1, y1); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_bp(const KConst& c, void* vol, int vt, const float* img, int pw, int ph, size_t pitchE, float lambda,
                      int os, float distMin, float distMax, int linear, cudaStream_t st) {
  const int nq = c.dimXQuarter, ny = (int)c.dim.y, nz = (int)c.dim.z;
  if (nq <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  const float inv = 1.0f / (float)os;
  dim3 blk(32, 4, 1), grd((nq + 31) / 32, (ny + 3) / 4, nz);
  switch (vt) {
    case ESB_VOXEL_F32: k_bp<ESB_VOXEL_F32><<<grd, blk, 0, st>>>(c, vol, img, pw, ph, pitchE, lambda, os, inv, distMin, distMax, linear); ESB_COUNT_LAUNCH(); break;
    case ESB_VOXEL_F16: k_bp<ESB_VOXEL_F16><<<grd, blk, 0, st>>>(c, vol, img, pw, ph, pitchE, lambda, os, inv, distMin, distMax, linear); ESB_COUNT_LAUNCH(); break;
    default: k_bp<ESB_VOXEL_BF16><<<grd, blk, 0, st>>>(c, vol, img, pw, ph, pitchE, lambda, os, inv, distMin, distMax, linear); ESB_COUNT_LAUNCH(); break;
  }
  return cudaGetLastError();
}

}  // namespace esb
