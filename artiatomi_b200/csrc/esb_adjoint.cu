// Adjoint of the fast forward projector and gradients of the projection loss.
//
// The fast projector (esb_projector_fast.cu) is linear in the volume: each
// sub-ray's value is a sum over its samples of the trilinear interpolant,
// which it evaluates per lattice cell in closed form from power sums of the
// sample index. Written per corner, a cell's contribution is
// sum_corners value(corner) * W(corner), with W the sum over the cell's
// samples of that corner's trilinear basis function, a polynomial in the
// same power sums. The adjoint walks the same cells with the same sample
// positions and scatters y(pixel) * W(corner) into the volume (atomic adds;
// clamp addressing folds out-of-range corners onto the border voxels exactly
// as the forward read them), so <A x, y> = <x, A^T y> up to float rounding.
//
// Loss and gradients of one tilt, L = 1/2 sum_pixels (A(x, s) - b)^2, where
// s = (s_u, s_v) is a detector offset in pixels applied as a rigid in-plane
// translation of the samples: every sample of every ray moves by
// s_u * u + s_v * v (the detector's pixel axes, through the magnification
// anisotropy matrix). The sample set of each ray stays the unshifted
// reference's, so the model is smooth in s (the float ray origin ~1e4 units
// away would otherwise quantise a sub-pixel shift at ~1e-3 voxel), equals
// the fast projector at s = 0, and dA/ds is the sum over samples of the
// interpolant's gradient along the translation. One launch per tilt: each
// sub-ray is walked once for its value and gradient sums, the 4 sub-rays of
// a pixel are reduced, the residual and the FP64 partial sums (loss, dL/ds,
// Gauss-Newton terms) are formed, and the ray is walked a second time to
// scatter the residual for dL/dx. Nothing is stored per ray: the second walk
// recomputes what it needs.
#include "esb_ray_core.cuh"

namespace esb {

namespace {

using namespace raycore;

// Power sums of one cell's samples: M samples at cell-local coordinates
// (a0, b0, e0) + k * (dqx, dqy, dqz), k = 0..M-1.
struct Sums {
  float M, sa, sb, sc, sab, sac, sbc, sabc;
};

__device__ __forceinline__ Sums power_sums(float a0, float b0, float e0, float M, float dqx, float dqy, float dqz) {
  const float S1 = 0.5f * M * (M - 1.f);
  const float S2 = S1 * (2.f * M - 1.f) * (1.f / 3.f);
  const float S3 = S1 * S1;
  Sums r;
  r.M = M;
  r.sa = M * a0 + S1 * dqx;
  r.sb = M * b0 + S1 * dqy;
  r.sc = M * e0 + S1 * dqz;
  r.sab = M * a0 * b0 + S1 * (a0 * dqy + b0 * dqx) + S2 * dqx * dqy;
  r.sac = M * a0 * e0 + S1 * (a0 * dqz + e0 * dqx) + S2 * dqx * dqz;
  r.sbc = M * b0 * e0 + S1 * (b0 * dqz + e0 * dqy) + S2 * dqy * dqz;
  r.sabc = M * a0 * b0 * e0 + S1 * (a0 * b0 * dqz + a0 * e0 * dqy + b0 * e0 * dqx) +
           S2 * (a0 * dqy * dqz + b0 * dqx * dqz + e0 * dqx * dqy) + S3 * dqx * dqy * dqz;
  return r;
}

// Sums of a single sample at (a, b, c).
__device__ __forceinline__ Sums single(float a, float b, float c) {
  Sums r;
  r.M = 1.f;
  r.sa = a;
  r.sb = b;
  r.sc = c;
  r.sab = a * b;
  r.sac = a * c;
  r.sbc = b * c;
  r.sabc = a * b * c;
  return r;
}

// 3-D cell walk of samples j0..J-1 at q + j*dq: the cell sequence and the
// split of samples between cells are those of the forward projector's
// cell_sum (same expressions).
template <class V>
__device__ void walk3(float qx, float qy, float qz, float dqx, float dqy, float dqz, int j0, int J, V& v) {
  if (j0 >= J) return;
  const float px = qpos(qx, j0, dqx), py = qpos(qy, j0, dqy), pz = qpos(qz, j0, dqz);
  const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  const float inf = FLT_MAX;
  const float isx = dqx != 0.f ? 1.0f / fabsf(dqx) : inf;
  const float isy = dqy != 0.f ? 1.0f / fabsf(dqy) : inf;
  const float isz = dqz != 0.f ? 1.0f / fabsf(dqz) : inf;
  float nxs = dqx > 0.f ? (fx + 1.f - px) * isx : (dqx < 0.f ? (px - fx) * isx : inf);
  float nys = dqy > 0.f ? (fy + 1.f - py) * isy : (dqy < 0.f ? (py - fy) * isy : inf);
  float nzs = dqz > 0.f ? (fz + 1.f - pz) * isz : (dqz < 0.f ? (pz - fz) * isz : inf);
  const int stx = dqx > 0.f ? 1 : -1, sty = dqy > 0.f ? 1 : -1, stz = dqz > 0.f ? 1 : -1;
  const int M_total = J - j0;
  int m0 = 0;
#pragma unroll 1
  for (int guard = 0; guard < 1 << 20; ++guard) {
    const float sexit = fminf(nxs, fminf(nys, nzs));
    int m1 = (sexit >= (float)M_total) ? M_total : (int)ceilf(sexit);
    if (m1 > M_total) m1 = M_total;
    if (m1 > m0) {
      const float a0 = __fsub_rn(qpos(qx, j0 + m0, dqx), (float)ix);
      const float b0 = __fsub_rn(qpos(qy, j0 + m0, dqy), (float)iy);
      const float e0 = __fsub_rn(qpos(qz, j0 + m0, dqz), (float)iz);
      v.cell(ix, iy, iz, power_sums(a0, b0, e0, (float)(m1 - m0), dqx, dqy, dqz));
      m0 = m1;
    }
    if (m0 >= M_total) break;
    if (nxs <= nys && nxs <= nzs) {
      ix += stx;
      nxs = stx > 0 ? ((float)(ix + 1) - px) * isx : (px - (float)ix) * isx;
    } else if (nys <= nzs) {
      iy += sty;
      nys = sty > 0 ? ((float)(iy + 1) - py) * isy : (py - (float)iy) * isy;
    } else {
      iz += stz;
      nzs = stz > 0 ? ((float)(iz + 1) - pz) * isz : (pz - (float)iz) * isz;
    }
  }
}

// 2-D walk in (x, z) of a ray whose y cell and weight b are fixed (the
// forward projector's cell_sum_xz).
template <class V>
__device__ void walk_xz(float qx, float b, int iy, float qz, float dqx, float dqz, int j0, int J, V& v) {
  if (j0 >= J) return;
  const float px = qpos(qx, j0, dqx), pz = qpos(qz, j0, dqz);
  const float fx = floorf(px), fz = floorf(pz);
  int ix = (int)fx, iz = (int)fz;
  const float inf = FLT_MAX;
  const float isx = dqx != 0.f ? 1.0f / fabsf(dqx) : inf;
  const float isz = dqz != 0.f ? 1.0f / fabsf(dqz) : inf;
  float nxs = dqx > 0.f ? (fx + 1.f - px) * isx : (dqx < 0.f ? (px - fx) * isx : inf);
  float nzs = dqz > 0.f ? (fz + 1.f - pz) * isz : (dqz < 0.f ? (pz - fz) * isz : inf);
  const int stx = dqx > 0.f ? 1 : -1, stz = dqz > 0.f ? 1 : -1;
  const int M_total = J - j0;
  int m0 = 0;
#pragma unroll 1
  for (int guard = 0; guard < 1 << 20; ++guard) {
    const float sexit = fminf(nxs, nzs);
    int m1 = (sexit >= (float)M_total) ? M_total : (int)ceilf(sexit);
    if (m1 > M_total) m1 = M_total;
    if (m1 > m0) {
      const float a0 = __fsub_rn(qpos(qx, j0 + m0, dqx), (float)ix);
      const float c0 = __fsub_rn(qpos(qz, j0 + m0, dqz), (float)iz);
      v.cell_xz(ix, iy, b, iz, power_sums(a0, 0.f, c0, (float)(m1 - m0), dqx, 0.f, dqz));
      m0 = m1;
    }
    if (m0 >= M_total) break;
    if (nxs <= nzs) {
      ix += stx;
      nxs = stx > 0 ? ((float)(ix + 1) - px) * isx : (px - (float)ix) * isx;
    } else {
      iz += stz;
      nzs = stz > 0 ? ((float)(iz + 1) - pz) * isz : (pz - (float)iz) * isz;
    }
  }
}

// The samples of one sub-ray from t0 to tout, as the forward projector's
// ray_sum (march mode) takes them.
template <class V>
__device__ void walk_ray(const KConst& c, float3 s, float t0, float tout, float3 d, V& v) {
  const float h = c.vs.x * 0.15f;
  float step;
  bool ok;
  const int J = progression(t0, tout, h, step, ok);
  if (!(t0 <= tout)) return;
  if (!ok) {  // sample by sample along the float recurrence
    float t = t0;
#pragma unroll 1
    for (int guard = 0; guard < 1 << 22 && t <= tout; ++guard) {
      float3 q = interp_coord(c, ray_point(c, s, t));
      q = make_float3(__fadd_rn(q.x, d.x), __fadd_rn(q.y, d.y), __fadd_rn(q.z, d.z));
      const float fx = floorf(q.x), fy = floorf(q.y), fz = floorf(q.z);
      const int ix = (int)fmaxf(fminf(fx, 1.0e9f), -1.0e9f), iy = (int)fmaxf(fminf(fy, 1.0e9f), -1.0e9f),
                iz = (int)fmaxf(fminf(fz, 1.0e9f), -1.0e9f);
      v.cell(ix, iy, iz, single(q.x - fx, q.y - fy, q.z - fz));
      t += h;
    }
    return;
  }
  float3 q0 = interp_coord(c, ray_point(c, s, t0));
  q0 = make_float3(__fadd_rn(q0.x, d.x), __fadd_rn(q0.y, d.y), __fadd_rn(q0.z, d.z));
  const float3 dq = interp_step(c, step);
  const float ylast = qpos(q0.y, J - 1, dq.y);
  if (fabsf(dq.y) * (float)J < 1e-5f && floorf(q0.y) == floorf(ylast)) {
    const float fy = floorf(q0.y);
    walk_xz(q0.x, q0.y - fy, (int)fy, q0.z, dq.x, dq.z, 0, J, v);
    return;
  }
  walk3(q0.x, q0.y, q0.z, dq.x, dq.y, dq.z, 0, J, v);
}

__device__ __forceinline__ int clampi(int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); }

// Value of the interpolant and its gradient (in interpolation coordinates)
// summed over the samples.
template <int VT>
struct FwdGrad {
  const void* __restrict__ vol;
  int nx, ny, nz;
  long sy, sz;
  float sum = 0.f, ga = 0.f, gb = 0.f, gc = 0.f;
  __device__ __forceinline__ float at(int x, int y, int z) const {
    return Voxel<VT>::load(vol, (long)clampi(z, nz) * sz + (long)clampi(y, ny) * sy + clampi(x, nx));
  }
  __device__ void cell(int ix, int iy, int iz, const Sums& s) {
    const float c000 = at(ix, iy, iz), c100 = at(ix + 1, iy, iz), c010 = at(ix, iy + 1, iz),
                c110 = at(ix + 1, iy + 1, iz);
    const float c001 = at(ix, iy, iz + 1), c101 = at(ix + 1, iy, iz + 1), c011 = at(ix, iy + 1, iz + 1),
                c111 = at(ix + 1, iy + 1, iz + 1);
    const float k1 = c100 - c000, k2 = c010 - c000, k3 = c001 - c000;
    const float k4 = c110 - c100 - c010 + c000, k5 = c101 - c100 - c001 + c000, k6 = c011 - c010 - c001 + c000;
    const float k7 = c111 - c110 - c101 - c011 + c100 + c010 + c001 - c000;
    sum += c000 * s.M + k1 * s.sa + k2 * s.sb + k3 * s.sc + k4 * s.sab + k5 * s.sac + k6 * s.sbc + k7 * s.sabc;
    ga += k1 * s.M + k4 * s.sb + k5 * s.sc + k7 * s.sbc;
    gb += k2 * s.M + k4 * s.sa + k6 * s.sc + k7 * s.sac;
    gc += k3 * s.M + k5 * s.sa + k6 * s.sb + k7 * s.sab;
  }
  __device__ void cell_xz(int ix, int iy, float b, int iz, const Sums& s) {
    const float ib = 1.0f - b;
    float e[4], d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int x = ix + (k & 1), z = iz + (k >> 1);
      const float v0 = at(x, iy, z), v1 = at(x, iy + 1, z);
      e[k] = ib * v0 + b * v1;
      d[k] = v1 - v0;
    }
    // e[0] = e00, e[1] = e10, e[2] = e01, e[3] = e11 (x, z)
    const float k1 = e[1] - e[0], k3 = e[2] - e[0], k5 = e[3] - e[1] - e[2] + e[0];
    sum += e[0] * s.M + k1 * s.sa + k3 * s.sc + k5 * s.sac;
    ga += k1 * s.M + k5 * s.sc;
    gc += k3 * s.M + k5 * s.sa;
    gb += d[0] * s.M + (d[1] - d[0]) * s.sa + (d[2] - d[0]) * s.sc + (d[3] - d[1] - d[2] + d[0]) * s.sac;
  }
};

// Scatters w * (sum over samples of each corner's basis function).
struct Scatter {
  float* __restrict__ g;
  int nx, ny, nz;
  long sy, sz;
  float w;
  __device__ __forceinline__ void add(int x, int y, int z, float val) {
    atomicAdd(g + (long)clampi(z, nz) * sz + (long)clampi(y, ny) * sy + clampi(x, nx), w * val);
  }
  __device__ void cell(int ix, int iy, int iz, const Sums& s) {
    add(ix, iy, iz, s.M - s.sa - s.sb - s.sc + s.sab + s.sac + s.sbc - s.sabc);
    add(ix + 1, iy, iz, s.sa - s.sab - s.sac + s.sabc);
    add(ix, iy + 1, iz, s.sb - s.sab - s.sbc + s.sabc);
    add(ix, iy, iz + 1, s.sc - s.sac - s.sbc + s.sabc);
    add(ix + 1, iy + 1, iz, s.sab - s.sabc);
    add(ix + 1, iy, iz + 1, s.sac - s.sabc);
    add(ix, iy + 1, iz + 1, s.sbc - s.sabc);
    add(ix + 1, iy + 1, iz + 1, s.sabc);
  }
  __device__ void cell_xz(int ix, int iy, float b, int iz, const Sums& s) {
    const float ib = 1.0f - b;
    const float W[4] = {s.M - s.sa - s.sc + s.sac, s.sa - s.sac, s.sc - s.sac, s.sac};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int x = ix + (k & 1), z = iz + (k >> 1);
      add(x, iy, z, ib * W[k]);
      add(x, iy + 1, z, b * W[k]);
    }
  }
};

// Thread layout of the fast projector: 4 sub-rays of a pixel in adjacent
// lanes, a warp spans 8 detector rows, 8 warps 8 detector columns.
struct PixelLanes {
  int lane, sub, x, y;
  bool active;
  __device__ PixelLanes(int x0, int y0, int x1, int y1) {
    lane = threadIdx.x & 31;
    sub = lane & 3;
    const int row = (threadIdx.x >> 2) & 7;
    const int warp = threadIdx.x >> 5;
    x = x0 + (int)blockIdx.x * 8 + warp;
    y = y0 + (int)blockIdx.y * 8 + row;
    active = x < x1 && y < y1;
  }
};

__device__ __forceinline__ float3 sub_ray_source(const KConst& c, const PixelLanes& P) {
  const float osx = (P.sub & 2) ? 0.75f : 0.25f, osy = (P.sub & 1) ? 0.75f : 0.25f;
  return ray_src(c, (float)P.x + osx, (float)P.y + osy);
}

// Translation of the interpolation coordinates per pixel of detector offset
// along u (tu) and v (tv): the world displacement of a pixel step
// (ray_src: d origin / d px = aniso[0] u + aniso[3] v, d / d py =
// aniso[1] u + aniso[4] v) in interpolation units.
__device__ __forceinline__ void shift_axes(const KConst& c, float3& tu, float3& tv) {
  const float3 S = make_float3(__fmul_rn(c.bbRcp.x, c.dim.x), __fmul_rn(c.bbRcp.y, c.dim.y),
                               __fmul_rn(c.bbRcp.z, c.dim.z));
  tu = make_float3((c.aniso[0] * c.u.x + c.aniso[3] * c.v.x) * S.x, (c.aniso[0] * c.u.y + c.aniso[3] * c.v.y) * S.y,
                   (c.aniso[0] * c.u.z + c.aniso[3] * c.v.z) * S.z);
  tv = make_float3((c.aniso[1] * c.u.x + c.aniso[4] * c.v.x) * S.x, (c.aniso[1] * c.u.y + c.aniso[4] * c.v.y) * S.y,
                   (c.aniso[1] * c.u.z + c.aniso[4] * c.v.z) * S.z);
}

__device__ __forceinline__ float3 shift_offset(const float3& tu, const float3& tv, float su, float sv) {
  return make_float3(su * tu.x + sv * tv.x, su * tu.y + sv * tv.y, su * tu.z + sv * tv.z);
}

__global__ void __launch_bounds__(256) k_fp_adjoint(KConst c, float* __restrict__ grad, const float* __restrict__ img,
                                                    size_t pitchE, float sx, float sy, int x0, int y0, int x1, int y1) {
  const PixelLanes P(x0, y0, x1, y1);
  if (!P.active) return;
  const float w = img[(size_t)P.y * pitchE + P.x] * (c.vs.x * 0.15f * 0.25f);
  if (w == 0.0f) return;
  const float3 s = sub_ray_source(c, P);
  float tin, tout;
  hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
  if (!(tout - tin > 0.0f)) return;
  float3 tu, tv;
  shift_axes(c, tu, tv);
  Scatter S{grad, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y, w};
  walk_ray(c, s, tin, tout, shift_offset(tu, tv, sx, sy), S);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// out: [0] loss, [1] dL/ds_u, [2] dL/ds_v, [3..5] Gauss-Newton terms
// sum (dp/ds_u)^2, sum dp/ds_u dp/ds_v, sum (dp/ds_v)^2, and with NOUT = 8
// [6] sum p^2, [7] sum p * b (all added to).
template <int VT, int NOUT>
__global__ void __launch_bounds__(256) k_loss_grad(KConst c, const void* __restrict__ vol,
                                                   const float* __restrict__ meas, size_t pitchE, float sx, float sy,
                                                   float* __restrict__ grad, float* __restrict__ proj_out,
                                                   double* __restrict__ out, int x0, int y0, int x1, int y1) {
  const PixelLanes P(x0, y0, x1, y1);
  const float kappa = c.vs.x * 0.15f * 0.25f;
  float3 s = make_float3(0.f, 0.f, 0.f);
  float tin = 0.f, tout = -1.f;
  bool hitray = false;
  float sum = 0.f, gx = 0.f, gy = 0.f;
  float3 tu, tv;
  shift_axes(c, tu, tv);
  const float3 d = shift_offset(tu, tv, sx, sy);
  if (P.active) {
    s = sub_ray_source(c, P);
    hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    hitray = tout - tin > 0.0f;
    if (hitray) {
      FwdGrad<VT> F{vol, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y};
      walk_ray(c, s, tin, tout, d, F);
      sum = F.sum;
      gx = F.ga * tu.x + F.gb * tu.y + F.gc * tu.z;
      gy = F.ga * tv.x + F.gb * tv.y + F.gc * tv.z;
    }
  }
  const float sum4 = quad_sum_ordered(sum), gx4 = quad_sum_ordered(gx), gy4 = quad_sum_ordered(gy);
  double part[NOUT];
#pragma unroll
  for (int q = 0; q < NOUT; ++q) part[q] = 0.0;
  float r = 0.f;
  if (P.active && P.sub == 0) {
    const size_t i = (size_t)P.y * pitchE + P.x;
    const float p = sum4 * kappa;
    if (proj_out) proj_out[i] = p;
    const float b = meas ? meas[i] : 0.f;
    r = p - b;
    const double dr = r, du = (double)gx4 * kappa, dv = (double)gy4 * kappa;
    part[0] = 0.5 * dr * dr;
    part[1] = dr * du;
    part[2] = dr * dv;
    part[3] = du * du;
    part[4] = du * dv;
    part[5] = dv * dv;
    if (NOUT == 8) {
      part[NOUT - 2] = (double)p * p;
      part[NOUT - 1] = (double)p * b;
    }
  }
  // block reduction of the partial sums, then one FP64 atomic each
  __shared__ double red[8][NOUT];
  const int warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NOUT; ++q) {
    const double v = warp_sum(part[q]);
    if (P.lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  if (threadIdx.x < NOUT) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[w][threadIdx.x];
    atomicAdd(out + threadIdx.x, v);
  }
  if (!grad) return;
  r = __shfl_sync(0xffffffffu, r, P.lane & ~3);
  if (!hitray || r == 0.0f) return;
  Scatter Sc{grad, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y, r * kappa};
  walk_ray(c, s, tin, tout, d, Sc);
}

}  // namespace

cudaError_t launch_fp_adjoint(const KConst& c, float* grad, const float* img, size_t pitchE, float sx, float sy, int w,
                              int h, cudaStream_t st) {
  if (w <= 0 || h <= 0) return cudaSuccess;
  dim3 blk(256), grd((w + 7) / 8, (h + 7) / 8);
  k_fp_adjoint<<<grd, blk, 0, st>>>(c, grad, img, pitchE, sx, sy, 0, 0, w, h);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_loss_grad(const KConst& c, const void* vol, int vt, const float* meas, size_t pitchE, float sx,
                             float sy, float* grad, float* proj_out, double* out, int w, int h, cudaStream_t st,
                             const int* roi) {
  if (w <= 0 || h <= 0) return cudaSuccess;
  // pixels [x0, x1) x [y0, y1): the whole detector, or a region of it (then
  // 8 sums, with the amplitude moments)
  const int x0 = roi ? roi[0] : 0, y0 = roi ? roi[1] : 0, x1 = roi ? roi[2] : w, y1 = roi ? roi[3] : h;
  if (x1 <= x0 || y1 <= y0) return cudaSuccess;
  dim3 blk(256), grd((x1 - x0 + 7) / 8, (y1 - y0 + 7) / 8);
#define ESB_LG(VT, N) \
  k_loss_grad<VT, N><<<grd, blk, 0, st>>>(c, vol, meas, pitchE, sx, sy, grad, proj_out, out, x0, y0, x1, y1)
  if (roi) {
    if (vt == ESB_VOXEL_F32) ESB_LG(ESB_VOXEL_F32, 8);
    else if (vt == ESB_VOXEL_F16) ESB_LG(ESB_VOXEL_F16, 8);
    else ESB_LG(ESB_VOXEL_BF16, 8);
  } else {
    if (vt == ESB_VOXEL_F32) ESB_LG(ESB_VOXEL_F32, 6);
    else if (vt == ESB_VOXEL_F16) ESB_LG(ESB_VOXEL_F16, 6);
    else ESB_LG(ESB_VOXEL_BF16, 6);
  }
#undef ESB_LG
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace esb
