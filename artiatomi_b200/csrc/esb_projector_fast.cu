// Forward projection by exact per-cell summation ("fast" projector).
//
// The reference's ray marcher (ForwardProjectionRayMarcher_TL.cu:130-151,
// ForwardProjectionSlicer.cu:130-151) samples the trilinear interpolant at
// t_j = t_in + j*h', j = 0..J-1, and sums the samples. Within one cell of
// the interpolation lattice the interpolant is a trilinear polynomial of the
// cell-local coordinates, and these are linear in j. So the sum over the
// samples inside a cell has a closed form in the power sums of j. Rays of a
// single-axis series stay in one y plane and take the branch-free layer walk
// (layer_sum_xz: one layer of the major axis per step, two cells per layer);
// other rays walk the cells they cross with a 3-D DDA (cell_sum), loading
// each cell's 8 corners once (4 when it enters through a face shared with
// the previous cell). Either replaces ~5 trilinear evaluations (40 loads)
// per cell with 4-8 loads and a few dozen FLOPs.
//
// The sample positions are the reference's: t is the reference's float
// recurrence t += 0.15*voxelSize, whose step on the float grid of t ~ 1e4 is
// a constant h' inside one binade (a power-of-two interval) of t. Rays whose
// samples leave the binade of t_in, or whose step alternates (a rounding
// tie), fall back to sample-by-sample marching. Sample positions are exact
// affine functions of j here, where the reference rounds each position
// computation: the difference is a ~1e-3 voxel jitter of the sample
// positions (rel-L2 ~1e-5 on projections).
//
// One thread per sub-ray. The 4 sub-rays of a pixel sit in adjacent lanes and
// are combined with warp shuffles.
#include <float.h>

#include "esb_ray_core.cuh"

namespace esb {

namespace {

using namespace raycore;

// Sum of the trilinear interpolant over samples j = j0 .. J-1 at coordinates
// q + j*dq, by exact cell-wise closed forms.
template <int VT>
__device__ float cell_sum(const Cell<VT>& C, float qx, float qy, float qz, float dqx, float dqy, float dqz, int j0,
                          int J) {
  if (j0 >= J) return 0.0f;
  // position of sample j0
  float px = qpos(qx, j0, dqx), py = qpos(qy, j0, dqy), pz = qpos(qz, j0, dqz);
  float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
  int ix = (int)fx, iy = (int)fy, iz = (int)fz;
  // sample parameter s (in units of j, relative to j0) of the next boundary per axis
  const float inf = FLT_MAX;
  float isx = dqx != 0.f ? 1.0f / fabsf(dqx) : inf;
  float isy = dqy != 0.f ? 1.0f / fabsf(dqy) : inf;
  float isz = dqz != 0.f ? 1.0f / fabsf(dqz) : inf;
  float nxs = dqx > 0.f ? (fx + 1.f - px) * isx : (dqx < 0.f ? (px - fx) * isx : inf);
  float nys = dqy > 0.f ? (fy + 1.f - py) * isy : (dqy < 0.f ? (py - fy) * isy : inf);
  float nzs = dqz > 0.f ? (fz + 1.f - pz) * isz : (dqz < 0.f ? (pz - fz) * isz : inf);
  const int stx = dqx > 0.f ? 1 : -1, sty = dqy > 0.f ? 1 : -1, stz = dqz > 0.f ? 1 : -1;
  float c000 = C.at(ix, iy, iz), c100 = C.at(ix + 1, iy, iz), c010 = C.at(ix, iy + 1, iz),
        c110 = C.at(ix + 1, iy + 1, iz);
  float c001 = C.at(ix, iy, iz + 1), c101 = C.at(ix + 1, iy, iz + 1), c011 = C.at(ix, iy + 1, iz + 1),
        c111 = C.at(ix + 1, iy + 1, iz + 1);
  const int M_total = J - j0;
  int m0 = 0;  // samples consumed so far (relative to j0)
  float acc = 0.0f;
#pragma unroll 1
  for (int guard = 0; guard < 1 << 20; ++guard) {
    // exit of the current cell in s; samples m0 .. m1-1 lie in it
    float sexit = fminf(nxs, fminf(nys, nzs));
    int m1 = (sexit >= (float)M_total) ? M_total : (int)ceilf(sexit);
    if (m1 > M_total) m1 = M_total;
    if (m1 > m0) {
      // local coordinates of sample m0 and per-sample increments
      const float a0 = __fsub_rn(qpos(qx, j0 + m0, dqx), (float)ix);
      const float b0 = __fsub_rn(qpos(qy, j0 + m0, dqy), (float)iy);
      const float e0 = __fsub_rn(qpos(qz, j0 + m0, dqz), (float)iz);
      const float M = (float)(m1 - m0);
      const float S1 = 0.5f * M * (M - 1.f);
      const float S2 = S1 * (2.f * M - 1.f) * (1.f / 3.f);
      const float S3 = S1 * S1;
      const float k1 = c100 - c000, k2 = c010 - c000, k3 = c001 - c000;
      const float k4 = c110 - c100 - c010 + c000, k5 = c101 - c100 - c001 + c000, k6 = c011 - c010 - c001 + c000;
      const float k7 = c111 - c110 - c101 - c011 + c100 + c010 + c001 - c000;
      const float sa = M * a0 + S1 * dqx, sb = M * b0 + S1 * dqy, sc = M * e0 + S1 * dqz;
      const float sab = M * a0 * b0 + S1 * (a0 * dqy + b0 * dqx) + S2 * dqx * dqy;
      const float sac = M * a0 * e0 + S1 * (a0 * dqz + e0 * dqx) + S2 * dqx * dqz;
      const float sbc = M * b0 * e0 + S1 * (b0 * dqz + e0 * dqy) + S2 * dqy * dqz;
      const float sabc = M * a0 * b0 * e0 + S1 * (a0 * b0 * dqz + a0 * e0 * dqy + b0 * e0 * dqx) +
                         S2 * (a0 * dqy * dqz + b0 * dqx * dqz + e0 * dqx * dqy) + S3 * dqx * dqy * dqz;
      acc += c000 * M + k1 * sa + k2 * sb + k3 * sc + k4 * sab + k5 * sac + k6 * sbc + k7 * sabc;
      m0 = m1;
    }
    if (m0 >= M_total) break;
    // step into the next cell through the nearest face, reusing the 4 shared
    // corners; face crossings are recomputed from the fixed start point, so
    // they carry no accumulated rounding
    if (nxs <= nys && nxs <= nzs) {
      ix += stx;
      nxs = stx > 0 ? ((float)(ix + 1) - px) * isx : (px - (float)ix) * isx;
      if (stx > 0) {
        c000 = c100; c010 = c110; c001 = c101; c011 = c111;
        c100 = C.at(ix + 1, iy, iz); c110 = C.at(ix + 1, iy + 1, iz);
        c101 = C.at(ix + 1, iy, iz + 1); c111 = C.at(ix + 1, iy + 1, iz + 1);
      } else {
        c100 = c000; c110 = c010; c101 = c001; c111 = c011;
        c000 = C.at(ix, iy, iz); c010 = C.at(ix, iy + 1, iz);
        c001 = C.at(ix, iy, iz + 1); c011 = C.at(ix, iy + 1, iz + 1);
      }
    } else if (nys <= nzs) {
      iy += sty;
      nys = sty > 0 ? ((float)(iy + 1) - py) * isy : (py - (float)iy) * isy;
      if (sty > 0) {
        c000 = c010; c100 = c110; c001 = c011; c101 = c111;
        c010 = C.at(ix, iy + 1, iz); c110 = C.at(ix + 1, iy + 1, iz);
        c011 = C.at(ix, iy + 1, iz + 1); c111 = C.at(ix + 1, iy + 1, iz + 1);
      } else {
        c010 = c000; c110 = c100; c011 = c001; c111 = c101;
        c000 = C.at(ix, iy, iz); c100 = C.at(ix + 1, iy, iz);
        c001 = C.at(ix, iy, iz + 1); c101 = C.at(ix + 1, iy, iz + 1);
      }
    } else {
      iz += stz;
      nzs = stz > 0 ? ((float)(iz + 1) - pz) * isz : (pz - (float)iz) * isz;
      if (stz > 0) {
        c000 = c001; c100 = c101; c010 = c011; c110 = c111;
        c001 = C.at(ix, iy, iz + 1); c101 = C.at(ix + 1, iy, iz + 1);
        c011 = C.at(ix, iy + 1, iz + 1); c111 = C.at(ix + 1, iy + 1, iz + 1);
      } else {
        c001 = c000; c101 = c100; c011 = c010; c111 = c110;
        c000 = C.at(ix, iy, iz); c100 = C.at(ix + 1, iy, iz);
        c010 = C.at(ix, iy + 1, iz); c110 = C.at(ix + 1, iy + 1, iz);
      }
    }
  }
  return acc;
}

// cell_sum for a ray whose y coordinate stays in one interpolation cell with
// a constant weight b (single-axis tilt about y: n.y is 0 or ~1e-10): the
// trilinear interpolant is a bilinear one in (x, z) of the y-interpolated
// corners.
//
// The walk goes layer by layer along the major axis (z or x, the one with the
// larger per-sample step). A layer holds at most one crossing of the minor
// axis, so every step sums two cells, the second empty when the ray does not
// cross in that layer, and the loop has no data-dependent branches: lanes
// whose rays cross in different layers stay converged. Both axes are
// mirrored so that the walk advances in the + direction of each.
//
// A cell's M samples have local coordinates (a0 + m da, c0 + m dc); with
// their mean (a, c) and the bilinear f = e00 + k1 a + k3 c + k5 a c,
//   sum_m f = M [f(a, c) + k5 da dc (M^2 - 1) / 12].
// Samples are assigned to cells exactly as by the cell-by-cell DDA (the
// sample parameter of each face crossing, rounded up).
template <int VT, bool ZMAJ, class Off>
__device__ float layer_sum_xz(const Cell<VT>& C, float qx, float b, int iy, float qz, float dqx, float dqz, int j0,
                              int J) {
  if (j0 >= J) return 0.0f;
  // major axis m (layers), minor axis n
  const float qm = ZMAJ ? qz : qx, dqm = ZMAJ ? dqz : dqx;
  const float qn = ZMAJ ? qx : qz, dqn = ZMAJ ? dqx : dqz;
  const int sm = dqm < 0.f ? -1 : 1, sn = dqn < 0.f ? -1 : 1;
  const float Mq = sm > 0 ? qm : -qm, dM = fabsf(dqm);
  const float Nq = sn > 0 ? qn : -qn, dN = fabsf(dqn);
  const float fj0 = (float)j0;
  const float pM = __fmaf_rn(fj0, dM, Mq), pN = __fmaf_rn(fj0, dN, Nq);
  float fcm = floorf(pM), fcn = floorf(pN);
  const float inf = FLT_MAX;
  const float isM = 1.0f / dM;  // dM > 0: the ray moves in x-z, and the major step is the larger one
  const float isN = dN > 0.f ? 1.0f / dN : inf;
  float nMs = ((fcm + 1.f) - pM) * isM;
  float nNs = dN > 0.f ? ((fcn + 1.f) - pN) * isN : inf;
  const float g = dN * dM * (1.0f / 12.0f);
  const float jb = fj0 - 0.5f;
  // element offsets of type Off: 32-bit below 2^32 voxels (cheaper address
  // arithmetic), 64-bit above (the launchers choose)
  const Off SM = ZMAJ ? (Off)C.sz : (Off)1, SN = ZMAJ ? (Off)1 : (Off)C.sz;
  const int nMax = ZMAJ ? C.nz - 1 : C.nx - 1, nNax = ZMAJ ? C.nx - 1 : C.nz - 1;
  auto clampM = [&](int i) { return (Off)(i < 0 ? 0 : (i > nMax ? nMax : i)) * SM; };
  auto clampN = [&](int i) { return (Off)(i < 0 ? 0 : (i > nNax ? nNax : i)) * SN; };
  const Off y0 = (Off)(iy < 0 ? 0 : (iy > C.ny - 1 ? C.ny - 1 : iy)) * (Off)C.sy;
  const Off y1 = (Off)(iy + 1 < 0 ? 0 : (iy + 1 > C.ny - 1 ? C.ny - 1 : iy + 1)) * (Off)C.sy;
  const float ib = 1.0f - b;
  auto ey = [&](Off o) {
    return ib * Voxel<VT>::load(C.vol, (long)(o + y0)) + b * Voxel<VT>::load(C.vol, (long)(o + y1));
  };
  // original indices of the current cell's near and far corners per axis
  int inF = sn * (int)fcn + sn;
  int imF = sm * (int)fcm + sm;
  Off on = clampN(inF - sn), of = clampN(inF);
  Off omn = clampM(imF - sm), omf = clampM(imF);
  float enn = ey(on + omn), efn = ey(of + omn);
  const float Mt = (float)(J - j0);
  float fm0 = 0.0f, acc = 0.0f;
  // two layers per iteration give the scheduler independent loads; the
  // 64-bit-offset instances stay at one (registers)
  constexpr int kUnroll = sizeof(Off) == 4 ? 2 : 1;
#pragma unroll kUnroll
  for (int guard = 0; guard < 1 << 20; ++guard) {
    // samples [fm0, fmA) lie in cell (n, m), [fmA, fmL) in cell (n + 1, m)
    const float fmL = nMs >= Mt ? Mt : ceilf(nMs);
    const bool X = nNs <= nMs;
    const float sA = fminf(nNs, nMs);
    const float fmA = fmaxf(sA >= Mt ? Mt : ceilf(sA), fm0);
    const int inF2 = inF + sn;
    const Off o2 = clampN(inF2);
    const float enf = ey(on + omf), eff = ey(of + omf);
    const float e2n = ey(o2 + omn), e2f = ey(o2 + omf);
    {
      const float M = fmA - fm0;
      const float jm = __fmaf_rn(0.5f, fm0 + fmA, jb);
      const float a = __fmaf_rn(jm, dN, Nq) - fcn, c = __fmaf_rn(jm, dM, Mq) - fcm;
      const float k1 = efn - enn, k3 = enf - enn, k5 = (eff - enf) - k1;
      const float f = fmaf(c, fmaf(a, k5, k3), fmaf(a, k1, enn));
      acc = fmaf(M, fmaf(k5, fmaf(M * M, g, -g), f), acc);
    }
    {
      const float M = fmL - fmA;
      const float jm = __fmaf_rn(0.5f, fmA + fmL, jb);
      const float a = __fmaf_rn(jm, dN, Nq) - (fcn + 1.f), c = __fmaf_rn(jm, dM, Mq) - fcm;
      const float k1 = e2n - efn, k3 = eff - efn, k5 = (e2f - eff) - k1;
      const float f = fmaf(c, fmaf(a, k5, k3), fmaf(a, k1, efn));
      acc = fmaf(M, fmaf(k5, fmaf(M * M, g, -g), f), acc);
    }
    fm0 = fmL;
    if (fm0 >= Mt) break;
    // next layer, one minor cell further when this layer crossed
    enn = X ? eff : enf;
    efn = X ? e2f : eff;
    if (X) {
      fcn += 1.f;
      inF = inF2;
      on = of;
      of = o2;
      nNs = ((fcn + 1.f) - pN) * isN;
    }
    fcm += 1.f;
    imF += sm;
    omn = omf;
    omf = clampM(imF);
    nMs = ((fcm + 1.f) - pM) * isM;
  }
  return acc;
}

template <int VT, class Off>
__device__ float cell_sum_xz(const Cell<VT>& C, float qx, float b, int iy, float qz, float dqx, float dqz, int j0,
                             int J) {
  if (fabsf(dqz) >= fabsf(dqx)) return layer_sum_xz<VT, true, Off>(C, qx, b, iy, qz, dqx, dqz, j0, J);
  return layer_sum_xz<VT, false, Off>(C, qx, b, iy, qz, dqx, dqz, j0, J);
}

// Sum over the samples of one sub-ray from t0 to tout (first_at_source: the
// slicer's first sample is taken at the ray start, ForwardProjectionSlicer.cu:126-141).
template <int VT, class Off>
__device__ float ray_sum(const KConst& c, const Cell<VT>& C, float3 s, float t0, float tout, bool first_at_source) {
  const float h = c.vs.x * 0.15f;
  float step;
  bool ok;
  int J = progression(t0, tout, h, step, ok);
  if (!(t0 <= tout)) return 0.0f;
  if (!ok) {  // sample-by-sample marching with the reference's float recurrence
    float sum = 0.0f, t = t0;
    bool first = true;
#pragma unroll 1
    while (t <= tout) {
      float3 p = first && first_at_source ? s : ray_point(c, s, t);
      float3 q = interp_coord(c, p);
      sum += trilinear<VT>(C, q.x, q.y, q.z);
      first = false;
      t += h;
    }
    return sum;
  }
  // q(j) = q(t0) + j * dq
  float3 q0 = interp_coord(c, ray_point(c, s, t0));
  const float3 dq = interp_step(c, step);
  const float dqx = dq.x, dqy = dq.y, dqz = dq.z;
  float sum = 0.0f;
  int j0 = 0;
  if (first_at_source) {
    float3 q = interp_coord(c, s);
    sum += trilinear<VT>(C, q.x, q.y, q.z);
    j0 = 1;
  }
  // y stays in one cell and moves by < 1e-5 voxel over the ray: bilinear x-z walk
  const float ylast = qpos(q0.y, J - 1, dqy);
  if (fabsf(dqy) * (float)J < 1e-5f && floorf(q0.y) == floorf(ylast)) {
    const float fy = floorf(q0.y);
    return sum + cell_sum_xz<VT, Off>(C, q0.x, q0.y - fy, (int)fy, q0.z, dqx, dqz, j0, J);
  }
  return sum + cell_sum<VT>(C, q0.x, q0.y, q0.z, dqx, dqy, dqz, j0, J);
}

// mode 0: march (proj += sum/4, dist = mean chord); mode 1: slicer (proj += sum/4 within [tmin, tmax])
// NW warps per block: NW detector columns x 8 rows; blocks of 128 threads
// fit 6 per SM at the walker's register count (256-thread blocks fit 3); the
// launch shape is picked per problem by the reconstructor's autotuner.
template <int VT, int MODE, class Off, int NW>
__global__ void __launch_bounds__(32 * NW, 24 / NW) k_project_fast(KConst c, const void* __restrict__ vol, float* __restrict__ proj,
                                                      float* __restrict__ dist, size_t pitchE, float tminDef,
                                                      float tmaxDef, int x0, int y0, int x1, int y1) {
  // lanes: 4 sub-rays of a pixel adjacent; a warp spans 8 detector rows (v);
  // the NW warps of a block, NW detector columns (u)
  const int lane = threadIdx.x & 31;
  const int sub = lane & 3;
  const int row = (threadIdx.x >> 2) & 7;
  const int warp = threadIdx.x >> 5;
  const int x = x0 + (int)blockIdx.x * NW + warp;
  const int y = y0 + (int)blockIdx.y * 8 + row;
  const bool active = x < x1 && y < y1;
  Cell<VT> C{vol, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y};
  float sum = 0.0f, gx = 0.0f, gz = 0.0f;
  if (active) {
    const float osx = (sub & 2) ? 0.75f : 0.25f, osy = (sub & 1) ? 0.75f : 0.25f;
    float3 s = ray_src(c, (float)x + osx, (float)y + osy);
    float tin, tout;
    hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    if (tout - tin > 0.0f) {
      gx = 1.0f;
      gz = tout - tin;
      if (MODE == 1) {
        tin = fmaxf(tin, tminDef);
        tout = fminf(tout, tmaxDef);
      }
      sum = ray_sum<VT, Off>(c, C, s, tin, tout, MODE == 1);
    }
  }
  sum = quad_sum_ordered(sum);
  if (MODE == 0) {
    gx = quad_sum_ordered(gx);
    gz = quad_sum_ordered(gz);
  }
  if (active && sub == 0) {
    const size_t i = (size_t)y * pitchE + x;
    proj[i] += sum * c.vs.x * 0.15f * 0.25f;
    if (MODE == 0) dist[i] = fmaxf(0.0f, gz / gx);
  }
}

// All defocus slabs of one projection in one launch: slab k's image gets
// the slicer's integral over [bound[k], bound[k+1]] (ForwardProjectionSlicer.cu:57-220,
// called once per slab by Reconstructor.cpp:515-585). The 4 lanes of a pixel
// walk the union of their slab ranges together so each slab's sum keeps the
// reference's sub-ray order.
template <int VT, class Off, int NW>
__global__ void __launch_bounds__(32 * NW, 24 / NW) k_slicer_fused(KConst c, const void* __restrict__ vol, float* __restrict__ imgs,
                                                      size_t img_stride, size_t pitchE, SlabTable slabs, int x0, int y0,
                                                      int x1, int y1) {
  const int lane = threadIdx.x & 31;
  const int sub = lane & 3;
  const int row = (threadIdx.x >> 2) & 7;
  const int warp = threadIdx.x >> 5;
  const int x = x0 + (int)blockIdx.x * NW + warp;
  const int y = y0 + (int)blockIdx.y * 8 + row;
  const bool active = x < x1 && y < y1;
  Cell<VT> C{vol, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y};
  float3 s = make_float3(0.f, 0.f, 0.f);
  float tin = 0.f, tout = -1.f;
  int klo = ESB_MAX_SLABS, khi = -1;
  bool hitray = false;
  if (active) {
    const float osx = (sub & 2) ? 0.75f : 0.25f, osy = (sub & 1) ? 0.75f : 0.25f;
    s = ray_src(c, (float)x + osx, (float)y + osy);
    hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    hitray = tout - tin > 0.0f;
    if (hitray) {
      for (int k = 0; k < slabs.count; ++k) {
        // slab k has samples when max(tin, b_k) <= min(tout, b_{k+1})
        if (fmaxf(tin, slabs.bound[k]) <= fminf(tout, slabs.bound[k + 1])) {
          klo = min(klo, k);
          khi = max(khi, k);
        }
      }
    }
  }
  for (int o = 1; o <= 2; o <<= 1) {
    klo = min(klo, __shfl_xor_sync(0xffffffffu, klo, o));
    khi = max(khi, __shfl_xor_sync(0xffffffffu, khi, o));
  }
  // the warp walks the union of its pixels' slab ranges (shuffles need all lanes)
  int wlo = klo, whi = khi;
  for (int o = 4; o <= 16; o <<= 1) {
    wlo = min(wlo, __shfl_xor_sync(0xffffffffu, wlo, o));
    whi = max(whi, __shfl_xor_sync(0xffffffffu, whi, o));
  }
  const size_t pix = (size_t)y * pitchE + x;
  for (int k = wlo; k <= whi; ++k) {
    float v = 0.0f;
    if (hitray && k >= klo && k <= khi) {
      const float t0 = fmaxf(tin, slabs.bound[k]);
      const float t1 = fminf(tout, slabs.bound[k + 1]);
      v = ray_sum<VT, Off>(c, C, s, t0, t1, true);
    }
    v = quad_sum_ordered(v);
    if (active && sub == 0 && k >= klo && k <= khi) imgs[(size_t)k * img_stride + pix] = v * c.vs.x * 0.15f * 0.25f;
  }
}

// ---------------------------------------------------------------------------
// Single-axis series: k_project_axis, k_slicer_axis.
//
// Every ray of a single-axis projection moves in the x-z plane with the same
// direction, so the major axis of the layer walk and the signs of both steps
// are the same for all rays of a launch: they become template parameters
// (ZMAJ, SM, SN), and the host picks the instance from the beam direction.
// The walk is layer_sum_xz's (same sample bookkeeping, cell sums and order)
// with cheaper loads: it keeps the near row of the current layer (3 corner
// values, interpolated in y) and loads the far row at 4 minor positions, so
// that after a minor crossing the next layer's near row is the far row moved
// by one. While the 4 positions and the far row lie inside the volume, the
// far-row corners are read through one running pointer per y plane at fixed
// offsets (compile-time offsets for the z-major walk), without clamping or
// index arithmetic; at the volume's faces the walk takes clamped reads.

template <int VT>
__device__ __forceinline__ float ldv(const char* p) {
  if (VT == ESB_VOXEL_F32) return __ldg((const float*)p);
  if (VT == ESB_VOXEL_F16) return __half2float(__ldg((const __half*)p));
  return __bfloat162float(__ldg((const __nv_bfloat16*)p));
}

// A voxel as loaded (float, or the 16 bits of a half / bfloat16), converted
// to float where it is used: the walk's prefetched far row stays in its
// loaded form until the next layer blends it.
template <int VT>
struct RawVoxel {
  typedef unsigned short T;
};
template <>
struct RawVoxel<ESB_VOXEL_F32> {
  typedef float T;
};
template <int VT>
__device__ __forceinline__ typename RawVoxel<VT>::T ldraw(const char* p) {
  if constexpr (VT == ESB_VOXEL_F32) return __ldg((const float*)p);
  else return __ldg((const unsigned short*)p);
}
template <int VT>
__device__ __forceinline__ float cvt(typename RawVoxel<VT>::T r) {
  if constexpr (VT == ESB_VOXEL_F32) return r;
  else if constexpr (VT == ESB_VOXEL_F16) return __half2float(__ushort_as_half(r));
  else return __uint_as_float((unsigned)r << 16);
}

// Sum of the trilinear interpolant over samples j0 .. J-1 of one ray whose y
// interpolation coordinate lies in cell iy with weight b, walked along major
// axis z (ZMAJ) or x with step signs SM (major) and SN (minor). Mq, Nq,
// dM, dN: mirrored major / minor coordinate of sample 0 and |steps|
// (dM >= dN).
template <int VT, bool ZMAJ, int SM, int SN>
__device__ float axis_walk(const Cell<VT>& C, float Mq, float Nq, float dM, float dN, float b, int iy, int j0,
                           int J) {
  constexpr long ES = VT == ESB_VOXEL_F32 ? 4 : 2;
  const long sM = ZMAJ ? C.sz : 1, sN = ZMAJ ? 1 : C.sz;  // element strides of the major and minor axes
  const int nM = ZMAJ ? C.nz : C.nx, nN = ZMAJ ? C.nx : C.nz;
  const char* const base = (const char*)C.vol;
  const float fj0 = (float)j0;
  const float pM = __fmaf_rn(fj0, dM, Mq), pN = __fmaf_rn(fj0, dN, Nq);
  float fcm = floorf(pM), fcn = floorf(pN);
  const float inf = FLT_MAX;
  const float isM = 1.0f / dM;
  const float isN = dN > 0.f ? 1.0f / dN : inf;
  float nMs = ((fcm + 1.f) - pM) * isM;
  float nNs = dN > 0.f ? ((fcn + 1.f) - pN) * isN : inf;
  const float g = dN * dM * (1.0f / 12.0f);
  const float jb = fj0 - 0.5f;
  const float Mt = (float)(J - j0);
  const float ib = 1.0f - b;
  const int ny = C.ny;
  const long y0 = (long)(iy < 0 ? 0 : (iy > ny - 1 ? ny - 1 : iy)) * C.sy;
  const long y1 = (long)(iy + 1 < 0 ? 0 : (iy + 1 > ny - 1 ? ny - 1 : iy + 1)) * C.sy;
  // original indices: far major row of the current layer, first minor position of the window
  int im = SM * ((int)fcm + 1), in0 = SN * (int)fcn;
  const char* P = base + ES * (y0 + (long)im * sM + (long)in0 * sN);  // far row, plane iy
  const long dy = ES * (y1 - y0);
  const long strideN = SN * ES * sN, strideM = SM * ES * sM;
  auto ld = [&](int mi, int ni) -> float {  // clamped, interpolated in y
    mi = mi < 0 ? 0 : (mi > nM - 1 ? nM - 1 : mi);
    ni = ni < 0 ? 0 : (ni > nN - 1 ? nN - 1 : ni);
    const char* p = base + ES * ((long)mi * sM + (long)ni * sN + y0);
    return fmaf(b, ldv<VT>(p + dy), ib * ldv<VT>(p));
  };
  // raw far-row values (plane iy, plane iy + 1 at minor positions 0..3)
  // of the layer whose far row is at major index mi and window start ni
  const bool canN = nN >= 4;
  typename RawVoxel<VT>::T r0, r1, r2, r3, r4, r5, r6, r7;
  auto fetch = [&](int mi, int ni, const char* q) {
    const int lo = SN > 0 ? ni : ni - 3;
    if (canN && (unsigned)lo <= (unsigned)(nN - 4) && (unsigned)mi < (unsigned)nM) {
      r0 = ldraw<VT>(q);
      r1 = ldraw<VT>(q + dy);
      r2 = ldraw<VT>(q + strideN);
      r3 = ldraw<VT>(q + strideN + dy);
      r4 = ldraw<VT>(q + 2 * strideN);
      r5 = ldraw<VT>(q + 2 * strideN + dy);
      r6 = ldraw<VT>(q + 3 * strideN);
      r7 = ldraw<VT>(q + 3 * strideN + dy);
    } else {
      mi = mi < 0 ? 0 : (mi > nM - 1 ? nM - 1 : mi);
      const char* row = base + ES * ((long)mi * sM + y0);
      auto at = [&](int n) {
        n = n < 0 ? 0 : (n > nN - 1 ? nN - 1 : n);
        return row + ES * ((long)n * sN);
      };
      const char* q0 = at(ni);
      const char* q1 = at(ni + SN);
      const char* q2 = at(ni + 2 * SN);
      const char* q3 = at(ni + 3 * SN);
      r0 = ldraw<VT>(q0);
      r1 = ldraw<VT>(q0 + dy);
      r2 = ldraw<VT>(q1);
      r3 = ldraw<VT>(q1 + dy);
      r4 = ldraw<VT>(q2);
      r5 = ldraw<VT>(q2 + dy);
      r6 = ldraw<VT>(q3);
      r7 = ldraw<VT>(q3 + dy);
    }
  };
  // near row of the first layer, and its far row
  float N0 = ld(im - SM, in0), N1 = ld(im - SM, in0 + SN), N2 = ld(im - SM, in0 + 2 * SN);
  fetch(im, in0, P);
  float F0 = fmaf(b, cvt<VT>(r1), ib * cvt<VT>(r0)), F1 = fmaf(b, cvt<VT>(r3), ib * cvt<VT>(r2)), F2 = fmaf(b, cvt<VT>(r5), ib * cvt<VT>(r4)), F3 = fmaf(b, cvt<VT>(r7), ib * cvt<VT>(r6));
  float fm0 = 0.0f, acc = 0.0f;
#pragma unroll 1
  for (int guard = 0; guard < 1 << 20; ++guard) {
    // samples [fm0, fmA) lie in cell (n, m), [fmA, fmL) in cell (n + 1, m)
    const float fmL = fminf(ceilf(nMs), Mt);
    const bool X = nNs <= nMs;
    const float fmA = fmaxf(fminf(ceilf(fminf(nNs, nMs)), Mt), fm0);
    // the next layer's far row, one minor position further when this layer
    // crosses: its loads are in flight during this layer's sums
    const char* Pn = P + strideM + (X ? strideN : 0);
    const int imn = im + SM, in0n = in0 + (X ? SN : 0);
    fetch(imn, in0n, Pn);
    {  // cell (n, m): near corners N0, N1, far corners F0, F1
      const float M = fmA - fm0;
      const float jm = __fmaf_rn(0.5f, fm0 + fmA, jb);
      const float a = __fmaf_rn(jm, dN, Nq) - fcn, c = __fmaf_rn(jm, dM, Mq) - fcm;
      const float k1 = N1 - N0, k3 = F0 - N0, k5 = (F1 - F0) - k1;
      const float f = fmaf(c, fmaf(a, k5, k3), fmaf(a, k1, N0));
      acc = fmaf(M, fmaf(k5, fmaf(M * M, g, -g), f), acc);
    }
    {  // cell (n + 1, m): near corners N1, N2, far corners F1, F2
      const float M = fmL - fmA;
      const float jm = __fmaf_rn(0.5f, fmA + fmL, jb);
      const float a = __fmaf_rn(jm, dN, Nq) - (fcn + 1.f), c = __fmaf_rn(jm, dM, Mq) - fcm;
      const float k1 = N2 - N1, k3 = F1 - N1, k5 = (F2 - F1) - k1;
      const float f = fmaf(c, fmaf(a, k5, k3), fmaf(a, k1, N1));
      acc = fmaf(M, fmaf(k5, fmaf(M * M, g, -g), f), acc);
    }
    fm0 = fmL;
    if (fm0 >= Mt) break;
    // next layer
    N0 = X ? F1 : F0;
    N1 = X ? F2 : F1;
    N2 = X ? F3 : F2;
    F0 = fmaf(b, cvt<VT>(r1), ib * cvt<VT>(r0));
    F1 = fmaf(b, cvt<VT>(r3), ib * cvt<VT>(r2));
    F2 = fmaf(b, cvt<VT>(r5), ib * cvt<VT>(r4));
    F3 = fmaf(b, cvt<VT>(r7), ib * cvt<VT>(r6));
    if (X) {
      fcn += 1.f;
      nNs = ((fcn + 1.f) - pN) * isN;
    }
    fcm += 1.f;
    nMs = ((fcm + 1.f) - pM) * isM;
    im = imn;
    in0 = in0n;
    P = Pn;
  }
  return acc;
}

// Sum over the samples of one sub-ray from t0 to tout (ray_sum) with the
// axis walk when the ray fits the launch's instance (its y in one cell, its
// major axis and step signs the instance's), else ray_sum's walkers.
template <int VT, bool ZMAJ, int SM, int SN>
__device__ float axis_ray_sum(const KConst& c, const Cell<VT>& C, float3 s, float t0, float tout,
                              bool first_at_source) {
  if (!(t0 <= tout)) return 0.0f;
  const float h = c.vs.x * 0.15f;
  float step;
  bool ok;
  const int J = progression(t0, tout, h, step, ok);
  if (!ok) return ray_sum<VT, unsigned long long>(c, C, s, t0, tout, first_at_source);
  const float3 q0 = interp_coord(c, ray_point(c, s, t0));
  const float3 dq = interp_step(c, step);
  float sum = 0.0f;
  int j0 = 0;
  if (first_at_source) {
    const float3 q = interp_coord(c, s);
    sum = trilinear<VT>(C, q.x, q.y, q.z);
    j0 = 1;
  }
  const float ylast = qpos(q0.y, J - 1, dq.y);
  if (!(fabsf(dq.y) * (float)J < 1e-5f && floorf(q0.y) == floorf(ylast)))
    return sum + cell_sum<VT>(C, q0.x, q0.y, q0.z, dq.x, dq.y, dq.z, j0, J);
  const float fy = floorf(q0.y);
  const float qm = ZMAJ ? q0.z : q0.x, dqm = ZMAJ ? dq.z : dq.x;
  const float qn = ZMAJ ? q0.x : q0.z, dqn = ZMAJ ? dq.x : dq.z;
  if ((fabsf(dq.z) >= fabsf(dq.x)) != ZMAJ || (dqm < 0.f ? -1 : 1) != SM || (dqn < 0.f ? -1 : 1) != SN)
    return sum + cell_sum_xz<VT, unsigned long long>(C, q0.x, q0.y - fy, (int)fy, q0.z, dq.x, dq.z, j0, J);
  if (j0 >= J) return sum;
  return sum + axis_walk<VT, ZMAJ, SM, SN>(C, SM > 0 ? qm : -qm, SN > 0 ? qn : -qn, fabsf(dqm), fabsf(dqn),
                                           q0.y - fy, (int)fy, j0, J);
}

// k_project_fast (march) for single-axis series; layout of k_project_fast.
template <int VT, bool ZMAJ, int SM, int SN>
__global__ void __launch_bounds__(256) k_project_axis(KConst c, const void* __restrict__ vol, float* __restrict__ proj,
                                                      float* __restrict__ dist, size_t pitchE, int x0, int y0, int x1,
                                                      int y1) {
  const int lane = threadIdx.x & 31;
  const int sub = lane & 3;
  const int row = lane >> 2;
  const int nw = blockDim.x >> 5;
  const int x = x0 + (int)blockIdx.x * nw + (int)(threadIdx.x >> 5);
  const int y = y0 + (int)blockIdx.y * 8 + row;
  const bool active = x < x1 && y < y1;
  Cell<VT> C{vol, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y};
  float sum = 0.0f, gx = 0.0f, gz = 0.0f;
  if (active) {
    const float osx = (sub & 2) ? 0.75f : 0.25f, osy = (sub & 1) ? 0.75f : 0.25f;
    const float3 s = ray_src(c, (float)x + osx, (float)y + osy);
    float tin, tout;
    hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    if (tout - tin > 0.0f) {
      gx = 1.0f;
      gz = tout - tin;
      sum = axis_ray_sum<VT, ZMAJ, SM, SN>(c, C, s, tin, tout, false);
    }
  }
  sum = quad_sum_ordered(sum);
  gx = quad_sum_ordered(gx);
  gz = quad_sum_ordered(gz);
  if (active && sub == 0) {
    const size_t i = (size_t)y * pitchE + x;
    proj[i] += sum * c.vs.x * 0.15f * 0.25f;
    dist[i] = fmaxf(0.0f, gz / gx);
  }
}

// k_slicer_fused for single-axis series; layout of k_slicer_fused.
// (16-bit volumes: at most 80 registers, 3 blocks of 256 threads per SM;
// uncapped, those instances take about 100 and fit 2. FP32 instances take
// 76-79 uncapped, and a cap changes their allocation for the worse.)
template <int VT, bool ZMAJ, int SM, int SN>
__global__ void __launch_bounds__(256, VT == ESB_VOXEL_F32 ? 0 : 3) k_slicer_axis(KConst c, const void* __restrict__ vol, float* __restrict__ imgs,
                                                     size_t img_stride, size_t pitchE, SlabTable slabs, int x0, int y0,
                                                     int x1, int y1) {
  const int lane = threadIdx.x & 31;
  const int sub = lane & 3;
  const int row = lane >> 2;
  const int nw = blockDim.x >> 5;
  const int x = x0 + (int)blockIdx.x * nw + (int)(threadIdx.x >> 5);
  const int y = y0 + (int)blockIdx.y * 8 + row;
  const bool active = x < x1 && y < y1;
  Cell<VT> C{vol, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z, (long)c.dim.x, (long)c.dim.x * (long)c.dim.y};
  float3 s = make_float3(0.f, 0.f, 0.f);
  float tin = 0.f, tout = -1.f;
  int klo = ESB_MAX_SLABS, khi = -1;
  bool hitray = false;
  if (active) {
    const float osx = (sub & 2) ? 0.75f : 0.25f, osy = (sub & 1) ? 0.75f : 0.25f;
    s = ray_src(c, (float)x + osx, (float)y + osy);
    hit(s, c.n, c.bbMin, c.bbMax, tin, tout);
    hitray = tout - tin > 0.0f;
    if (hitray) {
      for (int k = 0; k < slabs.count; ++k) {
        // slab k has samples when max(tin, b_k) <= min(tout, b_{k+1})
        if (fmaxf(tin, slabs.bound[k]) <= fminf(tout, slabs.bound[k + 1])) {
          klo = min(klo, k);
          khi = max(khi, k);
        }
      }
    }
  }
  for (int o = 1; o <= 2; o <<= 1) {
    klo = min(klo, __shfl_xor_sync(0xffffffffu, klo, o));
    khi = max(khi, __shfl_xor_sync(0xffffffffu, khi, o));
  }
  // the warp walks the union of its pixels' slab ranges (shuffles need all lanes)
  int wlo = klo, whi = khi;
  for (int o = 4; o <= 16; o <<= 1) {
    wlo = min(wlo, __shfl_xor_sync(0xffffffffu, wlo, o));
    whi = max(whi, __shfl_xor_sync(0xffffffffu, whi, o));
  }
  const size_t pix = (size_t)y * pitchE + x;
  for (int k = wlo; k <= whi; ++k) {
    float v = 0.0f;
    if (hitray && k >= klo && k <= khi)
      v = axis_ray_sum<VT, ZMAJ, SM, SN>(c, C, s, fmaxf(tin, slabs.bound[k]), fminf(tout, slabs.bound[k + 1]), true);
    v = quad_sum_ordered(v);
    if (active && sub == 0 && k >= klo && k <= khi) imgs[(size_t)k * img_stride + pix] = v * c.vs.x * 0.15f * 0.25f;
  }
}

// Beam directions whose rays all stay in one y plane take the axis kernels.
bool axis_projection(const KConst& c) { return fabsf(c.n.y) <= 1e-6f; }

// Instance of the axis kernels for the launch's beam direction: major axis z
// when |dq.z| >= |dq.x| (as each ray decides it), step signs.
void axis_orientation(const KConst& c, bool& zmaj, int& sm, int& sn) {
  const float qx = c.n.x * c.bbRcp.x * c.dim.x, qz = c.n.z * c.bbRcp.z * c.dim.z;
  zmaj = fabsf(qz) >= fabsf(qx);
  const float m = zmaj ? qz : qx, n = zmaj ? qx : qz;
  sm = m < 0.f ? -1 : 1;
  sn = n < 0.f ? -1 : 1;
}

// Volumes of 2^32 voxels or more take 64-bit element offsets in the walk.
bool big_volume(const KConst& c) { return (double)c.dim.x * c.dim.y * c.dim.z > 4294967295.0; }

}  // namespace

// nw: warps per block (2, 4 or 8; 64-bit-offset volumes always take 4).

// One launch of an axis kernel instance per beam orientation.
#define ESB_AXIS_ORIENT(KER, VT, GRD, BLK, ST, ...)                              \
  do {                                                                          \
    bool zmaj_;                                                                 \
    int sm_, sn_;                                                               \
    axis_orientation(c, zmaj_, sm_, sn_);                                       \
    const int o_ = (zmaj_ ? 4 : 0) + (sm_ > 0 ? 2 : 0) + (sn_ > 0 ? 1 : 0);     \
    switch (o_) {                                                               \
      case 0: KER<VT, false, -1, -1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;  \
      case 1: KER<VT, false, -1, 1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;   \
      case 2: KER<VT, false, 1, -1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;   \
      case 3: KER<VT, false, 1, 1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;    \
      case 4: KER<VT, true, -1, -1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;   \
      case 5: KER<VT, true, -1, 1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;    \
      case 6: KER<VT, true, 1, -1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;    \
      default: KER<VT, true, 1, 1><<<GRD, BLK, 0, ST>>>(__VA_ARGS__); break;    \
    }                                                                           \
  } while (0)

cudaError_t launch_slicer_fused(const KConst& c, const void* vol, int vt, float* imgs, size_t img_stride,
                                size_t pitchE, const SlabTable& slabs, int x0, int y0, int x1, int y1,
                                cudaStream_t st, int nw) {
  if (x1 <= x0 || y1 <= y0 || slabs.count <= 0) return cudaSuccess;
  if (axis_projection(c)) {  // the axis walk, one sub-ray per thread
    if (nw != 2 && nw != 8) nw = 4;
    dim3 blk(32 * nw), grd((x1 - x0 + nw - 1) / nw, (y1 - y0 + 7) / 8);
    if (vt == ESB_VOXEL_F32)
      ESB_AXIS_ORIENT(k_slicer_axis, ESB_VOXEL_F32, grd, blk, st, c, vol, imgs, img_stride, pitchE, slabs, x0, y0, x1, y1);
    else if (vt == ESB_VOXEL_F16)
      ESB_AXIS_ORIENT(k_slicer_axis, ESB_VOXEL_F16, grd, blk, st, c, vol, imgs, img_stride, pitchE, slabs, x0, y0, x1, y1);
    else
      ESB_AXIS_ORIENT(k_slicer_axis, ESB_VOXEL_BF16, grd, blk, st, c, vol, imgs, img_stride, pitchE, slabs, x0, y0, x1, y1);
    ESB_COUNT_LAUNCH();
    return cudaGetLastError();
  }
  const bool big = big_volume(c);
  if (big || (nw != 2 && nw != 8)) nw = 4;
  dim3 blk(32 * nw), grd((x1 - x0 + nw - 1) / nw, (y1 - y0 + 7) / 8);
#define ESB_LAUNCH(VT, OFF, NW) \
  k_slicer_fused<VT, OFF, NW><<<grd, blk, 0, st>>>(c, vol, imgs, img_stride, pitchE, slabs, x0, y0, x1, y1)
#define ESB_LAUNCH_VT(OFF, NW)                                  \
  do {                                                          \
    if (vt == ESB_VOXEL_F32) ESB_LAUNCH(ESB_VOXEL_F32, OFF, NW);   \
    else if (vt == ESB_VOXEL_F16) ESB_LAUNCH(ESB_VOXEL_F16, OFF, NW); \
    else ESB_LAUNCH(ESB_VOXEL_BF16, OFF, NW);                   \
  } while (0)
  if (big) ESB_LAUNCH_VT(unsigned long long, 4);
  else if (nw == 2) ESB_LAUNCH_VT(unsigned, 2);
  else if (nw == 8) ESB_LAUNCH_VT(unsigned, 8);
  else ESB_LAUNCH_VT(unsigned, 4);
#undef ESB_LAUNCH_VT
#undef ESB_LAUNCH
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_project_fast(const KConst& c, const void* vol, int vt, int mode, float* proj, float* dist,
                                size_t pitchE, float tmin, float tmax, int x0, int y0, int x1, int y1,
                                cudaStream_t st, int nw) {
  if (x1 <= x0 || y1 <= y0) return cudaSuccess;
  if (mode == 0 && axis_projection(c)) {  // the axis walk, one sub-ray per thread
    if (nw != 2 && nw != 8) nw = 4;
    dim3 blk(32 * nw), grd((x1 - x0 + nw - 1) / nw, (y1 - y0 + 7) / 8);
    if (vt == ESB_VOXEL_F32)
      ESB_AXIS_ORIENT(k_project_axis, ESB_VOXEL_F32, grd, blk, st, c, vol, proj, dist, pitchE, x0, y0, x1, y1);
    else if (vt == ESB_VOXEL_F16)
      ESB_AXIS_ORIENT(k_project_axis, ESB_VOXEL_F16, grd, blk, st, c, vol, proj, dist, pitchE, x0, y0, x1, y1);
    else
      ESB_AXIS_ORIENT(k_project_axis, ESB_VOXEL_BF16, grd, blk, st, c, vol, proj, dist, pitchE, x0, y0, x1, y1);
    ESB_COUNT_LAUNCH();
    return cudaGetLastError();
  }
  const bool big = big_volume(c);
  if (big || (nw != 2 && nw != 8)) nw = 4;
  dim3 blk(32 * nw), grd((x1 - x0 + nw - 1) / nw, (y1 - y0 + 7) / 8);
#define ESB_LAUNCH(VT, M, OFF, NW) \
  k_project_fast<VT, M, OFF, NW><<<grd, blk, 0, st>>>(c, vol, proj, dist, pitchE, tmin, tmax, x0, y0, x1, y1)
#define ESB_LAUNCH_VT(M, OFF, NW)                                  \
  do {                                                             \
    if (vt == ESB_VOXEL_F32) ESB_LAUNCH(ESB_VOXEL_F32, M, OFF, NW);   \
    else if (vt == ESB_VOXEL_F16) ESB_LAUNCH(ESB_VOXEL_F16, M, OFF, NW); \
    else ESB_LAUNCH(ESB_VOXEL_BF16, M, OFF, NW);                   \
  } while (0)
#define ESB_LAUNCH_NW(M)                                      \
  do {                                                        \
    if (big) ESB_LAUNCH_VT(M, unsigned long long, 4);          \
    else if (nw == 2) ESB_LAUNCH_VT(M, unsigned, 2);           \
    else if (nw == 8) ESB_LAUNCH_VT(M, unsigned, 8);           \
    else ESB_LAUNCH_VT(M, unsigned, 4);                        \
  } while (0)
  if (mode == 0) ESB_LAUNCH_NW(0);
  else ESB_LAUNCH_NW(1);
#undef ESB_LAUNCH_NW
#undef ESB_LAUNCH_VT
#undef ESB_LAUNCH
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace esb
