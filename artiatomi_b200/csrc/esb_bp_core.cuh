// Device core of the per-voxel-shadow back-projection, shared by the
// single-volume kernel (esb_backprojector_fast.cu) and the batched sub-volume
// kernel (esb_subvolume.cu).
#pragma once

#include <float.h>

#include "esb_device.cuh"

namespace esb {
namespace bpcore {

// Image texel (ix, iy): row-major [y][x] with pitch, or transposed [x][y]
// (the reconstructor's layout: threads of a warp walk the volume's x axis,
// which maps to the detector's y axis, so a transposed image keeps their
// reads contiguous).
__device__ __forceinline__ float texel(const float* __restrict__ img, int h, size_t pitchE, bool transposed, int ix,
                                       int iy) {
  return __ldg(img + (transposed ? (size_t)ix * h + iy : (size_t)iy * pitchE + ix));
}

__device__ __forceinline__ float sample_image(const float* __restrict__ img, int w, int h, size_t pitchE, float x,
                                              float y, bool linear, bool transposed) {
  if (!linear) {
    int ix = clamp_texel(floorf(x), w), iy = clamp_texel(floorf(y), h);
    return texel(img, h, pitchE, transposed, ix, iy);
  }
  float xb = x - 0.5f, yb = y - 0.5f;
  float fx = floorf(xb), fy = floorf(yb);
  float a = xb - fx, b = yb - fy;
  int x0 = clamp_texel(fx, w), x1 = clamp_texel(fx + 1.0f, w);
  int y0 = clamp_texel(fy, h), y1 = clamp_texel(fy + 1.0f, h);
  float t00 = texel(img, h, pitchE, transposed, x0, y0), t10 = texel(img, h, pitchE, transposed, x1, y0);
  float t01 = texel(img, h, pitchE, transposed, x0, y1), t11 = texel(img, h, pitchE, transposed, x1, y1);
  return (1.0f - b) * ((1.0f - a) * t00 + a * t10) + b * ((1.0f - a) * t01 + a * t11);
}

struct BpGeom {
  // detector coordinate of a world point p: u = U.p + U0, v = V.p + V0
  float3 U, V;
  float U0, V0;
  float3 u, v;   // detector axes (world per pixel)
  float3 inv_n;  // 1 / ray direction per axis
  // entry and exit face offsets per axis: the ray c + d + tau*n enters the
  // slab |p - c| <= hb of axis j at tau = (cn_j - d_j) / n_j and leaves it
  // at (cf_j - d_j) / n_j (cn = -hb, cf = +hb for n_j > 0, swapped else)
  float3 cn, cf;
  float hu, hv;  // half extent of a voxel's shadow in pixels
  float3 hb;     // half voxel size
  int exact_grid;      // oversampling is a power of two: the recurrence is exact
  int aniso_identity;  // no magnification anisotropy: samples read at (px, py)
};

__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }

// Chord of the line c + d + tau*n through the box |p - c| <= hb per axis.
// With the entry/exit faces resolved by the sign of n, each axis costs two
// subtractions and two products; a zero component (1/n infinite) leaves the
// axis unconstrained while |d| < hb and empties the chord when |d| > hb.
__device__ __forceinline__ float chord(float dx, float dy, float dz, const BpGeom& g) {
  const float tin = fmaxf(fmaxf((g.cn.x - dx) * g.inv_n.x, (g.cn.y - dy) * g.inv_n.y), (g.cn.z - dz) * g.inv_n.z);
  const float tout = fminf(fminf((g.cf.x - dx) * g.inv_n.x, (g.cf.y - dy) * g.inv_n.y), (g.cf.z - dz) * g.inv_n.z);
  return tout - tin;
}

// Macro-cell rectangle of the quad (BackProjectionSquareOS.cu:344-509),
// evaluated with the reference's expressions; returns false when the quad's
// first corner is outside [distMin, distMax) (or its depth in *depth).
__device__ __forceinline__ void macro_footprint(const KConst& k, int x, int y, int z, int pw, int ph, float& depth,
                                                int& pbx, int& pby, int& pbz, int& pbw) {
  const float mnx = fadd(k.bbMin.x, fmul((float)x, k.vs.x)), mny = fadd(k.bbMin.y, fmul((float)y, k.vs.y)),
              mnz = fadd(k.bbMin.z, fmul((float)z, k.vs.z));
  const float mxx = fadd(k.bbMin.x, fmul((float)(x + 5), k.vs.x)), mxy = fadd(k.bbMin.y, fmul((float)(y + 1), k.vs.y)),
              mxz = fadd(k.bbMin.z, fmul((float)(z + 1), k.vs.z));
  const float ndet = fadd(fadd(fmul(-k.n.x, k.det.x), -fmul(k.n.y, k.det.y)), -fmul(k.n.z, k.det.z));
  float bminx = FLT_MAX, bminy = FLT_MAX, bminz = FLT_MAX;
  float bmaxx = -200000.f, bmaxy = -200000.f, bmaxz = -200000.f;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const float px = (c & 4) ? fadd(mnx, fadd(mxx, -mnx)) : mnx;
    const float py = (c & 2) ? fadd(mny, fadd(mxy, -mny)) : mny;
    const float pz = (c & 1) ? fadd(mnz, fadd(mxz, -mnz)) : mnz;
    float t = fadd(fadd(fmul(k.n.x, px), fmul(k.n.y, py)), fmul(k.n.z, pz));
    t = fabsf(fadd(t, ndet));
    if (c == 0) depth = t;
    const float hx = fadd(fmul(t, -k.n.x), px), hy = fadd(fmul(t, -k.n.y), py), hz = fadd(fmul(t, -k.n.z), pz);
    bminx = fminf(hx, bminx); bminy = fminf(hy, bminy); bminz = fminf(hz, bminz);
    bmaxx = fmaxf(hx, bmaxx); bmaxy = fmaxf(hy, bmaxy); bmaxz = fmaxf(hz, bmaxz);
  }
  float lox = fminf(bminx, bmaxx), loy = fminf(bminy, bmaxy), loz = fminf(bminz, bmaxz);
  float hix = fmaxf(bminx, bmaxx), hiy = fmaxf(bminy, bmaxy), hiz = fmaxf(bminz, bmaxz);
  if (k.n.x <= 0.0f) {
    const float tmp = lox;
    lox = hix;
    hix = tmp;
  }
  auto row = [&](const float4& m, float a, float b, float c) {
    return fadd(fadd(fadd(fmul(m.x, a), fmul(m.y, b)), fmul(m.z, c)), fmul(1.0f, m.w));
  };
  const float plx = row(k.detMat[0], lox, loy, loz), ply = row(k.detMat[1], lox, loy, loz);
  const float phx = row(k.detMat[0], hix, hiy, hiz), phy = row(k.detMat[1], hix, hiy, hiz);
  pbx = (int)floorf(fminf(plx, phx));
  pbz = (int)floorf(fminf(ply, phy));
  pby = (int)ceilf(fmaxf(plx, phx));
  pbw = (int)ceilf(fmaxf(ply, phy));
  pbx = (int)fminf(fmaxf((float)pbx, 0.0f), (float)(pw - 1));
  pby = (int)fminf(fmaxf((float)pby, 0.0f), (float)(pw - 1));
  pbz = (int)fminf(fmaxf((float)pbz, 0.0f), (float)(ph - 1));
  pbw = (int)fminf(fmaxf((float)pbw, 0.0f), (float)(ph - 1));
}

// First sample index and position of the recurrence s_0 = lo + inv/2,
// s_{k+1} = s_k + inv (float) that is >= a.
__device__ __forceinline__ float first_sample(int lo, float inv, float a, bool exact, int os) {
  if (exact) {  // s_k = lo + (k + 0.5)/os exactly
    int k = (int)ceilf((a - (float)lo) * os - 0.5f);
    k = k < 0 ? 0 : k;
    return (float)lo + ((float)k + 0.5f) * inv;
  }
  float s = fadd((float)lo, fmul(inv, 0.5f));
#pragma unroll 1
  for (int guard = 0; s < a && guard < 1 << 16; ++guard) s = fadd(s, inv);
  return s;
}


// Image sample without clamping, for samples known to lie inside the image
// (the generic path's clamps are then no-ops): texel (ix, iy) at
// img + ix * sx + iy * sy.
__device__ __forceinline__ float sample_interior(const float* __restrict__ img, size_t sx, size_t sy, float x,
                                                 float y, bool linear) {
  if (!linear) return __ldg(img + (size_t)(int)x * sx + (size_t)(int)y * sy);  // x, y >= 0
  const float xb = x - 0.5f, yb = y - 0.5f;
  const float fx = floorf(xb), fy = floorf(yb);
  const float a = xb - fx, b = yb - fy;
  const float* p = img + (size_t)(int)fx * sx + (size_t)(int)fy * sy;
  const float t00 = __ldg(p), t10 = __ldg(p + sx), t01 = __ldg(p + sy), t11 = __ldg(p + sx + sy);
  return (1.0f - b) * ((1.0f - a) * t00 + a * t10) + b * ((1.0f - a) * t01 + a * t11);
}

// sum(sample*chord) and sum(chord) of voxel (x + i, y, z) of the quad at
// (x, y, z) whose macro-cell rectangle is pb*, over the reference's sub-pixel
// recurrence restricted to the voxel's shadow.
//
// Samples run over [pbx, pby) x [pbz, pbw) with pby <= pw - 1 and
// pbw <= ph - 1, so a nearest-texel read never leaves the image and a
// bilinear read only does so below a lower edge: with no anisotropy the
// clamps are skipped unless pbx or pbz is 0 under bilinear interpolation.
//
// up (may be NULL): the image pre-sampled at every point of the sub-pixel
// grid, up[mu][mv] = image at ((mu + 0.5) / os, (mv + 0.5) / os) with row
// length upH = ph * os (k_upsample). With a power-of-two oversampling and no
// anisotropy the recurrence visits exactly those points, so each sample is
// one load instead of a filtered read.
__device__ __forceinline__ void voxel_sums(const KConst& k, const BpGeom& g, const float* __restrict__ img, int pw,
                                           int ph, size_t pitchE, int os, float inv, bool linear, bool transposed,
                                           int x, int y, int z, int pbx, int pby, int pbz, int pbw, float& acc,
                                           float& dacc, const float* __restrict__ up = nullptr, int upH = 0) {
  const float cx = k.bbMin.x + ((float)x + 0.5f) * k.vs.x, cy = k.bbMin.y + ((float)y + 0.5f) * k.vs.y,
              cz = k.bbMin.z + ((float)z + 0.5f) * k.vs.z;
  const float uc = g.U.x * cx + g.U.y * cy + g.U.z * cz + g.U0;
  const float vc = g.V.x * cx + g.V.y * cy + g.V.z * cz + g.V0;
  const float ua = uc - g.hu, ub = uc + g.hu, va = vc - g.hv, vb = vc + g.hv;
  const bool exact = g.exact_grid != 0;
  const bool fast = g.aniso_identity != 0 && (!linear || (pbx >= 1 && pbz >= 1));
  const size_t sx = transposed ? (size_t)ph : 1, sy = transposed ? 1 : pitchE;
  float a = 0.f, da = 0.f;
  const float py0 = first_sample(pbz, inv, va, exact, os), px0 = first_sample(pbx, inv, ua, exact, os);
  const float du0 = px0 - uc;
  // in-plane offset d = du * u + dv * v, advanced by inv * u per sample
  const float ix = inv * g.u.x, iy = inv * g.u.y, iz = inv * g.u.z;
  if (up) {
    const float fos = (float)os;
    const size_t mu0 = (size_t)(int)(px0 * fos - 0.5f);  // exact: px0 = (mu0 + 0.5) / os
#pragma unroll 1
    for (float py = py0; py < (float)pbw && py <= vb; py = fadd(py, inv)) {
      const float dv = py - vc;
      float dx = du0 * g.u.x + dv * g.v.x, dy = du0 * g.u.y + dv * g.v.y, dz = du0 * g.u.z + dv * g.v.z;
      const float* p = up + mu0 * (size_t)upH + (size_t)(int)(py * fos - 0.5f);
#pragma unroll 1
      for (float px = px0; px < (float)pby && px <= ub; px = fadd(px, inv)) {
        const float L = chord(dx, dy, dz, g);
        if (L > 0.0f) {
          a += __ldg(p) * L;
          da += L;
        }
        dx += ix;
        dy += iy;
        dz += iz;
        p += upH;
      }
    }
    acc = a;
    dacc = da;
    return;
  }
#pragma unroll 1
  for (float py = py0; py < (float)pbw && py <= vb; py = fadd(py, inv)) {
    const float dv = py - vc;
    float dx = du0 * g.u.x + dv * g.v.x, dy = du0 * g.u.y + dv * g.v.y, dz = du0 * g.u.z + dv * g.v.z;
#pragma unroll 1
    for (float px = px0; px < (float)pby && px <= ub; px = fadd(px, inv)) {
      const float L = chord(dx, dy, dz, g);
      if (L > 0.0f) {
        float s;
        if (fast) {
          s = sample_interior(img, sx, sy, px, py, linear);
        } else {
          const float xA = k.anisoInv[0] * px + k.anisoInv[1] * py + k.anisoInv[2];
          const float yA = k.anisoInv[3] * px + k.anisoInv[4] * py + k.anisoInv[5];
          s = sample_image(img, pw, ph, pitchE, xA, yA, linear, transposed);
        }
        a += s * L;
        da += L;
      }
      dx += ix;
      dy += iy;
      dz += iz;
    }
  }
  acc = a;
  dacc = da;
}

inline BpGeom make_geom(const KConst& k, int os) {
  BpGeom g;
  g.U = make_float3(k.detMat[0].x, k.detMat[0].y, k.detMat[0].z);
  g.V = make_float3(k.detMat[1].x, k.detMat[1].y, k.detMat[1].z);
  g.U0 = k.detMat[0].w;
  g.V0 = k.detMat[1].w;
  g.u = k.u;
  g.v = k.v;
  g.inv_n = make_float3(1.0f / k.n.x, 1.0f / k.n.y, 1.0f / k.n.z);
  g.hb = make_float3(0.5f * k.vs.x, 0.5f * k.vs.y, 0.5f * k.vs.z);
  g.cn = make_float3(signbit(g.inv_n.x) ? g.hb.x : -g.hb.x, signbit(g.inv_n.y) ? g.hb.y : -g.hb.y,
                     signbit(g.inv_n.z) ? g.hb.z : -g.hb.z);
  g.cf = make_float3(-g.cn.x, -g.cn.y, -g.cn.z);
  // shadow half extents, widened by a hair so that samples on the edge of a
  // shadow are tested (their chord decides)
  g.hu = 0.5f * (fabsf(g.U.x) * k.vs.x + fabsf(g.U.y) * k.vs.y + fabsf(g.U.z) * k.vs.z) * 1.0001f + 1e-5f;
  g.hv = 0.5f * (fabsf(g.V.x) * k.vs.x + fabsf(g.V.y) * k.vs.y + fabsf(g.V.z) * k.vs.z) * 1.0001f + 1e-5f;
  g.exact_grid = (os & (os - 1)) == 0;
  static const float ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  g.aniso_identity = 1;
  for (int i = 0; i < 9; ++i)
    if (k.anisoInv[i] != ident[i]) g.aniso_identity = 0;
  return g;
}

}  // namespace bpcore
}  // namespace esb
