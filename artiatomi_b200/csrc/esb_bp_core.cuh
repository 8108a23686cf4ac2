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
                                           float& dacc, const float2* __restrict__ up = nullptr, int upH = 0) {
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
      const float2* p = up + mu0 * (size_t)upH + (size_t)(int)(py * fos - 0.5f);
#pragma unroll 1
      for (float px = px0; px < (float)pby && px <= ub; px = fadd(px, inv)) {
        const float L = chord(dx, dy, dz, g);
        if (L > 0.0f) {
          a += __ldg(p).x * L;
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

// Voxel row of a sample's ray in a single-axis projection. With n.y = 0 a
// ray runs parallel to the voxels' y faces, so it passes through a voxel
// row fully or not at all: the row test is a step. Where the sub-pixel
// sample grid lines up with the voxel grid (the in-plane rotation of the
// tilt axis makes some detector region do so on every projection) rays
// graze the faces within ~1e-5 of a voxel, and an offset taken from a
// voxel centre's float detector coordinate decides them at random. The
// test is therefore made from the world y of the ray of sample (mu, mv) at
// the volume's centre depth, Y = ry0 + mu u + mv v with u = u_pitch.y / os
// and v = v_pitch.y / os (exact floats for power-of-two os), taken relative
// to a voxel row without rounding error in its large terms (row_offset).
// A is ry0 - bbMin.y - vs / 2 as an unevaluated float pair (A + Al).
struct RowGeom {
  float A, Al;
  float u, v;  // Y per sample along the detector's u and v axes
  float vs;    // voxel size in y
  int ny;      // voxel rows
};

inline RowGeom make_row_geom(const KConst& k, int os) {
  RowGeom r;
  double t0 = 0.0;  // depth of the volume's centre along n from the detector plane
  const double nn[3] = {k.n.x, k.n.y, k.n.z}, dd[3] = {k.det.x, k.det.y, k.det.z};
  const double lo[3] = {k.bbMin.x, k.bbMin.y, k.bbMin.z}, hv[3] = {k.vs.x, k.vs.y, k.vs.z};
  const double nd[3] = {k.dim.x, k.dim.y, k.dim.z};
  for (int j = 0; j < 3; ++j) t0 += nn[j] * (lo[j] + 0.5 * hv[j] * nd[j] - dd[j]);
  r.u = k.u.y / (float)os;
  r.v = k.v.y / (float)os;
  const double ry0 = (double)k.det.y + t0 * (double)k.n.y + 0.5 * ((double)r.u + (double)r.v);
  const double A = ry0 - (double)k.bbMin.y - 0.5 * (double)k.vs.y;
  r.A = (float)A;
  r.Al = (float)(A - (double)r.A);
  r.vs = k.vs.y;
  r.ny = (int)k.dim.y;
  return r;
}

// Error-free transformations (Knuth's two-sum, and the product's rounding
// error from a fused multiply-add): s + e == a + b and p + e == a * b
// exactly.
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
__device__ __forceinline__ void two_prod(float a, float b, float& p, float& e) {
  p = __fmul_rn(a, b);
  e = __fmaf_rn(a, b, -p);
}

// Offset of the ray of sample (mu, mv) from the centre plane of voxel row
// yrow: A + mu u + mv v - yrow vs. The terms are hundreds of voxels while
// the sum near a voxel is below about a voxel, so it is formed without
// rounding error in the large terms; the result is exact to its own float
// rounding.
__device__ __forceinline__ float row_offset(const RowGeom& r, int yrow, int mu, int mv) {
  float p1, e1, p2, e2, p3, e3, s1, t1, s2, t2, s3, t3;
  two_prod((float)mu, r.u, p1, e1);
  two_prod((float)mv, r.v, p2, e2);
  two_prod(-(float)yrow, r.vs, p3, e3);
  two_sum(r.A, p1, s1, t1);
  two_sum(s1, p3, s2, t2);
  two_sum(s2, p2, s3, t3);
  return __fadd_rn(s3, __fadd_rn(__fadd_rn(__fadd_rn(r.Al, e1), __fadd_rn(e2, e3)), __fadd_rn(t1, __fadd_rn(t2, t3))));
}

// Voxel row whose interior holds the ray of sample (mu, mv), or -1 (a ray on
// a face, or outside the volume): the reference's slab test evaluated
// exactly, which counts a ray strictly inside the row.
__device__ __forceinline__ int sample_row(const RowGeom& r, int mu, int mv) {
  const float h = 0.5f * r.vs;
  int y = (int)floorf(row_offset(r, 0, mu, mv) / r.vs + 0.5f);  // within a row of the answer
  float o = row_offset(r, y, mu, mv);
  if (o >= h) {
    ++y;
    o = row_offset(r, y, mu, mv);
  } else if (o <= -h) {
    --y;
    o = row_offset(r, y, mu, mv);
  }
  return (fabsf(o) < h && y >= 0 && y < r.ny) ? y : -1;
}

// Geometry of the single-axis back-projection (axis_sums): tilt axis along
// y (n.y = 0), power-of-two oversampling, no magnification anisotropy.
struct AxisGeom {
  float3 U, V;     // detector coordinate of a world point: u = U.p + U0, v = V.p + V0
  float U0, V0;
  float hu, hv;    // half shadow extents in pixels (as BpGeom)
  float wu, wv;    // in-plane offset of a sample perpendicular to n in x-z, per pixel of u and v
  float yu, yv;    // its y component per pixel of u and v
  float hby;       // half voxel size in y
  RowGeom r;       // the row test of a sample's ray (RowGeom)
  float L0, w1K, K;  // chord trapezoid: L(w) = min(L0, max(0, w1K - |w| K))
  // macro-cell rectangle of quad (x, y, z), affine in the quad position:
  // u_lo/hi = ru.w + x ru.x + y ru.y + z ru.z + (ulo, uhi), same for v
  float4 ru, rv;
  float ulo, uhi, vlo, vhi;
  // The rectangle can be smaller than the macro cell's shadow (detector axes
  // rotated against the volume axes). Its integer bounds (floor / ceil of the
  // extremes) decide which samples of the clipped band are taken; the affine
  // extremes agree with the reference's to ~1e-3 pixel, so they give the
  // same samples unless the band reaches the nearest sub-pixel sample beyond
  // an integer bound (0.5 / os). Then the rectangle is evaluated per quad
  // with the reference's expressions (macro_footprint).
  int clips;
};

// Depth of the macro cell's first corner (macro_footprint's corner 0, the
// reference's expression), which selects the quad's CTF slab.
__device__ __forceinline__ float macro_depth(const KConst& k, int x, int y, int z) {
  const float mnx = fadd(k.bbMin.x, fmul((float)x, k.vs.x)), mny = fadd(k.bbMin.y, fmul((float)y, k.vs.y)),
              mnz = fadd(k.bbMin.z, fmul((float)z, k.vs.z));
  const float ndet = fadd(fadd(fmul(-k.n.x, k.det.x), -fmul(k.n.y, k.det.y)), -fmul(k.n.z, k.det.z));
  const float t = fadd(fadd(fmul(k.n.x, mnx), fmul(k.n.y, mny)), fmul(k.n.z, mnz));
  return fabsf(fadd(t, ndet));
}

// The reference's macro-cell rectangle (macro_footprint): the cell's 8
// corners are projected along n onto the detector plane, the bounding box
// (lo, hi) of those hit points is taken in world coordinates (x swapped when
// n.x <= 0) and only lo and hi are mapped to the detector. With the hit point
// h = A p + b linear in the corner p, lo and hi are affine in the quad
// position, and so are their detector coordinates; the rectangle is the
// reference's up to float rounding. It can be smaller than the voxels'
// shadows when the detector axes are rotated against the volume axes, and
// then clips samples as the reference does.
__device__ __forceinline__ void macro_rect(const AxisGeom& g, int x, int y, int z, int pw, int ph, int& pbx, int& pby,
                                           int& pbz, int& pbw) {
  const float uL = fmaf((float)z, g.ru.z, fmaf((float)y, g.ru.y, fmaf((float)x, g.ru.x, g.ru.w)));
  const float vL = fmaf((float)z, g.rv.z, fmaf((float)y, g.rv.y, fmaf((float)x, g.rv.x, g.rv.w)));
  const float plx = uL + g.ulo, phx = uL + g.uhi, ply = vL + g.vlo, phy = vL + g.vhi;
  pbx = (int)fminf(fmaxf(floorf(fminf(plx, phx)), 0.0f), (float)(pw - 1));
  pby = (int)fminf(fmaxf(ceilf(fmaxf(plx, phx)), 0.0f), (float)(pw - 1));
  pbz = (int)fminf(fmaxf(floorf(fminf(ply, phy)), 0.0f), (float)(ph - 1));
  pbw = (int)fminf(fmaxf(ceilf(fmaxf(ply, phy)), 0.0f), (float)(ph - 1));
}

inline AxisGeom make_axis_geom(const KConst& k, const BpGeom& b, int os) {
  AxisGeom g;
  g.U = b.U;
  g.V = b.V;
  g.U0 = b.U0;
  g.V0 = b.V0;
  g.hu = b.hu;
  g.hv = b.hv;
  // offset d = du * u + dv * v; w = d.x n.z - d.z n.x
  g.wu = k.u.x * k.n.z - k.u.z * k.n.x;
  g.wv = k.v.x * k.n.z - k.v.z * k.n.x;
  g.yu = k.u.y;
  g.yv = k.v.y;
  g.hby = b.hb.y;
  g.r = make_row_geom(k, os);
  const float anx = fabsf(k.n.x), anz = fabsf(k.n.z);
  const float hx = b.hb.x, hz = b.hb.z;
  g.L0 = fminf(anx > 0.f ? 2.f * hx / anx : FLT_MAX, anz > 0.f ? 2.f * hz / anz : FLT_MAX);
  const float prod = anx * anz;
  g.K = prod > 1e-30f ? 1.0f / prod : 1e30f;
  g.w1K = (hx * anz + hz * anx) * g.K;
  // macro-cell rectangle: h = A p + b with A = I - sg n n^T, b = -sg ndet n,
  // sg the sign of n.p + ndet over the volume (the detector lies outside it)
  const double n[3] = {k.n.x, k.n.y, k.n.z};
  const double det[3] = {k.det.x, k.det.y, k.det.z};
  const double ndet = -n[0] * det[0] - n[1] * det[1] - n[2] * det[2];
  const double bmin[3] = {k.bbMin.x, k.bbMin.y, k.bbMin.z}, vs[3] = {k.vs.x, k.vs.y, k.vs.z};
  const double ext[3] = {5.0 * vs[0], vs[1], vs[2]};  // the 5 x 1 x 1 macro cell
  const double dim[3] = {k.dim.x, k.dim.y, k.dim.z};
  double ctr = ndet;  // n.p + ndet at the volume centre
  for (int j = 0; j < 3; ++j) ctr += n[j] * (bmin[j] + 0.5 * vs[j] * dim[j]);
  const double sg = ctr < 0.0 ? -1.0 : 1.0;
  double A[3][3], base[3], dlo[3], dhi[3];
  for (int r = 0; r < 3; ++r) {
    base[r] = -sg * ndet * n[r];
    dlo[r] = dhi[r] = 0.0;
    for (int c = 0; c < 3; ++c) {
      A[r][c] = (r == c ? 1.0 : 0.0) - sg * n[r] * n[c];
      base[r] += A[r][c] * bmin[c];
      const double e = A[r][c] * ext[c];
      dlo[r] += e < 0.0 ? e : 0.0;
      dhi[r] += e > 0.0 ? e : 0.0;
    }
  }
  if (k.n.x <= 0.0f) {  // the reference swaps lo.x and hi.x
    const double t = dlo[0];
    dlo[0] = dhi[0];
    dhi[0] = t;
  }
  const double U[3] = {b.U.x, b.U.y, b.U.z}, V[3] = {b.V.x, b.V.y, b.V.z};
  double ru[4] = {0, 0, 0, b.U0}, rv[4] = {0, 0, 0, b.V0};
  double ulo = 0, uhi = 0, vlo = 0, vhi = 0;
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) {
      ru[c] += U[r] * A[r][c] * vs[c];
      rv[c] += V[r] * A[r][c] * vs[c];
    }
    ru[3] += U[r] * base[r];
    rv[3] += V[r] * base[r];
    ulo += U[r] * dlo[r];
    uhi += U[r] * dhi[r];
    vlo += V[r] * dlo[r];
    vhi += V[r] * dhi[r];
  }
  // true extent of the macro cell's shadow around the projection of A m:
  // sum_c min/max(0, (U A)_c ext_c); the rectangle clips when its own
  // extent (U dlo, U dhi) is narrower
  double su_lo = 0, su_hi = 0, sv_lo = 0, sv_hi = 0;
  for (int c = 0; c < 3; ++c) {
    double ua = 0, va = 0;
    for (int r = 0; r < 3; ++r) {
      ua += U[r] * A[r][c];
      va += V[r] * A[r][c];
    }
    su_lo += ua * ext[c] < 0 ? ua * ext[c] : 0;
    su_hi += ua * ext[c] > 0 ? ua * ext[c] : 0;
    sv_lo += va * ext[c] < 0 ? va * ext[c] : 0;
    sv_hi += va * ext[c] > 0 ? va * ext[c] : 0;
  }
  const double band = fmax(fmax(fmin(ulo, uhi) - su_lo, su_hi - fmax(ulo, uhi)),
                           fmax(fmin(vlo, vhi) - sv_lo, sv_hi - fmax(vlo, vhi)));
  g.clips = band > 0.5 / os - 0.01 ? 1 : 0;
  g.ru = make_float4((float)ru[0], (float)ru[1], (float)ru[2], (float)ru[3]);
  g.rv = make_float4((float)rv[0], (float)rv[1], (float)rv[2], (float)rv[3]);
  g.ulo = (float)ulo;
  g.uhi = (float)uhi;
  g.vlo = (float)vlo;
  g.vhi = (float)vhi;
  return g;
}

// Whether a projection takes the single-axis sums: beam without a y
// component, exact sub-pixel lattice, samples read at (px, py).
inline bool axis_eligible(const KConst& k, const BpGeom& g) {
  return g.exact_grid && g.aniso_identity && fabsf(k.n.y) <= 1e-6f;
}

// row_offset of the samples of the voxels of one row (the 4 voxels of a
// quad): formed once, at sample (mu, mv) near the first voxel's centre
// projection (|y| below about a voxel), and stepped from there in float by
// the few sample positions to each voxel's first sample, which keeps the
// value exact to float rounding of a sub-voxel offset.
struct RowAnchor {
  int mu, mv;
  float y;
  __device__ __forceinline__ RowAnchor(const AxisGeom& g, int yrow, float uc, float vc, float fos)
      : mu((int)floorf(uc * fos)), mv((int)floorf(vc * fos)) {
    y = row_offset(g.r, yrow, mu, mv);
  }
  __device__ __forceinline__ float at(const AxisGeom& g, int mu_, int mv_) const {
    return fmaf((float)(mv_ - mv), g.r.v, fmaf((float)(mu_ - mu), g.r.u, y));
  }
};

// sum(sample*chord) and sum(chord) of one voxel (of the row of `anchor`)
// whose centre projects to (uc, vc), for a single-axis projection. With
// n.y = 0 the chord of a sample's ray through the voxel depends only on the
// ray's offset w from the voxel centre perpendicular to n in the x-z plane
// (a trapezoid: the plateau min(2 hx / |n.x|, 2 hz / |n.z|), falling
// linearly to 0 at |w| = hx |n.z| + hz |n.x| with slope 1 / (|n.x| |n.z|)),
// and is 0 where the ray lies outside the voxel row (RowGeom). Samples are
// the sub-pixel grid points (m + 0.5) / os inside the voxel's shadow and
// inside [mu_min, mu_max] x [mv_min, mv_max] (the quad's macro-cell
// rectangle); read(mu, mv) returns the image at grid point (mu, mv), a
// filtered read taken only for samples with a nonzero chord.
template <class Read>
__device__ __forceinline__ void axis_sums(const AxisGeom& g, float uc, float vc, float fos, float inv, float dwv,
                                          const RowAnchor& anchor, int mu_min, int mu_max, int mv_min, int mv_max,
                                          const Read& read, float& acc, float& dacc) {
  const int mu0 = max((int)ceilf((uc - g.hu) * fos - 0.5f), mu_min);
  const int mu1 = min((int)floorf((uc + g.hu) * fos - 0.5f), mu_max);
  const int mv0 = max((int)ceilf((vc - g.hv) * fos - 0.5f), mv_min);
  const int mv1 = min((int)floorf((vc + g.hv) * fos - 0.5f), mv_max);
  const float dv0 = ((float)mv0 + 0.5f) * inv - vc;
  float a = 0.f, da = 0.f;
  const int rows = mu1 - mu0 + 1;
  const int cnt = mv1 - mv0 + 1;
  const float y00 = anchor.at(g, mu0, mv0);
#pragma unroll 1
  for (int r = 0; r < rows; ++r) {
    const int mu = mu0 + r;
    const float du = ((float)mu + 0.5f) * inv - uc;
    const float w = du * g.wu + dv0 * g.wv, dy = fmaf((float)r, g.r.u, y00);
#pragma unroll 1
    for (int j = 0; j < cnt; ++j) {
      const float ww = fmaf((float)j, dwv, w), yy = fmaf((float)j, g.r.v, dy);
      const float L = fminf(g.L0, fmaxf(0.f, fmaf(-fabsf(ww), g.K, g.w1K)));
      if (fabsf(yy) < g.hby && L > 0.f) {
        a = fmaf(read(mu, mv0 + j), L, a);
        da += L;
      }
    }
  }
  acc = a;
  dacc = da;
}

// axis_sums on images pre-sampled with the voxel row of every sample's ray
// (k_upsample): read(mu, mv) returns (value, row as int bits), and a sample
// counts for voxel row yrow when its row is yrow. One 8-byte load per sample;
// the first 2 x 3 samples of a voxel's shadow are unrolled and read
// unconditionally.
template <class Read>
__device__ __forceinline__ void axis_sums_rows(const AxisGeom& g, float uc, float vc, float fos, float inv, float dwv,
                                               int yrow, int mu_min, int mu_max, int mv_min, int mv_max,
                                               const Read& read, float& acc, float& dacc) {
  const int mu0 = max((int)ceilf((uc - g.hu) * fos - 0.5f), mu_min);
  const int mu1 = min((int)floorf((uc + g.hu) * fos - 0.5f), mu_max);
  const int mv0 = max((int)ceilf((vc - g.hv) * fos - 0.5f), mv_min);
  const int mv1 = min((int)floorf((vc + g.hv) * fos - 0.5f), mv_max);
  const float dv0 = ((float)mv0 + 0.5f) * inv - vc;
  float a = 0.f, da = 0.f;
  // a voxel's shadow holds 2-3 sub-pixel samples per axis at OS 2
  const int rows = mu1 - mu0 + 1;
  const int cnt = mv1 - mv0 + 1;
  auto row = [&](int mu) {
    const float du = ((float)mu + 0.5f) * inv - uc;
    const float w = du * g.wu + dv0 * g.wv;
    auto body = [&](int j) {
      const float ww = fmaf((float)j, dwv, w);
      const float2 s = read(mu, mv0 + j);
      float L = fminf(g.L0, fmaxf(0.f, fmaf(-fabsf(ww), g.K, g.w1K)));
      L = __float_as_int(s.y) == yrow ? L : 0.f;
      a = fmaf(s.x, L, a);
      da += L;
    };
#pragma unroll
    for (int j = 0; j < 3; ++j)
      if (j < cnt) body(j);
#pragma unroll 1
    for (int j = 3; j < cnt; ++j) body(j);
  };
#pragma unroll
  for (int r = 0; r < 2; ++r)
    if (r < rows) row(mu0 + r);
#pragma unroll 1
  for (int r = 2; r < rows; ++r) row(mu0 + r);
  acc = a;
  dacc = da;
}


// axis_sums for oversampling 2 with bilinear reads of an image whose samples
// all lie in its interior (texel (ix, iy) at img + ix * sx + iy * sy). The
// sub-pixel samples then sit at quarter-texel offsets: sample m reads the
// texel pair ((m - 1) >> 1, +1) with weight 0.75 on the second texel for m
// even and 0.25 for m odd. The (up to) 3 x 3 samples of a voxel's shadow
// therefore read one 3 x 3 texel patch: it is loaded once, each sample's
// value is formed from it exactly as sample_interior forms it (x then y),
// and the samples are weighted by their chords. Returns false (nothing
// accumulated) when the shadow holds more than 3 samples along an axis.
__device__ __forceinline__ bool axis_sums_os2(const AxisGeom& g, float uc, float vc, float dwv,
                                              const RowAnchor& anchor, int mu_min,
                                              int mu_max, int mv_min, int mv_max, const float* __restrict__ img,
                                              size_t sx, size_t sy, int pw, int ph, float& acc, float& dacc) {
  const int mu0 = max((int)ceilf((uc - g.hu) * 2.0f - 0.5f), mu_min);
  const int mu1 = min((int)floorf((uc + g.hu) * 2.0f - 0.5f), mu_max);
  const int mv0 = max((int)ceilf((vc - g.hv) * 2.0f - 0.5f), mv_min);
  const int mv1 = min((int)floorf((vc + g.hv) * 2.0f - 0.5f), mv_max);
  const int nu = mu1 - mu0 + 1, nv = mv1 - mv0 + 1;
  if (nu > 3 || nv > 3) return false;
  if (nu <= 0 || nv <= 0) {
    acc = 0.f;
    dacc = 0.f;
    return true;
  }
  const int fxa = (mu0 - 1) >> 1, fya = (mv0 - 1) >> 1;
  float T[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const size_t col = (size_t)min(fxa + c, pw - 1) * sx;
#pragma unroll
    for (int r = 0; r < 3; ++r) T[c][r] = __ldg(img + col + (size_t)min(fya + r, ph - 1) * sy);
  }
  const bool ou = (mu0 & 1) != 0, ov = (mv0 & 1) != 0;
  // sample columns: texel pair and weight of the second texel
  const float a0 = ou ? 0.25f : 0.75f, a1 = ou ? 0.75f : 0.25f, a2 = a0;
  const float b0 = ov ? 0.25f : 0.75f, b1 = ov ? 0.75f : 0.25f, b2 = b0;
  float C[3][3];  // C[i][r]: sample column i interpolated at texel row r
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    C[0][r] = (1.0f - a0) * T[0][r] + a0 * T[1][r];
    const float l1 = ou ? T[0][r] : T[1][r], h1 = ou ? T[1][r] : T[2][r];
    C[1][r] = (1.0f - a1) * l1 + a1 * h1;
    C[2][r] = (1.0f - a2) * T[1][r] + a2 * T[2][r];
  }
  const float du0 = ((float)mu0 + 0.5f) * 0.5f - uc, dv0 = ((float)mv0 + 0.5f) * 0.5f - vc;
  const float w0 = du0 * g.wu + dv0 * g.wv, y0 = anchor.at(g, mu0, mv0);
  const float dwu = 0.5f * g.wu;
  float a = 0.f, da = 0.f;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float ww = fmaf((float)j, dwv, fmaf((float)i, dwu, w0));
      const float yy = fmaf((float)j, g.r.v, fmaf((float)i, g.r.u, y0));
      float L = fminf(g.L0, fmaxf(0.f, fmaf(-fabsf(ww), g.K, g.w1K)));
      L = (fabsf(yy) < g.hby && i < nu && j < nv) ? L : 0.f;
      const float bj = j == 0 ? b0 : (j == 1 ? b1 : b2);
      const float lo = j == 0 ? C[i][0] : (j == 1 ? (ov ? C[i][0] : C[i][1]) : C[i][1]);
      const float hi = j == 0 ? C[i][1] : (j == 1 ? (ov ? C[i][1] : C[i][2]) : C[i][2]);
      const float v = (1.0f - bj) * lo + bj * hi;
      a = fmaf(v, L, a);
      da += L;
    }
  }
  acc = a;
  dacc = da;
  return true;
}


}  // namespace bpcore
}  // namespace esb
