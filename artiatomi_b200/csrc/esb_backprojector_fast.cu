// Ray-length-normalised back-projection by per-voxel shadows ("fast").
//
// The reference kernel (BackProjectionSquareOS.cu:263-782) bounds the
// 5x1x1-voxel macro cell of a 4-voxel quad on the detector, walks the
// sub-pixel samples of that rectangle (pixel += 1/OS from the rectangle's
// clamped integer corner) and intersects each sample's ray with each of the
// 4 voxels. Most of those tests miss, and each hit is computed from a ray
// origin 1e5 units away, so float rounding is ~1e-2 on a chord of ~1.
//
// This kernel computes the same macro-cell rectangle and walks the same
// sub-pixel recurrence. For each voxel it visits only the samples inside
// that voxel's own shadow, and computes the chord in voxel-local coordinates:
// the sample's ray is c + d + tau*n, with d the sample's in-plane offset from
// the projected voxel centre c. The result is the reference's
// sum(sample*chord)/sum(chord) over the reference's samples, with exact
// rather than noisy chords.
//
// CTF mode: the reference launches the back-projection once per defocus
// slab, each launch re-reading the whole volume, and updates a quad in the
// slab that holds its first corner's depth (:365-369). Here one launch
// covers all slabs of a projection: each quad looks its slab up in the
// table of slab boundaries (the reference's float recurrence
// ray += thickness) and reads that slab's filtered image.
#include <float.h>

#include "esb_bp_core.cuh"

namespace esb {

namespace {

using namespace bpcore;

template <int VT>
__global__ void __launch_bounds__(128) k_bp_fast(KConst k, BpGeom g, void* __restrict__ vol,
                                                 const float* __restrict__ imgs, size_t img_stride, SlabTable slabs,
                                                 int pw, int ph, size_t pitchE, float lambda, int os, float inv,
                                                 float distMin, float distMax, int linear, int transposed,
                                                 const float* __restrict__ ups, size_t up_stride) {
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int z = (int)blockIdx.z;
  const int ny = (int)k.dim.y, nz = (int)k.dim.z;
  if (q >= k.dimXQuarter || y >= ny || z >= nz) return;
  const int x = 4 * q;
  float depth;
  int pbx, pby, pbz, pbw;
  macro_footprint(k, x, y, z, pw, ph, depth, pbx, pby, pbz, pbw);
  const float* img = imgs;
  const float* up = ups;
  if (slabs.count > 0) {  // fused CTF slabs
    if (!(depth >= slabs.bound[0] && depth < slabs.bound[slabs.count])) return;
    int s = 0;
    while (s + 1 < slabs.count && depth >= slabs.bound[s + 1]) ++s;
    img = imgs + (size_t)s * img_stride;
    if (up) up += (size_t)s * up_stride;
  } else if (!(depth >= distMin && depth < distMax)) {
    return;
  }
  const long base = ((long)z * ny + y) * (long)k.dim.x + x;
  float acc[4], dacc[4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
    voxel_sums(k, g, img, pw, ph, pitchE, os, inv, linear != 0, transposed != 0, x + i, y, z, pbx, pby, pbz, pbw,
               acc[i], dacc[i], up, ph * os);
  if (VT == ESB_VOXEL_F32 && (((uintptr_t)((float*)vol + base)) & 15) == 0) {
    float4 v = *((float4*)((float*)vol + base));
    if (dacc[0] > 0.f) v.x += lambda * acc[0] / dacc[0];
    if (dacc[1] > 0.f) v.y += lambda * acc[1] / dacc[1];
    if (dacc[2] > 0.f) v.z += lambda * acc[2] / dacc[2];
    if (dacc[3] > 0.f) v.w += lambda * acc[3] / dacc[3];
    *((float4*)((float*)vol + base)) = v;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (dacc[i] > 0.f) Voxel<VT>::store(vol, base + i, Voxel<VT>::loadrw(vol, base + i) + lambda * acc[i] / dacc[i]);
    }
  }
}

// Geometry of k_bp_axis: single-axis tilt (n.y = 0), power-of-two
// oversampling, no anisotropy, pre-sampled images.
struct AxisGeom {
  float3 U, V;     // detector coordinate of a world point: u = U.p + U0, v = V.p + V0
  float U0, V0;
  float hu, hv;    // half shadow extents in pixels (as BpGeom)
  float wu, wv;    // in-plane offset of a sample perpendicular to n in x-z, per pixel of u and v
  float yu, yv;    // its y component per pixel of u and v
  float hby;       // half voxel size in y
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

// k_bp_fast for single-axis tilt series on pre-sampled images. With n.y = 0
// the chord of a sample's ray through a voxel depends only on the ray's
// offset w from the voxel centre perpendicular to n in the x-z plane (a
// trapezoid: the plateau min(2 hx / |n.x|, 2 hz / |n.z|), falling linearly to
// 0 at |w| = hx |n.z| + hz |n.x| with slope 1 / (|n.x| |n.z|)), cut to 0 when
// the offset's y component leaves the voxel. Samples are the sub-pixel grid
// points (m + 0.5) / os inside the voxel's shadow and inside the quad's
// macro-cell rectangle [pbx, pby) x [pbz, pbw) (macro_rect).
template <int VT>
__global__ void __launch_bounds__(128) k_bp_axis(KConst k, AxisGeom g, void* __restrict__ vol, SlabTable slabs,
                                                 int pw, int ph, float lambda, int os, float inv, float distMin,
                                                 float distMax, const float* __restrict__ ups, size_t up_stride) {
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int z = (int)blockIdx.z;
  const int ny = (int)k.dim.y, nz = (int)k.dim.z;
  if (q >= k.dimXQuarter || y >= ny || z >= nz) return;
  const int x = 4 * q;
  const float depth = macro_depth(k, x, y, z);
  const float* up = ups;
  if (slabs.count > 0) {
    if (!(depth >= slabs.bound[0] && depth < slabs.bound[slabs.count])) return;
    int s = 0;
    while (s + 1 < slabs.count && depth >= slabs.bound[s + 1]) ++s;
    up += (size_t)s * up_stride;
  } else if (!(depth >= distMin && depth < distMax)) {
    return;
  }
  int pbx, pby, pbz, pbw;
  if (g.clips) {
    float d;
    macro_footprint(k, x, y, z, pw, ph, d, pbx, pby, pbz, pbw);
  } else {
    macro_rect(g, x, y, z, pw, ph, pbx, pby, pbz, pbw);
  }
  const int upH = ph * os;
  const float fos = (float)os;
  const int mu_min = pbx * os, mu_max = pby * os - 1, mv_min = pbz * os, mv_max = pbw * os - 1;
  const float cy = k.bbMin.y + ((float)y + 0.5f) * k.vs.y, cz = k.bbMin.z + ((float)z + 0.5f) * k.vs.z;
  const float uyz = g.U.y * cy + g.U.z * cz + g.U0, vyz = g.V.y * cy + g.V.z * cz + g.V0;
  const float dwv = inv * g.wv, dyv = inv * g.yv;
  const long base = ((long)z * ny + y) * (long)k.dim.x + x;
  float res[4], has[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float cx = k.bbMin.x + ((float)(x + i) + 0.5f) * k.vs.x;
    const float uc = g.U.x * cx + uyz, vc = g.V.x * cx + vyz;
    const int mu0 = max((int)ceilf((uc - g.hu) * fos - 0.5f), mu_min);
    const int mu1 = min((int)floorf((uc + g.hu) * fos - 0.5f), mu_max);
    const int mv0 = max((int)ceilf((vc - g.hv) * fos - 0.5f), mv_min);
    const int mv1 = min((int)floorf((vc + g.hv) * fos - 0.5f), mv_max);
    const float dv0 = ((float)mv0 + 0.5f) * inv - vc;
    float a = 0.f, da = 0.f;
    // a voxel's shadow holds 2-3 sub-pixel samples per axis at OS 2: the
    // first rows and samples are unrolled (predicated), any further ones loop
    const int rows = mu1 - mu0 + 1;
    auto row = [&](int mu) {
      const float du = ((float)mu + 0.5f) * inv - uc;
      float w = du * g.wu + dv0 * g.wv, dy = du * g.yu + dv0 * g.yv;
      const float* p = up + (size_t)mu * upH + mv0;
      const int cnt = mv1 - mv0 + 1;
      auto body = [&](int j) {
        const float ww = fmaf((float)j, dwv, w), yy = fmaf((float)j, dyv, dy);
        float L = fminf(g.L0, fmaxf(0.f, fmaf(-fabsf(ww), g.K, g.w1K)));
        L = fabsf(yy) <= g.hby ? L : 0.f;
        a = fmaf(__ldg(p + j), L, a);
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
    res[i] = a;
    has[i] = da;
  }
  if (VT == ESB_VOXEL_F32 && (((uintptr_t)((float*)vol + base)) & 15) == 0) {
    float4 v = *((float4*)((float*)vol + base));
    if (has[0] > 0.f) v.x += __fdividef(lambda * res[0], has[0]);
    if (has[1] > 0.f) v.y += __fdividef(lambda * res[1], has[1]);
    if (has[2] > 0.f) v.z += __fdividef(lambda * res[2], has[2]);
    if (has[3] > 0.f) v.w += __fdividef(lambda * res[3], has[3]);
    *((float4*)((float*)vol + base)) = v;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (has[i] > 0.f) Voxel<VT>::store(vol, base + i, Voxel<VT>::loadrw(vol, base + i) + __fdividef(lambda * res[i], has[i]));
    }
  }
}

AxisGeom make_axis_geom(const KConst& k, const BpGeom& b, int os) {
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

// The slab images (transposed, [x][y], stride img_stride) sampled at every
// sub-pixel grid point: up[s][mu][mv] = image s at ((mu + 0.5) / os,
// (mv + 0.5) / os), clamp addressing, nearest or bilinear as the
// back-projection reads it.
__global__ void __launch_bounds__(256) k_upsample(const float* __restrict__ imgs, size_t img_stride, int pw, int ph,
                                                  int os, float inv, int linear, float* __restrict__ up,
                                                  size_t up_stride) {
  const int mv = blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  const int s = blockIdx.z;
  const int upH = ph * os;
  if (mv >= upH) return;
  const float px = ((float)mu + 0.5f) * inv, py = ((float)mv + 0.5f) * inv;
  up[(size_t)s * up_stride + (size_t)mu * upH + mv] =
      sample_image(imgs + (size_t)s * img_stride, pw, ph, (size_t)pw, px, py, linear != 0, true);
}

}  // namespace

cudaError_t launch_bp_fast_slabs(const KConst& k, void* vol, int vt, const float* imgs, size_t img_stride,
                                 const SlabTable& slabs, int pw, int ph, size_t pitchE, float lambda, int os,
                                 float distMin, float distMax, int linear, cudaStream_t st, int transposed,
                                 const float* ups, size_t up_stride) {
  const int nq = k.dimXQuarter, ny = (int)k.dim.y, nz = (int)k.dim.z;
  if (nq <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  const BpGeom g = make_geom(k, os);
  const float inv = 1.0f / (float)os;
  dim3 blk(32, 4, 1), grd((nq + 31) / 32, (ny + 3) / 4, nz);
  if (ups && g.exact_grid && g.aniso_identity && fabsf(k.n.y) <= 1e-6f) {
    const AxisGeom a = make_axis_geom(k, g, os);
    switch (vt) {
      case ESB_VOXEL_F32: k_bp_axis<ESB_VOXEL_F32><<<grd, blk, 0, st>>>(k, a, vol, slabs, pw, ph, lambda, os, inv, distMin, distMax, ups, up_stride); break;
      case ESB_VOXEL_F16: k_bp_axis<ESB_VOXEL_F16><<<grd, blk, 0, st>>>(k, a, vol, slabs, pw, ph, lambda, os, inv, distMin, distMax, ups, up_stride); break;
      default: k_bp_axis<ESB_VOXEL_BF16><<<grd, blk, 0, st>>>(k, a, vol, slabs, pw, ph, lambda, os, inv, distMin, distMax, ups, up_stride); break;
    }
    ESB_COUNT_LAUNCH();
    return cudaGetLastError();
  }
  switch (vt) {
    case ESB_VOXEL_F32: k_bp_fast<ESB_VOXEL_F32><<<grd, blk, 0, st>>>(k, g, vol, imgs, img_stride, slabs, pw, ph, pitchE, lambda, os, inv, distMin, distMax, linear, transposed, ups, up_stride); ESB_COUNT_LAUNCH(); break;
    case ESB_VOXEL_F16: k_bp_fast<ESB_VOXEL_F16><<<grd, blk, 0, st>>>(k, g, vol, imgs, img_stride, slabs, pw, ph, pitchE, lambda, os, inv, distMin, distMax, linear, transposed, ups, up_stride); ESB_COUNT_LAUNCH(); break;
    default: k_bp_fast<ESB_VOXEL_BF16><<<grd, blk, 0, st>>>(k, g, vol, imgs, img_stride, slabs, pw, ph, pitchE, lambda, os, inv, distMin, distMax, linear, transposed, ups, up_stride); ESB_COUNT_LAUNCH(); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_bp_fast(const KConst& k, void* vol, int vt, const float* img, int pw, int ph, size_t pitchE,
                           float lambda, int os, float distMin, float distMax, int linear, cudaStream_t st) {
  SlabTable none;
  none.count = 0;
  return launch_bp_fast_slabs(k, vol, vt, img, 0, none, pw, ph, pitchE, lambda, os, distMin, distMax, linear, st, 0,
                              nullptr, 0);
}

// Pre-sampled slab images for k_bp_fast (transposed input images, up_stride
// floats per output image of (pw * os) x (ph * os)).
cudaError_t launch_upsample(const float* imgs, size_t img_stride, int count, int pw, int ph, int os, int linear,
                            float* up, size_t up_stride, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  dim3 blk(256), grd((ph * os + 255) / 256, pw * os, count);
  k_upsample<<<grd, blk, 0, st>>>(imgs, img_stride, pw, ph, os, 1.0f / (float)os, linear, up, up_stride);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

// Whether k_bp_fast may read pre-sampled images: the sub-pixel recurrence is
// exact (power-of-two oversampling) and samples are read at (px, py) (no
// magnification anisotropy).
bool bp_can_upsample(const KConst& k, int os) {
  const BpGeom g = make_geom(k, os);
  return g.exact_grid && g.aniso_identity;
}

}  // namespace esb
