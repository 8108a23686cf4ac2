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
                                                 const float2* __restrict__ ups, size_t up_stride) {
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
  const float2* up = ups;
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

// k_bp_fast for single-axis tilt series (axis_sums): on pre-sampled slab
// images (UP: one load per sample) or reading the slab images directly.
template <int VT, bool UP>
__global__ void __launch_bounds__(128) k_bp_axis(KConst k, AxisGeom g, void* __restrict__ vol,
                                                 const float* __restrict__ imgs, size_t img_stride, SlabTable slabs,
                                                 int pw, int ph, size_t pitchE, float lambda, int os, float inv,
                                                 float distMin, float distMax, int linear, int transposed,
                                                 const float2* __restrict__ ups, size_t up_stride, int z0) {
  // plane z0 + blockIdx.z of the geometry, stored at plane blockIdx.z of vol
  // (z0 = 0 but for the autotuner's trial launches on a scratch slab)
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int zl = (int)blockIdx.z;
  const int z = z0 + zl;
  const int ny = (int)k.dim.y, nz = (int)k.dim.z;
  if (q >= k.dimXQuarter || y >= ny || z >= nz) return;
  const int x = 4 * q;
  const float depth = macro_depth(k, x, y, z);
  const float* img = imgs;
  const float2* up = ups;
  if (slabs.count > 0) {
    if (!(depth >= slabs.bound[0] && depth < slabs.bound[slabs.count])) return;
    int s = 0;
    while (s + 1 < slabs.count && depth >= slabs.bound[s + 1]) ++s;
    if (UP)
      up += (size_t)s * up_stride;
    else
      img += (size_t)s * img_stride;
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
  const float cy = k.bbMin.y + ((float)y + 0.5f) * k.vs.y, cz = k.bbMin.z + ((float)z + 0.5f) * k.vs.z;
  const float uyz = g.U.y * cy + g.U.z * cz + g.U0, vyz = g.V.y * cy + g.V.z * cz + g.V0;
  const float dwv = inv * g.wv;
  const bool lin = linear != 0, tr = transposed != 0;
  const bool interior = !lin || (pbx >= 1 && pbz >= 1);
  const size_t sx = tr ? (size_t)ph : 1, sy = tr ? 1 : pitchE;
  const long base = ((long)zl * ny + y) * (long)k.dim.x + x;
  float res[4], has[4];
  if (UP) {
    auto read = [&](int mu, int mv) -> float2 { return __ldg(up + (size_t)mu * upH + mv); };
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float cx = k.bbMin.x + ((float)(x + i) + 0.5f) * k.vs.x;
      const float uc = g.U.x * cx + uyz, vc = g.V.x * cx + vyz;
      axis_sums_rows(g, uc, vc, fos, inv, dwv, y, pbx * os, pby * os - 1, pbz * os, pbw * os - 1, read, res[i],
                     has[i]);
    }
  } else {
    auto read = [&](int mu, int mv) -> float {
      const float px = ((float)mu + 0.5f) * inv, py = ((float)mv + 0.5f) * inv;
      return interior ? sample_interior(img, sx, sy, px, py, lin) : sample_image(img, pw, ph, pitchE, px, py, lin, tr);
    };
    const bool patch = os == 2 && lin && interior;
    const float cx0 = k.bbMin.x + ((float)x + 0.5f) * k.vs.x;
    const RowAnchor anchor(g, y, g.U.x * cx0 + uyz, g.V.x * cx0 + vyz, fos);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float cx = k.bbMin.x + ((float)(x + i) + 0.5f) * k.vs.x;
      const float uc = g.U.x * cx + uyz, vc = g.V.x * cx + vyz;
      if (!(patch && axis_sums_os2(g, uc, vc, dwv, anchor, pbx * 2, pby * 2 - 1, pbz * 2, pbw * 2 - 1, img, sx, sy,
                                   pw, ph, res[i], has[i])))
        axis_sums(g, uc, vc, fos, inv, dwv, anchor, pbx * os, pby * os - 1, pbz * os, pbw * os - 1, read, res[i],
                  has[i]);
    }
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
      if (has[i] > 0.f)
        Voxel<VT>::store(vol, base + i, Voxel<VT>::loadrw(vol, base + i) + __fdividef(lambda * res[i], has[i]));
    }
  }
}

// One ordered subset back-projected in one pass over the volume (the
// SIRTCount back-projections of EmSart.cpp:649-673): each quad is read once,
// the updates of the subset's projections are added to it in the order of
// the subset, as the per-projection launches add them, and it is stored once.
// Every projection contributes exactly what k_bp_axis<VT, true> adds for it
// (pre-sampled slab images, CTF slab chosen by the first corner's depth).
// FP32 volumes: the result is bit for bit that of the per-projection
// launches. FP16 / BF16 volumes: the sum is rounded to the storage type once
// per subset instead of once per projection.
struct BpSetItem {
  KConst k;
  AxisGeom a;
  const float2* up;  // pre-sampled slab images of this projection
  int nslab;         // 0: no CTF slabs
  float bound[ESB_BP_SET_MAX_SLABS + 1];
};
struct BpSet {
  int count;
  size_t up_stride;
  BpSetItem p[ESB_BP_SET_MAX];
};

template <int VT>
__global__ void __launch_bounds__(128) k_bp_axis_set(const __grid_constant__ BpSet set, void* __restrict__ vol,
                                                     int pw, int ph, float lambda, int os, float inv) {
  const int q = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int z = (int)blockIdx.z;
  const KConst& k0 = set.p[0].k;
  const int ny = (int)k0.dim.y, nz = (int)k0.dim.z;
  if (q >= k0.dimXQuarter || y >= ny || z >= nz) return;
  const int x = 4 * q;
  const long base = ((long)z * ny + y) * (long)k0.dim.x + x;
  const bool vec = VT == ESB_VOXEL_F32 && (((uintptr_t)((float*)vol + base)) & 15) == 0;
  float v[4];
  if (vec) {
    const float4 t = *((const float4*)((const float*)vol + base));
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) v[i] = Voxel<VT>::loadrw(vol, base + i);
  }
  const int upH = ph * os;
  const float fos = (float)os;
  bool touched = false;
#pragma unroll 1
  for (int j = 0; j < set.count; ++j) {
    const BpSetItem& it = set.p[j];
    const KConst& k = it.k;
    const AxisGeom& g = it.a;
    const float depth = macro_depth(k, x, y, z);
    const float2* up = it.up;
    if (it.nslab > 0) {
      if (!(depth >= it.bound[0] && depth < it.bound[it.nslab])) continue;
      int s = 0;
      while (s + 1 < it.nslab && depth >= it.bound[s + 1]) ++s;
      up += (size_t)s * set.up_stride;
    }
    int pbx, pby, pbz, pbw;
    if (g.clips) {
      float d;
      macro_footprint(k, x, y, z, pw, ph, d, pbx, pby, pbz, pbw);
    } else {
      macro_rect(g, x, y, z, pw, ph, pbx, pby, pbz, pbw);
    }
    const float cy = k.bbMin.y + ((float)y + 0.5f) * k.vs.y, cz = k.bbMin.z + ((float)z + 0.5f) * k.vs.z;
    const float uyz = g.U.y * cy + g.U.z * cz + g.U0, vyz = g.V.y * cy + g.V.z * cz + g.V0;
    const float dwv = inv * g.wv;
    auto read = [&](int mu, int mv) -> float2 { return __ldg(up + (size_t)mu * upH + mv); };
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float cx = k.bbMin.x + ((float)(x + i) + 0.5f) * k.vs.x;
      const float uc = g.U.x * cx + uyz, vc = g.V.x * cx + vyz;
      float res, has;
      axis_sums_rows(g, uc, vc, fos, inv, dwv, y, pbx * os, pby * os - 1, pbz * os, pbw * os - 1, read, res, has);
      if (has > 0.f) {
        v[i] += __fdividef(lambda * res, has);
        touched = true;
      }
    }
  }
  if (!touched) return;
  if (vec) {
    *((float4*)((float*)vol + base)) = make_float4(v[0], v[1], v[2], v[3]);
  } else {
#pragma unroll
    for (int i = 0; i < 4; ++i) Voxel<VT>::store(vol, base + i, v[i]);
  }
}

// The slab images (transposed, [x][y], stride img_stride) sampled at every
// sub-pixel grid point, with the voxel row of the grid point's ray:
// up[s][mu][mv] = (image s at ((mu + 0.5) / os, (mv + 0.5) / os), row as int
// bits), clamp addressing, nearest or bilinear as the back-projection reads
// it (sample_row; meaningful for single-axis projections, which read it).
// The row depends on the grid point and the projection only: it is formed
// once per grid point and stored with the point's value in every slab image.
__global__ void __launch_bounds__(256) k_upsample(const float* __restrict__ imgs, size_t img_stride, int count, int pw,
                                                  int ph, int os, float inv, int linear, RowGeom rg,
                                                  float2* __restrict__ up, size_t up_stride) {
  const int mv = blockIdx.x * blockDim.x + threadIdx.x;
  const int mu = blockIdx.y;
  const int upH = ph * os;
  if (mv >= upH) return;
  const float px = ((float)mu + 0.5f) * inv, py = ((float)mv + 0.5f) * inv;
  const float row = __int_as_float(sample_row(rg, mu, mv));
  float2* out = up + (size_t)mu * upH + mv;
#pragma unroll 1
  for (int s = 0; s < count; ++s)
    out[(size_t)s * up_stride] =
        make_float2(sample_image(imgs + (size_t)s * img_stride, pw, ph, (size_t)pw, px, py, linear != 0, true), row);
}

}  // namespace

cudaError_t launch_bp_fast_slabs(const KConst& k, void* vol, int vt, const float* imgs, size_t img_stride,
                                 const SlabTable& slabs, int pw, int ph, size_t pitchE, float lambda, int os,
                                 float distMin, float distMax, int linear, cudaStream_t st, int transposed,
                                 const float2* ups, size_t up_stride, const BpShape* shape) {
  const int nq = k.dimXQuarter, ny = (int)k.dim.y, nz = (int)k.dim.z;
  if (nq <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  const BpGeom g = make_geom(k, os);
  const float inv = 1.0f / (float)os;
  dim3 blk(32, 4, 1), grd((nq + 31) / 32, (ny + 3) / 4, nz);
  if (axis_eligible(k, g)) {
    const AxisGeom a = make_axis_geom(k, g, os);
    int z0 = 0;
    if (shape) {  // block of bx quads x by rows (bx * by <= 128); planes [z0, z0 + nz)
      blk = dim3(shape->bx, shape->by, 1);
      z0 = shape->z0;
      grd = dim3((nq + shape->bx - 1) / shape->bx, (ny + shape->by - 1) / shape->by,
                 shape->nz > 0 ? shape->nz : nz - z0);
    }
#define ESB_AXIS(VT, UP)                                                                                          \
  k_bp_axis<VT, UP><<<grd, blk, 0, st>>>(k, a, vol, imgs, img_stride, slabs, pw, ph, pitchE, lambda, os, inv, distMin, \
                                         distMax, linear, transposed, ups, up_stride, z0)
    if (ups) {
      if (vt == ESB_VOXEL_F32) ESB_AXIS(ESB_VOXEL_F32, true);
      else if (vt == ESB_VOXEL_F16) ESB_AXIS(ESB_VOXEL_F16, true);
      else ESB_AXIS(ESB_VOXEL_BF16, true);
    } else {
      if (vt == ESB_VOXEL_F32) ESB_AXIS(ESB_VOXEL_F32, false);
      else if (vt == ESB_VOXEL_F16) ESB_AXIS(ESB_VOXEL_F16, false);
      else ESB_AXIS(ESB_VOXEL_BF16, false);
    }
#undef ESB_AXIS
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
                              nullptr, 0, nullptr);
}

// Whether projection k can join a subset launch (launch_bp_axis_set): the
// single-axis kernel on pre-sampled images, at most ESB_BP_SET_MAX_SLABS
// CTF slabs.
bool bp_set_eligible(const KConst& k, int os, int nslab) {
  const BpGeom g = make_geom(k, os);
  return axis_eligible(k, g) && g.exact_grid && g.aniso_identity && nslab <= ESB_BP_SET_MAX_SLABS;
}

// The back-projections of `count` (<= ESB_BP_SET_MAX) projections of one
// ordered subset in one launch (k_bp_axis_set): ks[j] the constants of
// projection j, ups[j] its pre-sampled slab images (up_stride apart),
// slabs[j] its CTF slabs (count 0: none); all bp_set_eligible, all on the
// same volume geometry. The block shape is shape's (bx, by); its planes are
// the whole volume.
cudaError_t launch_bp_axis_set(const KConst* ks, const float2* const* ups, const SlabTable* slabs, int count,
                               size_t up_stride, void* vol, int vt, int pw, int ph, float lambda, int os,
                               const BpShape* shape, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  if (count > ESB_BP_SET_MAX) return cudaErrorInvalidValue;
  const KConst& k0 = ks[0];
  const int nq = k0.dimXQuarter, ny = (int)k0.dim.y, nz = (int)k0.dim.z;
  if (nq <= 0 || ny <= 0 || nz <= 0) return cudaSuccess;
  BpSet set;  // the kernel parameter (copied into the launch)
  set.count = count;
  set.up_stride = up_stride;
  for (int j = 0; j < count; ++j) {
    const BpGeom g = make_geom(ks[j], os);
    if (!(axis_eligible(ks[j], g) && g.exact_grid && g.aniso_identity) || slabs[j].count > ESB_BP_SET_MAX_SLABS ||
        !ups[j])
      return cudaErrorInvalidValue;
    BpSetItem& it = set.p[j];
    it.k = ks[j];
    it.a = make_axis_geom(ks[j], g, os);
    it.up = ups[j];
    it.nslab = slabs[j].count;
    for (int b = 0; b <= it.nslab; ++b) it.bound[b] = slabs[j].bound[b];
  }
  const int bx = shape ? shape->bx : 32, by = shape ? shape->by : 4;
  const dim3 blk(bx, by, 1), grd((nq + bx - 1) / bx, (ny + by - 1) / by, nz);
  const float inv = 1.0f / (float)os;
  if (vt == ESB_VOXEL_F32) k_bp_axis_set<ESB_VOXEL_F32><<<grd, blk, 0, st>>>(set, vol, pw, ph, lambda, os, inv);
  else if (vt == ESB_VOXEL_F16) k_bp_axis_set<ESB_VOXEL_F16><<<grd, blk, 0, st>>>(set, vol, pw, ph, lambda, os, inv);
  else k_bp_axis_set<ESB_VOXEL_BF16><<<grd, blk, 0, st>>>(set, vol, pw, ph, lambda, os, inv);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

// Pre-sampled slab images for k_bp_fast / k_bp_axis (transposed input
// images, up_stride (value, row) pairs per output image of (pw * os) x
// (ph * os)); k gives the geometry of the rows.
cudaError_t launch_upsample(const KConst& k, const float* imgs, size_t img_stride, int count, int pw, int ph, int os,
                            int linear, float2* up, size_t up_stride, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  dim3 blk(256), grd((ph * os + 255) / 256, pw * os, 1);
  k_upsample<<<grd, blk, 0, st>>>(imgs, img_stride, count, pw, ph, os, 1.0f / (float)os, linear, make_row_geom(k, os),
                                  up, up_stride);
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

// Whether launch_bp_fast_slabs takes the single-axis kernel (whose launch
// shape BpShape sets).
bool bp_uses_axis(const KConst& k, int os) { return axis_eligible(k, make_geom(k, os)); }

}  // namespace esb
