// CPU oracle for the EmSART reconstruction hot path.
//
// TEST INFRASTRUCTURE ONLY. Nothing in the product library links, loads or
// calls this file; only the tests, the smoke check and the CPU-baseline leg
// of the benchmark do, and there only as what results are compared with (or
// as the timed CPU baseline).  It restates, statement by statement, the device code and the
// host geometry of uermel/Artiatomi's EmSART so that the CUDA kernels of this
// repository can be compared against the reference's algorithm on the same
// inputs.  Every function cites the reference file and lines it follows
// (paths relative to the Artiatomi source tree).
//
// Precision modes (template parameter R):
//   float  - "FP32": every arithmetic step in IEEE float in the reference's
//            order (compile with -ffp-contract=off so no FMA is formed).
//   double - "FP64": all arithmetic in double, except the forward-projection
//            ray parameter t, which the reference advances in float
//            (ForwardProjectionRayMarcher_TL.cu:141); that float step is
//            part of the reference's defined output (its effective step is
//            not 0.15 but 0.15 rounded to the float grid of t ~ 1e4), so the
//            FP64 oracle keeps it.  Pass exact_step=1 to drop it.
//
// Texture emulation: tex3D/tex2D with cudaFilterModeLinear use texel centres
// at +0.5, clamp addressing and a weight stored with 8 fractional bits
// (published description of linear filtering).  The 8-bit weight is optional
// (q9 flag); by default the weight is the full-precision fraction.

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------- threading
template <class F>
void parallel_for(int n, int nthreads, F f) {
  if (nthreads <= 1 || n <= 1) {
    for (int i = 0; i < n; ++i) f(i);
    return;
  }
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  int nt = std::min(nthreads, n);
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        int i = next.fetch_add(1);
        if (i >= n) break;
        f(i);
      }
    });
  for (auto& th : pool) th.join();
}

// ------------------------------------------------------------ half floats
// IEEE binary16 conversions written from the format definition
// (round-to-nearest-even on the way down).
float half_to_float(uint16_t h) {
  uint32_t sign = (h >> 15) & 1u, ex = (h >> 10) & 0x1fu, man = h & 0x3ffu;
  float v;
  if (ex == 0)
    v = std::ldexp((float)man, -24);
  else if (ex == 31)
    v = man ? NAN : INFINITY;
  else
    v = std::ldexp((float)(man | 0x400u), (int)ex - 25);
  return sign ? -v : v;
}

uint16_t float_to_half_rn(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  uint32_t sign = (x >> 16) & 0x8000u;
  uint32_t ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (uint16_t)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
  if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);  // rounds to inf
  int e = (int)(ax >> 23) - 127;
  uint32_t m = (ax & 0x7fffffu) | 0x800000u;
  if (e < -24) {
    // below half of the smallest subnormal (ties handled below by shift)
    if (e < -25) return (uint16_t)sign;
  }
  int shift;
  uint32_t base;
  if (e >= -14) {  // normal half
    shift = 13;
    base = (uint32_t)(e + 15) << 10;
    m &= 0x7fffffu;
  } else {  // subnormal half
    shift = 13 + (-14 - e);
    base = 0;
  }
  uint32_t q = m >> shift;
  uint32_t rem = m & ((1u << shift) - 1u);
  uint32_t half = 1u << (shift - 1);
  if (rem > half || (rem == half && (q & 1u))) q += 1;
  return (uint16_t)(sign | (base + q));  // carries into the exponent correctly
}

// bfloat16 with round-to-nearest-even
float bf16_to_float(uint16_t h) {
  uint32_t x = (uint32_t)h << 16;
  float f;
  std::memcpy(&f, &x, 4);
  return f;
}
uint16_t float_to_bf16_rn(float f) {
  uint32_t x;
  std::memcpy(&x, &f, 4);
  if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);
  uint32_t lsb = (x >> 16) & 1u;
  x += 0x7fffu + lsb;
  return (uint16_t)(x >> 16);
}

}  // namespace

extern "C" {

// Geometry handed to the projector/back-projector: the values the reference
// writes into __constant__ memory (DeviceVariables.cuh:13-34) through
// SetConstantValues (Kernels.cpp:949-1101).
struct OrcGeom {
  float det[3];      // c_detektor   (Projection::GetPosition)
  float u[3];        // c_uPitch     (Projection::GetPixelUPitch)
  float v[3];        // c_vPitch     (Projection::GetPixelVPitch)
  float n[3];        // c_projNorm   (Projection::GetNormalVector)
  float detMat[16];  // c_DetectorMatrix (Projection::GetDetectorMatrix, os=1)
  float bbMin[3];    // c_bBoxMin    (sub-volume bbox min)
  float bbMax[3];    // c_bBoxMax
  float bbRcp[3];    // c_volumeBBoxRcp
  float dim[3];      // c_volumeDim  (sub-volume dimension)
  float vs[3];       // c_voxelSize
  float zShift;      // c_zShiftForPartialVolume (0 in FP, Kernels.cpp:987)
  int dimXQuarter;   // c_volumeDim_x_quarter (full dim.x / 4, Kernels.cpp:1093)
  float aniso[9];    // c_magAniso    row-major 3x3
  float anisoInv[9]; // c_magAnisoInv row-major 3x3
};

}  // extern "C"

namespace {

// Volume storage: 0 = float32, 1 = float16, 2 = bfloat16 ([z][y][x], x fastest)
struct VolView {
  const void* data;
  int nx, ny, nz;
  int dtype;
  inline float at(long i) const {
    if (dtype == 0) return ((const float*)data)[i];
    if (dtype == 1) return half_to_float(((const uint16_t*)data)[i]);
    return bf16_to_float(((const uint16_t*)data)[i]);
  }
};

template <class R>
inline R quant8(R a) {  // 1.8 fixed-point weight of the texture unit
  return std::floor(a * R(256) + R(0.5)) / R(256);
}

// tex3D<float>(tex, x, y, z): linear filtering, unnormalised coordinates,
// clamp addressing on all axes (EmSart.cpp:421).
template <class R>
R tex3d(const VolView& v, R x, R y, R z, bool q9) {
  R xb = x - R(0.5), yb = y - R(0.5), zb = z - R(0.5);
  R fx = std::floor(xb), fy = std::floor(yb), fz = std::floor(zb);
  R a = xb - fx, b = yb - fy, c = zb - fz;
  if (q9) { a = quant8(a); b = quant8(b); c = quant8(c); }
  auto clampi = [](double f, int n) -> long {
    if (!(f > 0)) return 0;  // also NaN -> 0
    if (f > n - 1) return n - 1;
    return (long)f;
  };
  long x0 = clampi((double)fx, v.nx), x1 = clampi((double)fx + 1, v.nx);
  long y0 = clampi((double)fy, v.ny), y1 = clampi((double)fy + 1, v.ny);
  long z0 = clampi((double)fz, v.nz), z1 = clampi((double)fz + 1, v.nz);
  long sy = v.nx, sz = (long)v.nx * v.ny;
  R t000 = v.at(z0 * sz + y0 * sy + x0), t100 = v.at(z0 * sz + y0 * sy + x1);
  R t010 = v.at(z0 * sz + y1 * sy + x0), t110 = v.at(z0 * sz + y1 * sy + x1);
  R t001 = v.at(z1 * sz + y0 * sy + x0), t101 = v.at(z1 * sz + y0 * sy + x1);
  R t011 = v.at(z1 * sz + y1 * sy + x0), t111 = v.at(z1 * sz + y1 * sy + x1);
  R ia = R(1) - a, ib = R(1) - b, ic = R(1) - c;
  return ic * (ib * (ia * t000 + a * t100) + b * (ia * t010 + a * t110)) +
         c * (ib * (ia * t001 + a * t101) + b * (ia * t011 + a * t111));
}

// tex2D(tex, x, y) on the projection image, clamp addressing; POINT filtering
// when CTF is off, LINEAR when on (Reconstructor.cpp:318-327).
template <class R>
R tex2d(const float* img, int w, int h, size_t pitchElems, R x, R y, bool linear, bool q9) {
  auto clampi = [](double f, int n) -> long {
    if (!(f > 0)) return 0;
    if (f > n - 1) return n - 1;
    return (long)f;
  };
  if (!linear) {
    long ix = clampi(std::floor((double)x), w), iy = clampi(std::floor((double)y), h);
    return R(img[iy * pitchElems + ix]);
  }
  R xb = x - R(0.5), yb = y - R(0.5);
  R fx = std::floor(xb), fy = std::floor(yb);
  R a = xb - fx, b = yb - fy;
  if (q9) { a = quant8(a); b = quant8(b); }
  long x0 = clampi((double)fx, w), x1 = clampi((double)fx + 1, w);
  long y0 = clampi((double)fy, h), y1 = clampi((double)fy + 1, h);
  R t00 = img[y0 * pitchElems + x0], t10 = img[y0 * pitchElems + x1];
  R t01 = img[y1 * pitchElems + x0], t11 = img[y1 * pitchElems + x1];
  return (R(1) - b) * ((R(1) - a) * t00 + a * t10) + b * ((R(1) - a) * t01 + a * t11);
}

template <class R>
inline R fmn(R a, R b) { return std::fmin(a, b); }  // CUDA fminf: NaN-ignoring
template <class R>
inline R fmx(R a, R b) { return std::fmax(a, b); }

// Slab intersection of the ray src + t*dir with the box [lo, hi]
// (ForwardProjectionRayMarcher_TL.cu:92-107).
template <class R>
inline void box_hit(const R src[3], const R dir[3], const R lo[3], const R hi[3], R& tin, R& tout) {
  R tmin[3], tmax[3];
  for (int k = 0; k < 3; ++k) {
    R te = (lo[k] - src[k]) / dir[k];
    R tx = (hi[k] - src[k]) / dir[k];
    tmin[k] = fmn(te, tx);
    tmax[k] = fmx(te, tx);
  }
  tin = fmx(fmx(tmin[0], tmin[1]), tmin[2]);
  tout = fmn(fmn(tmax[0], tmax[1]), tmax[2]);
}

// Ray start for sub-pixel (px, py) of the detector with mag anisotropy:
// MatrixVector3Mul(c_magAniso, ...) then c_detektor + xA*u + yA*v
// (ForwardProjectionRayMarcher_TL.cu:84-90, DeviceVariables.cuh:42-47).
template <class R>
inline void ray_source(const OrcGeom& g, R px, R py, R src[3]) {
  R xA = R(g.aniso[0]) * px + R(g.aniso[1]) * py + R(g.aniso[2]) * R(1);
  R yA = R(g.aniso[3]) * px + R(g.aniso[4]) * py + R(g.aniso[5]) * R(1);
  for (int k = 0; k < 3; ++k) {
    R s = R(g.det[k]);
    s = s + xA * R(g.u[k]);
    s = s + yA * R(g.v[k]);
    src[k] = s;
  }
}

// Line integral of one pixel: kernel `march`
// (ForwardProjectionRayMarcher_TL.cu:58-160).  proj += Σ/4, dist = mean chord.
template <class R>
void march_pixel(const OrcGeom& g, const VolView& vol, int x, int y, bool q9, bool exact_step,
                 float* proj, float* dist) {
  R lo[3], hi[3], nrm[3];
  for (int k = 0; k < 3; ++k) { lo[k] = g.bbMin[k]; hi[k] = g.bbMax[k]; nrm[k] = g.n[k]; }
  R temp = 0, gx = 0, gz = 0;
  const float hf = g.vs[0] * 0.15f;  // c_voxelSize.x * 0.15f (float in the reference)
  const R h = exact_step ? R(g.vs[0]) * R(0.15) : R(hf);
  for (int ox = 0; ox < 2; ++ox)
    for (int oy = 0; oy < 2; ++oy) {
      R osx = R(0.25f + 0.5f * ox), osy = R(0.25f + 0.5f * oy);
      R src[3];
      ray_source<R>(g, R(x) + osx, R(y) + osy, src);
      R tin, tout;
      box_hit<R>(src, nrm, lo, hi, tin, tout);
      if (tout - tin > R(0)) {
        gx += R(1);
        gz += tout - tin;
        // The ray parameter is a float in the reference; keep it one here.
        float tf = (float)tin;
        const float toutf = (float)tout;
        R t = exact_step ? tin : R(tf);
        R f[3];
        for (int k = 0; k < 3; ++k) f[k] = src[k] + t * nrm[k];
        while (exact_step ? (t <= tout) : (tf <= toutf)) {
          R cx = (f[0] - lo[0]) * R(g.bbRcp[0]) * R(g.dim[0]);
          R cy = (f[1] - lo[1]) * R(g.bbRcp[1]) * R(g.dim[1]);
          R cz = (f[2] - lo[2]) * R(g.bbRcp[2]) * R(g.dim[2]) - R(g.zShift);
          R s = tex3d<R>(vol, cx, cy, cz, q9);
          temp += s * R(g.vs[0]) * R(0.15f);
          if (exact_step) {
            t += h;
          } else {
            tf += hf;
            t = R(tf);
          }
          for (int k = 0; k < 3; ++k) f[k] = src[k] + t * nrm[k];
        }
      }
    }
  *proj += (float)(temp * R(0.25f));
  R d = gz / gx;
  *dist = (float)fmx(R(0), d);
}

// Slab-restricted line integral: kernel `slicer`
// (ForwardProjectionSlicer.cu:57-220).  Mirrors the reference's first sample
// taken at the un-advanced ray start (f = c_source, :126-141) unless
// fix_first_sample is set.
template <class R>
void slicer_pixel(const OrcGeom& g, const VolView& vol, int x, int y, float tminDef, float tmaxDef,
                  bool q9, bool fix_first_sample, float* proj) {
  R lo[3], hi[3], nrm[3];
  for (int k = 0; k < 3; ++k) { lo[k] = g.bbMin[k]; hi[k] = g.bbMax[k]; nrm[k] = g.n[k]; }
  R temp = 0;
  const float hf = g.vs[0] * 0.15f;
  for (int ox = 0; ox < 2; ++ox)
    for (int oy = 0; oy < 2; ++oy) {
      R osx = R(0.25f + 0.5f * ox), osy = R(0.25f + 0.5f * oy);
      R src[3];
      ray_source<R>(g, R(x) + osx, R(y) + osy, src);
      R tin, tout;
      box_hit<R>(src, nrm, lo, hi, tin, tout);
      if (tout - tin > R(0)) {
        tin = fmx(tin, R(tminDef));
        tout = fmn(tout, R(tmaxDef));
        float tf = (float)tin;
        const float toutf = (float)tout;
        R f[3];
        for (int k = 0; k < 3; ++k) f[k] = fix_first_sample ? src[k] + R(tf) * nrm[k] : src[k];
        while (tf <= toutf) {
          R cx = (f[0] - lo[0]) * R(g.bbRcp[0]) * R(g.dim[0]);
          R cy = (f[1] - lo[1]) * R(g.bbRcp[1]) * R(g.dim[1]);
          R cz = (f[2] - lo[2]) * R(g.bbRcp[2]) * R(g.dim[2]) - R(g.zShift);
          R s = tex3d<R>(vol, cx, cy, cz, q9);
          temp += s * R(g.vs[0]) * R(0.15f);
          tf += hf;
          for (int k = 0; k < 3; ++k) f[k] = src[k] + R(tf) * nrm[k];
        }
      }
    }
  *proj += (float)(temp * R(0.25f));
}

// Central-ray chord length: kernel `volTraversalLength`
// (ForwardProjectionSlicer.cu:224-288).  dist += t_out - t_in.
template <class R>
void travlen_pixel(const OrcGeom& g, int x, int y, float* dist) {
  R lo[3], hi[3], nrm[3];
  for (int k = 0; k < 3; ++k) { lo[k] = g.bbMin[k]; hi[k] = g.bbMax[k]; nrm[k] = g.n[k]; }
  R src[3];
  ray_source<R>(g, R(x) + R(0.5f), R(y) + R(0.5f), src);
  R tin, tout, val = 0;
  box_hit<R>(src, nrm, lo, hi, tin, tout);
  if (tout > tin) val = tout - tin;
  *dist += (float)val;
}

// Gaussian edge factor 1 - exp(-9 w^2), w clipped at 0 (Compare.cu:82-127).
inline float taper(float w) {
  if (w < 0) w = 0;
  return 1.0f - std::exp(-(w * w * 9.0f));
}

// One 4-voxel quad of kernel `backProjection` / `backProjectionFP16`
// (BackProjectionSquareOS.cu:263-782, 786-1291).  Returns false when the
// quad's first corner lies outside [distMin, distMax) (slab test :365-369).
//
// R is the arithmetic of the chords and sums, D that of the decisions: the
// quad's depth against the slab bounds and the macro-cell rectangle whose
// integer bounds pick the samples. R = D = float is the reference; R = D =
// double its FP64 evaluation; R = double, D = float keeps the reference's
// float decisions with exact chords (what the library's FAST kernels
// compute), to attribute differences between the two.
template <class R, class D>
void bp_quad(const OrcGeom& g, void* volData, int dtype, int qx, int y, int z, const float* img, int pw,
             int ph, size_t pitchElems, float lambda, int os, float distMin, float distMax, bool linear,
             bool q9) {
  const int nxq = g.dimXQuarter;
  (void)nxq;
  const long nx = (long)g.dim[0], ny = (long)g.dim[1];
  const long base = ((long)z * ny + y) * nx + 4L * qx;
  float vb[4];
  for (int k = 0; k < 4; ++k) {
    if (dtype == 0) vb[k] = ((float*)volData)[base + k];
    else if (dtype == 1) vb[k] = half_to_float(((uint16_t*)volData)[base + k]);
    else vb[k] = bf16_to_float(((uint16_t*)volData)[base + k]);
  }
  const int x = 4 * qx;
  const D dbbMin[3] = {D(g.bbMin[0]), D(g.bbMin[1]), D(g.bbMin[2])};
  const D dvs[3] = {D(g.vs[0]), D(g.vs[1]), D(g.vs[2])};
  const D dn[3] = {D(g.n[0]), D(g.n[1]), D(g.n[2])};
  const D ddet[3] = {D(g.det[0]), D(g.det[1]), D(g.det[2])};
  D mcMin[3] = {dbbMin[0] + D(x) * dvs[0], dbbMin[1] + D(y) * dvs[1], dbbMin[2] + D(z) * dvs[2]};
  D mcMax[3] = {dbbMin[0] + D(x + 5) * dvs[0], dbbMin[1] + D(y + 1) * dvs[1], dbbMin[2] + D(z + 1) * dvs[2]};
  D ndet = -dn[0] * ddet[0] - dn[1] * ddet[1] - dn[2] * ddet[2];
  D bmin[3] = {D(FLT_MAX), D(FLT_MAX), D(FLT_MAX)};
  D bmax[3] = {D(-200000.f), D(-200000.f), D(-200000.f)};
  for (int c = 0; c < 8; ++c) {
    // corner order of the unrolled loop: (x, y, z) bits = (c>>2, c>>1, c)&1
    D p[3] = {(c & 4) ? mcMin[0] + (mcMax[0] - mcMin[0]) : mcMin[0],
              (c & 2) ? mcMin[1] + (mcMax[1] - mcMin[1]) : mcMin[1],
              (c & 1) ? mcMin[2] + (mcMax[2] - mcMin[2]) : mcMin[2]};
    D t = (dn[0] * p[0] + dn[1] * p[1] + dn[2] * p[2]);
    t += ndet;
    t = std::fabs(t);
    if (c == 0 && !(t >= D(distMin) && t < D(distMax))) return;
    for (int k = 0; k < 3; ++k) {
      D hp = t * (-dn[k]) + p[k];
      bmin[k] = fmn(hp, bmin[k]);
      bmax[k] = fmx(hp, bmax[k]);
    }
  }
  D lo[3], hi[3];
  for (int k = 0; k < 3; ++k) { lo[k] = fmn(bmin[k], bmax[k]); hi[k] = fmx(bmin[k], bmax[k]); }
  if (dn[0] <= D(0)) std::swap(lo[0], hi[0]);
  auto detmul = [&](const D p[3], D o[3]) {
    for (int r = 0; r < 3; ++r)
      o[r] = D(g.detMat[r * 4 + 0]) * p[0] + D(g.detMat[r * 4 + 1]) * p[1] + D(g.detMat[r * 4 + 2]) * p[2] +
             D(1) * D(g.detMat[r * 4 + 3]);
  };
  R bbMin[3] = {R(g.bbMin[0]), R(g.bbMin[1]), R(g.bbMin[2])};
  R vs[3] = {R(g.vs[0]), R(g.vs[1]), R(g.vs[2])};
  R n[3] = {R(g.n[0]), R(g.n[1]), R(g.n[2])};
  R det[3] = {R(g.det[0]), R(g.det[1]), R(g.det[2])};
  D plo[3], phi[3];
  detmul(lo, plo);
  detmul(hi, phi);
  int pb_x = (int)std::floor(fmn(plo[0], phi[0]));
  int pb_z = (int)std::floor(fmn(plo[1], phi[1]));
  int pb_y = (int)std::ceil(fmx(plo[0], phi[0]));
  int pb_w = (int)std::ceil(fmx(plo[1], phi[1]));
  auto clampf = [](int v, int hiv) -> int { return (int)std::fmin(std::fmax((float)v, 0.f), (float)hiv); };
  pb_x = clampf(pb_x, pw - 1);
  pb_y = clampf(pb_y, pw - 1);
  pb_z = clampf(pb_z, ph - 1);
  pb_w = clampf(pb_w, ph - 1);

  const float inv = 1.0f / (float)os;  // maxOverSampleInv (Reconstructor.cpp:885)
  R acc[4] = {0, 0, 0, 0}, dacc[4] = {0, 0, 0, 0};
  R u[3] = {R(g.u[0]), R(g.u[1]), R(g.u[2])}, v[3] = {R(g.v[0]), R(g.v[1]), R(g.v[2])};
  for (float pyf = (float)pb_z + inv * 0.5f; pyf < (float)pb_w; pyf += inv) {
    for (float pxf = (float)pb_x + inv * 0.5f; pxf < (float)pb_y; pxf += inv) {
      R px = pxf, py = pyf;
      R xA = R(g.anisoInv[0]) * px + R(g.anisoInv[1]) * py + R(g.anisoInv[2]) * R(1);
      R yA = R(g.anisoInv[3]) * px + R(g.anisoInv[4]) * py + R(g.anisoInv[5]) * R(1);
      R ray[3], src[3];
      for (int k = 0; k < 3; ++k) {
        R r = det[k];
        r = r + px * u[k];
        r = r + py * v[k];
        ray[k] = r;
      }
      // c_source = ray + 100000.0 * n is evaluated in double and stored as
      // float in the reference (:534-536); ray = normalize(ray - c_source).
      for (int k = 0; k < 3; ++k) src[k] = R((double)ray[k] + 100000.0 * (double)n[k]);
      for (int k = 0; k < 3; ++k) ray[k] = ray[k] - src[k];
      R inv_len = R(1) / std::sqrt(ray[0] * ray[0] + ray[1] * ray[1] + ray[2] * ray[2]);
      for (int k = 0; k < 3; ++k) ray[k] = ray[k] * inv_len;
      R sample = 0;
      bool sampled = false;
      for (int q = 0; q < 4; ++q) {
        R blo[3] = {bbMin[0] + R(x + q) * vs[0], bbMin[1] + R(y) * vs[1], bbMin[2] + R(z) * vs[2]};
        R bhi[3] = {bbMin[0] + R(x + q + 1) * vs[0], bbMin[1] + R(y + 1) * vs[1], bbMin[2] + R(z + 1) * vs[2]};
        R tin, tout;
        box_hit<R>(src, ray, blo, bhi, tin, tout);
        if (tout - tin > R(0)) {
          if (!sampled) {
            sample = tex2d<R>(img, pw, ph, pitchElems, xA, yA, linear, q9);
            sampled = true;
          }
          acc[q] += sample * (tout - tin);
          dacc[q] += (tout - tin);
        }
      }
    }
  }
  for (int q = 0; q < 4; ++q) {
    R d = fmx(R(0), dacc[q]);
    if (d != R(0)) vb[q] = (float)(R(vb[q]) + (R(lambda) * acc[q] / d));
  }
  for (int k = 0; k < 4; ++k) {
    if (dtype == 0) ((float*)volData)[base + k] = vb[k];
    else if (dtype == 1) ((uint16_t*)volData)[base + k] = float_to_half_rn(vb[k]);
    else ((uint16_t*)volData)[base + k] = float_to_bf16_rn(vb[k]);
  }
}

// ------------------------------------------------------------------ FFT
// Complex DFT in double, sign -1 forward: iterative radix-2 for power-of-two
// lengths, direct O(n^2) summation otherwise (the oracle's sizes are small
// when they are not powers of two).
using cd = std::complex<double>;
void dft_direct(cd* a, int n, int sign) {
  std::vector<cd> out(n), tw(n);
  for (int k = 0; k < n; ++k) tw[k] = cd(std::cos(sign * 2.0 * M_PI * k / n), std::sin(sign * 2.0 * M_PI * k / n));
  for (int k = 0; k < n; ++k) {
    cd s(0);
    for (int j = 0; j < n; ++j) s += a[j] * tw[(long)j * k % n];
    out[k] = s;
  }
  for (int k = 0; k < n; ++k) a[k] = out[k];
}

void fft1d(cd* a, int n, int sign) {
  if (n & (n - 1)) {
    dft_direct(a, n, sign);
    return;
  }
  for (int i = 1, j = 0; i < n; ++i) {
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    double ang = sign * 2.0 * M_PI / len;
    cd wl(std::cos(ang), std::sin(ang));
    for (int i = 0; i < n; i += len) {
      cd w(1);
      for (int j = 0; j < len / 2; ++j) {
        cd u = a[i + j], v = a[i + j + len / 2] * w;
        a[i + j] = u + v;
        a[i + j + len / 2] = u - v;
        w *= wl;
      }
    }
  }
}

// N x N real [y][x] -> half spectrum [y][N/2+1] (cuFFT R2C layout, unnormalised)
void r2c_2d(const float* in, std::complex<float>* out, int n, int nthreads) {
  std::vector<cd> tmp((size_t)n * n);
  parallel_for(n, nthreads, [&](int y) {
    std::vector<cd> row(n);
    for (int x = 0; x < n; ++x) row[x] = cd(in[(size_t)y * n + x], 0);
    fft1d(row.data(), n, -1);
    for (int x = 0; x < n; ++x) tmp[(size_t)y * n + x] = row[x];
  });
  int nh = n / 2 + 1;
  parallel_for(nh, nthreads, [&](int x) {
    std::vector<cd> col(n);
    for (int y = 0; y < n; ++y) col[y] = tmp[(size_t)y * n + x];
    fft1d(col.data(), n, -1);
    for (int y = 0; y < n; ++y) out[(size_t)y * nh + x] = std::complex<float>((float)col[y].real(), (float)col[y].imag());
  });
}

// Half spectrum -> N x N real (cuFFT C2R, unnormalised).  The missing half is
// taken as the conjugate mirror of the stored half.
void c2r_2d(const std::complex<float>* in, float* out, int n, int nthreads) {
  int nh = n / 2 + 1;
  std::vector<cd> tmp((size_t)n * n);
  parallel_for(nh, nthreads, [&](int x) {
    std::vector<cd> col(n);
    for (int y = 0; y < n; ++y) col[y] = cd(in[(size_t)y * nh + x].real(), in[(size_t)y * nh + x].imag());
    fft1d(col.data(), n, +1);
    for (int y = 0; y < n; ++y) tmp[(size_t)y * n + x] = col[y];
  });
  parallel_for(n, nthreads, [&](int y) {
    std::vector<cd> row(n);
    for (int x = 0; x < nh; ++x) row[x] = tmp[(size_t)y * n + x];
    // The full spectrum obeys X(ky, N-kx) = conj(X(-ky, kx)); after the
    // inverse transform along y this becomes Z(y, N-kx) = conj(Z(y, kx)).
    for (int x = nh; x < n; ++x) row[x] = std::conj(tmp[(size_t)y * n + (n - x)]);
    fft1d(row.data(), n, +1);
    for (int x = 0; x < n; ++x) out[(size_t)y * n + x] = (float)row[x].real();
  });
}

}  // namespace

// =====================================================================
// C ABI used by the Python test harness (ctypes)
// =====================================================================
extern "C" {

// Kernel `rot3d` (wbpWeighting.cu:389-405) as RotKernel::operator()
// launches it (Kernels.cpp:1338-1381): output voxel p = size^3 input read
// through tex3D at c + R^T (p - c) + 0.5, c = size / 2 (integer division),
// rot row-major [3][3]. q9: 8-bit filter weights.
int orc_rotate_volume(const float* in, float* out, int size, const float* rot, int q9, int nthreads) {
  VolView vv{in, size, size, size, 0};
  const float c = (float)(size / 2);
  parallel_for(size * size, nthreads, [&](int zy) {
    const int z = zy / size, y = zy % size;
    for (int x = 0; x < size; ++x) {
      const float vx = (float)x - c, vy = (float)y - c, vz = (float)z - c;
      const float px = c + rot[0] * vx + rot[3] * vy + rot[6] * vz;
      const float py = c + rot[1] * vx + rot[4] * vy + rot[7] * vz;
      const float pz = c + rot[2] * vx + rot[5] * vy + rot[8] * vz;
      out[((size_t)z * size + y) * size + x] = tex3d<float>(vv, px + 0.5f, py + 0.5f, pz + 0.5f, q9 != 0);
    }
  });
  return 0;
}

// Kernel `march` over the ROI (ForwardProjectionRayMarcher_TL.cu:58-160).
// precision: 0 = FP32, 1 = FP64.  proj/dist are dense [proj_y][proj_x].
int orc_fp_march(const OrcGeom* g, const void* vol, int dtype, int proj_x, int proj_y, float* proj, float* dist,
                 int roi_x0, int roi_y0, int roi_x1, int roi_y1, int precision, int q9, int exact_step,
                 int nthreads) {
  VolView vv{vol, (int)g->dim[0], (int)g->dim[1], (int)g->dim[2], dtype};
  parallel_for(proj_y, nthreads, [&](int y) {
    if (y < roi_y0 || y >= roi_y1) return;
    for (int x = roi_x0; x < std::min(roi_x1, proj_x); ++x) {
      size_t i = (size_t)y * proj_x + x;
      if (precision) march_pixel<double>(*g, vv, x, y, q9, exact_step, &proj[i], &dist[i]);
      else march_pixel<float>(*g, vv, x, y, q9, exact_step, &proj[i], &dist[i]);
    }
  });
  return 0;
}

// Kernel `slicer` (ForwardProjectionSlicer.cu:57-220); proj += slab integral.
int orc_fp_slicer(const OrcGeom* g, const void* vol, int dtype, int proj_x, int proj_y, float* proj, float tmin,
                  float tmax, int precision, int q9, int fix_first_sample, int nthreads) {
  VolView vv{vol, (int)g->dim[0], (int)g->dim[1], (int)g->dim[2], dtype};
  parallel_for(proj_y, nthreads, [&](int y) {
    for (int x = 0; x < proj_x; ++x) {
      size_t i = (size_t)y * proj_x + x;
      if (precision) slicer_pixel<double>(*g, vv, x, y, tmin, tmax, q9, fix_first_sample, &proj[i]);
      else slicer_pixel<float>(*g, vv, x, y, tmin, tmax, q9, fix_first_sample, &proj[i]);
    }
  });
  return 0;
}

// Kernel `volTraversalLength` (ForwardProjectionSlicer.cu:224-288); dist +=.
int orc_vol_traversal_length(const OrcGeom* g, int proj_x, int proj_y, float* dist, int precision, int nthreads) {
  parallel_for(proj_y, nthreads, [&](int y) {
    for (int x = 0; x < proj_x; ++x) {
      size_t i = (size_t)y * proj_x + x;
      if (precision) travlen_pixel<double>(*g, x, y, &dist[i]);
      else travlen_pixel<float>(*g, x, y, &dist[i]);
    }
  });
  return 0;
}

// Kernel `compare` (Compare.cu:50-130): virt <- tapered residual per unit length.
int orc_compare(int proj_x, int proj_y, const float* real, float* virt, const float* dist, float realLength,
                const float* cut4, const float* dim4, float scale) {
  for (int y = 0; y < proj_y; ++y)
    for (int x = 0; x < proj_x; ++x) {
      size_t i = (size_t)y * proj_x + x;
      float val = dist[i], error;
      if (val >= 1.0f) error = ((real[i]) - ((virt[i] / scale) / val * realLength)) / realLength * scale;
      else error = 0;
      float yb = 1, ya = 1, xb = 1, xa = 1;
      float fy = (float)(unsigned)y, fx = (float)(unsigned)x;
      if (fy < cut4[2] + dim4[2]) yb = taper((fy - cut4[2]) / dim4[2]);
      if (fy > (float)proj_y - dim4[3] - cut4[3] - 1)
        ya = taper(((float)(unsigned)(proj_y - y - 1) - cut4[3] - (float)(proj_y - 1)) / dim4[3]);
      if (fx < cut4[1] + dim4[1]) xb = taper((fx - cut4[1]) / dim4[1]);
      if (fx > (float)proj_x - dim4[0] - cut4[0] - 1)
        xa = taper(((float)(unsigned)(proj_x - x - 1) - cut4[0] - (float)(proj_x - 1)) / dim4[0]);
      virt[i] = xa * xb * ya * yb * error;
    }
  return 0;
}

static float seg_dist(int vx, int vy, int wx, int wy, int x, int y) {  // Compare.cu:137-163
  auto d = [](float ax, float ay, float bx, float by) { return std::sqrt((ax - bx) * (ax - bx) + (ay - by) * (ay - by)); };
  float l2 = (float)((vx - wx) * (vx - wx) + (vy - wy) * (vy - wy));
  if (l2 == 0) return d((float)vx, (float)vy, (float)x, (float)y);
  float x1 = (float)(x - vx), y1 = (float)(y - vy), x2 = (float)(wx - vx), y2 = (float)(wy - vy);
  float t = (x1 * x2 + y1 * y2) / l2;
  if (t < 0.0f) return d((float)x, (float)y, (float)vx, (float)vy);
  if (t > 1.0f) return d((float)x, (float)y, (float)wx, (float)wy);
  float x3 = vx + t * (wx - vx), y3 = vy + t * (wy - vy);
  return d((float)x, (float)y, x3, y3);
}

// Kernel `cropBorder` (Compare.cu:171-277); p = 8 ints (p1..p4 as x,y pairs).
int orc_crop_border(int proj_x, int proj_y, float* img, const float* cut2, const float* dim2, const int* p) {
  int p1x = p[0], p1y = p[1], p2x = p[2], p2y = p[3], p3x = p[4], p3y = p[5], p4x = p[6], p4y = p[7];
  for (int y = 0; y < proj_y; ++y)
    for (int x = 0; x < proj_x; ++x) {
      size_t i = (size_t)y * proj_x + x;
      float dX = 0, dY = 0;
      if ((p2x - p1x) * (y - p1y) - (p2y - p1y) * (x - p1x) < 0 && (p3x - p4x) * (y - p4y) - (p3y - p4y) * (x - p4x) < 0 &&
          (p1x - p3x) * (y - p3y) - (p1y - p3y) * (x - p3x) < 0 && (p4x - p2x) * (y - p2y) - (p4y - p2y) * (x - p2x) < 0) {
        dX = 1;
        dY = 1;
        float mx = 3.0f * proj_x, my = 3.0f * proj_y;
        mx = std::fmin(mx, seg_dist(p1x, p1y, p2x, p2y, x, y));
        mx = std::fmin(mx, seg_dist(p4x, p4y, p3x, p3y, x, y));
        mx = std::fmin(mx, (float)x);
        mx = std::fmin(mx, (float)(proj_x - x - 1));
        my = std::fmin(my, seg_dist(p3x, p3y, p1x, p1y, x, y));
        my = std::fmin(my, seg_dist(p2x, p2y, p4x, p4y, x, y));
        my = std::fmin(my, (float)y);
        my = std::fmin(my, (float)(proj_y - y - 1));
        if (mx < cut2[0] + dim2[0]) dX = taper((mx - cut2[0]) / dim2[0]);
        if (my < cut2[1] + dim2[1]) dY = taper((my - cut2[1]) / dim2[1]);
      }
      img[i] = dX * dY * img[i];
    }
  return 0;
}

// Kernel `backProjection` (FP32 storage, dtype 0) / `backProjectionFP16`
// (dtype 1); dtype 2 stores bfloat16.  img is dense [proj_y][proj_x].
int orc_bp(const OrcGeom* g, void* vol, int dtype, const float* img, int proj_x, int proj_y, float lambda, int os,
           float distMin, float distMax, int linear, int precision, int q9, int nthreads) {
  const int nq = g->dimXQuarter, ny = (int)g->dim[1], nz = (int)g->dim[2];
  parallel_for(nz * ny, nthreads, [&](int zy) {
    int z = zy / ny, y = zy % ny;
    for (int q = 0; q < nq; ++q) {
      if (precision == 2)  // float decisions, double chords and sums
        bp_quad<double, float>(*g, vol, dtype, q, y, z, img, proj_x, proj_y, proj_x, lambda, os, distMin, distMax,
                               linear, q9);
      else if (precision)
        bp_quad<double, double>(*g, vol, dtype, q, y, z, img, proj_x, proj_y, proj_x, lambda, os, distMin, distMax,
                                linear, q9);
      else
        bp_quad<float, float>(*g, vol, dtype, q, y, z, img, proj_x, proj_y, proj_x, lambda, os, distMin, distMax,
                              linear, q9);
    }
  });
  return 0;
}

// Kernel `makeSquare` (CopyToSquare.cu:38-92); stride in floats.
int orc_make_square(int proj_x, int proj_y, int maxsize, int stride, const float* in, float* out, int bx, int by,
                    int mirrorY, int fillZero) {
  for (int y = 0; y < maxsize; ++y)
    for (int x = 0; x < maxsize; ++x) {
      if (fillZero) {
        float val = 0;
        int xi = x - bx, yi = y - by;
        if (xi >= 0 && xi < proj_x && yi >= 0 && yi < proj_y) {
          if (mirrorY) yi = proj_y - yi - 1;
          val = in[(size_t)yi * stride + xi];
        }
        out[(size_t)y * maxsize + x] = val;
      } else {
        int xi = x - bx;
        if (xi < 0) xi = -xi - 1;
        if (xi >= proj_x) { xi = xi - proj_x; xi = proj_x - xi - 1; }
        int yi = y - by;
        if (yi < 0) yi = -yi - 1;
        if (yi >= proj_y) { yi = yi - proj_y; yi = proj_y - yi - 1; }
        if (mirrorY) yi = proj_y - yi - 1;
        out[(size_t)y * maxsize + x] = in[(size_t)yi * stride + xi];
      }
    }
  return 0;
}

// Kernel `ctf` (ctf.cu:82-240) on the (N/2+1) x N half spectrum, with the
// constants of SetConstantValues(CTFKernel, ...) (Kernels.cpp:1104-1131) and
// the unit conversions of CTFKernel::operator() (Kernels.cpp:395-436):
// defocus in nm, angle in degrees, pixel size in nm, Cs in mm, voltage in kV.
int orc_ctf(float* spec, int n, float defocusMin_nm, float defocusMax_nm, float angle_deg, int applyForFP,
            int phaseFlipOnly, float wiener, const float* betaFac, float cs_mm, float voltage_kV, float ampContrast,
            float pixelsize_nm, int precision) {
  const int nh = n / 2 + 1;
  const double PI = 3.14159265358979323846;
  float pixelsize = pixelsize_nm * std::pow(10.0f, -9.0f);
  float pixelcount = (float)n;
  float maxFreq = (float)(1.0 / (pixelsize * 2.0f));
  float freqStep = maxFreq / (pixelcount / 2.0f);
  float phaseC = std::sqrt(1 - ampContrast * ampContrast);
  float d0 = defocusMin_nm * 0.000000001f, d1 = defocusMax_nm * 0.000000001f;
  float ang = angle_deg / 180.0f * (float)PI;
  // lambda: relativistic electron wavelength as the reference's macro (ctf.cu:62)
  float hc = ((float)6.63E-34) * ((float)3.00E+08);
  double X = (double)(2 * 511 * voltage_kV * 1000.0f * 1000.0f) + (double)(voltage_kV * voltage_kV * 1000.0f * 1000.0f);
  float lam = hc / (float)std::sqrt((float)(X * 1.602E-19 * 1.602E-19));
  float Cs = cs_mm * 0.001f;
  std::complex<float>* c = (std::complex<float>*)spec;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nh; ++x) {
      double xpos = x, ypos = y;
      if (ypos > pixelcount * 0.5f) ypos = (pixelcount - ypos) * -1.0f;
      double alpha = (xpos == 0) ? PI * 0.5 : std::atan2(ypos, xpos);
      double beta = alpha - ang;
      double defocus = d0 + (1 - std::cos(2 * beta)) * (d1 - d0);
      double radius = std::sqrt(xpos * xpos + ypos * ypos);
      double length = radius * freqStep;
      double L = lam;
      double m = (PI / 2.0) * (Cs * L * L * L * length * length * length * length - 2 * defocus * L * length * length);
      double nn = phaseC * std::sin(m) + ampContrast * std::cos(m);
      if (!precision) {  // FP32 evaluation of the same expressions
        float xf = (float)xpos, yf = (float)ypos;
        float al = (xf == 0) ? (float)(PI * 0.5) : std::atan2(yf, xf);
        float be = al - ang;
        float de = d0 + (1 - std::cos(2 * be)) * (d1 - d0);
        float le = std::sqrt(xf * xf + yf * yf) * freqStep;
        float mf = ((float)PI / 2.0f) * (Cs * lam * lam * lam * le * le * le * le - 2 * de * lam * le * le);
        nn = phaseC * std::sin(mf) + ampContrast * std::cos(mf);
        length = le;
      }
      std::complex<float> res = c[(size_t)y * nh + x];
      if (applyForFP && radius > betaFac[0] && !phaseFlipOnly) {
        double l = length / 100000000.0;
        double e = std::exp(-betaFac[1] * l - betaFac[2] * l * l - betaFac[3] * l * l * l);
        e = std::max(e, 0.01);
        double val = nn * e;
        if (std::fabs(val) < 0.0001 && val >= 0) val = 0.0001;
        if (std::fabs(val) < 0.0001 && val < 0) val = -0.0001;
        res = std::complex<float>((float)(res.real() * -val), (float)(res.imag() * -val));
      }
      if (!applyForFP && radius > betaFac[0] && !phaseFlipOnly) {
        double l = length / 100000000.0;
        double e = std::exp(-betaFac[1] * l - betaFac[2] * l * l - betaFac[3] * l * l * l);
        e = std::max(e, (double)wiener);
        double val = nn * e;
        double f = -val / (val * val + wiener);
        res = std::complex<float>((float)(res.real() * f), (float)(res.imag() * f));
      }
      if (phaseFlipOnly && nn >= 0) res = -res;
      c[(size_t)y * nh + x] = res;
    }
  return 0;
}

// Kernel `wbpWeighting` (wbpWeighting.cu:50-144); psi in degrees as passed to
// WbpWeightingKernel::operator() (angle = -psi/180*pi, Kernels.cpp:456).
// fm: 0 RAMP, 1 EXACT (weight 1), 2 CONTRAST2, 3 CONTRAST10, 4 CONTRAST30.
int orc_wbp_weighting(float* spec, int n, float psi_deg, int fm) {
  const int nh = n / 2 + 1;
  float a = -psi_deg / 180.0f * 3.14159265358979f;
  double s = std::sin((double)a), co = std::cos((double)a);
  static const double P[3][4] = {{1.000654227857550, 0.006008581017124, 0.004159659493151, 0.000975903396538},
                                 {1.003784816598589, 0.029016377161629, 0.019582940715148, 0.004559409669984},
                                 {0.999884616010943, 0.000307646262566, 0.004742915272196, 0.004806551368900}};
  std::complex<float>* c = (std::complex<float>*)spec;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nh; ++x) {
      double xp = x, yp = y;
      if (yp > n * 0.5f) yp = (n - yp) * -1.0;
      double yr = s * xp + co * yp;
      double length = yr / n / 2.0;
      double w = 1;
      if (fm == 0) w = std::min(std::fabs(length), 1.0);
      else if (fm >= 2 && fm <= 4) {
        const double* p = P[fm - 2];
        if (length == 0) w = 0;
        else {
          double lf = std::log(std::fabs(length));
          w = p[0] + p[1] * lf + p[2] * lf * lf + p[3] * lf * lf * lf;
        }
        w = std::max(0.0, std::min(w, 1.0));
      }
      c[(size_t)y * nh + x] *= (float)w;
    }
  return 0;
}

// Kernel `fourierFilter` (wbpWeighting.cu:148-212).
int orc_fourier_filter(float* spec, int n, float lp, float hp, float lps, float hps) {
  const int nh = n / 2 + 1;
  std::complex<float>* c = (std::complex<float>*)spec;
  lp = lp - lps;
  hp = hp + hps;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nh; ++x) {
      float mx = (float)x, my = (float)y;
      if (my > n * 0.5f) my = (n - my) * -1.0f;
      float dist = std::sqrt(mx * mx + my * my);
      float fil = 0;
      if (lp > 0) { if (dist <= lp) fil = 1; }
      else { if (dist <= n / 2 - 1) fil = 1; }
      if (lps > 0) {
        float fil2 = (-fil + 1.0f) * std::exp(-((dist - lp) * (dist - lp) / (2 * lps * lps)));
        if (fil2 > 0.001f) fil = fil2;
      }
      if (lps > 0 && lp == 0 && hp == 0 && hps == 0) fil = std::exp(-((dist - lp) * (dist - lp) / (2 * lps * lps)));
      if (hp > 0) {
        float fil2 = 0;
        if (dist >= hp) fil2 = 1;
        fil *= fil2;
        if (hps > 0) {
          float fil3 = (-fil2 + 1) * std::exp(-((dist - hp) * (dist - hp) / (2 * hps * hps)));
          if (fil3 > 0.001f) fil = fil3;
        }
      }
      c[(size_t)y * nh + x] *= fil;
    }
  return 0;
}

// Kernel `doseWeighting` (wbpWeighting.cu:216-240).
int orc_dose_weighting(float* spec, int n, float dose, float pixelsize) {
  const int nh = n / 2 + 1;
  std::complex<float>* c = (std::complex<float>*)spec;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < nh; ++x) {
      float mx = (float)x, my = (float)y;
      if (my > n * 0.5f) my = (n - my) * -1.0f;
      float dist = std::sqrt(mx * mx + my * my);
      dist = dist / (float)(n / 2 / pixelsize);
      c[(size_t)y * nh + x] *= std::exp(-dose * dist);
    }
  return 0;
}

int orc_r2c(const float* in, float* out, int n, int nthreads) {
  r2c_2d(in, (std::complex<float>*)out, n, nthreads);
  return 0;
}
int orc_c2r(const float* in, float* out, int n, int nthreads) {
  c2r_2d((const std::complex<float>*)in, out, n, nthreads);
  return 0;
}

int orc_float_to_half(const float* in, uint16_t* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = float_to_half_rn(in[i]);
  return 0;
}
int orc_half_to_float(const uint16_t* in, float* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = half_to_float(in[i]);
  return 0;
}
int orc_float_to_bf16(const float* in, uint16_t* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = float_to_bf16_rn(in[i]);
  return 0;
}

}  // extern "C"

// ------------------------------------------ differentiable projection model
// CPU counterpart of esb_projection_loss_grad / esb_fp_adjoint (the GPU
// library's esb_adjoint.cu). The reference has no gradient; the model is the
// fast projector's: each sub-ray sums the trilinear interpolant over the
// samples of the reference's float ray recurrence, and a detector offset
// (s_u, s_v) in pixels translates every sample rigidly by s_u * u + s_v * v
// (pixel axes through the magnification anisotropy). This function places
// the unshifted samples with the GPU's float operations (ray source, box
// entry, step, first sample, per-sample step), adds the translation in
// double and evaluates values, gradients, the loss and the adjoint scatter
// in double, sample by sample.
namespace {

struct ModelOut {
  double part[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> grad;
};

// trilinear value and gradient (interpolation coordinates) at q, clamp
// addressing; optional scatter of w * basis into g
inline void model_sample(const VolView& V, double qx, double qy, double qz, double& val, double& ga, double& gb,
                         double& gc, double* g, double w) {
  const double fx = std::floor(qx), fy = std::floor(qy), fz = std::floor(qz);
  const double a = qx - fx, b = qy - fy, c = qz - fz;
  auto cl = [](double f, int n) -> long {
    long i = (long)std::max(std::min(f, 1.0e9), -1.0e9);
    return i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
  };
  const long x0 = cl(fx, V.nx), x1 = cl(fx + 1, V.nx), y0 = cl(fy, V.ny), y1 = cl(fy + 1, V.ny);
  const long z0 = cl(fz, V.nz), z1 = cl(fz + 1, V.nz);
  const long sy = V.nx, sz = (long)V.nx * V.ny;
  const long idx[8] = {z0 * sz + y0 * sy + x0, z0 * sz + y0 * sy + x1, z0 * sz + y1 * sy + x0,
                       z0 * sz + y1 * sy + x1, z1 * sz + y0 * sy + x0, z1 * sz + y0 * sy + x1,
                       z1 * sz + y1 * sy + x0, z1 * sz + y1 * sy + x1};
  double cv[8];
  for (int k = 0; k < 8; ++k) cv[k] = V.at(idx[k]);
  const double ia = 1 - a, ib = 1 - b, ic = 1 - c;
  const double B[8] = {ia * ib * ic, a * ib * ic, ia * b * ic, a * b * ic, ia * ib * c, a * ib * c, ia * b * c, a * b * c};
  val = 0;
  for (int k = 0; k < 8; ++k) val += B[k] * cv[k];
  ga = ib * ic * (cv[1] - cv[0]) + b * ic * (cv[3] - cv[2]) + ib * c * (cv[5] - cv[4]) + b * c * (cv[7] - cv[6]);
  gb = ia * ic * (cv[2] - cv[0]) + a * ic * (cv[3] - cv[1]) + ia * c * (cv[6] - cv[4]) + a * c * (cv[7] - cv[5]);
  gc = ia * ib * (cv[4] - cv[0]) + a * ib * (cv[5] - cv[1]) + ia * b * (cv[6] - cv[2]) + a * b * (cv[7] - cv[3]);
  if (g)
    for (int k = 0; k < 8; ++k) g[idx[k]] += w * B[k];
}

// float operations of the GPU model
struct ModelRayGeom {
  float s[3];
  float tin, tout;
};

inline void model_ray_geom(const OrcGeom& G, float px, float py, ModelRayGeom& R) {
  const float xA = (G.aniso[0] * px + G.aniso[1] * py) + G.aniso[2] * 1.0f;
  const float yA = (G.aniso[3] * px + G.aniso[4] * py) + G.aniso[5] * 1.0f;
  for (int k = 0; k < 3; ++k) R.s[k] = yA * G.v[k] + (xA * G.u[k] + G.det[k]);
  float lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    const float e = (G.bbMin[k] - R.s[k]) / G.n[k], x = (G.bbMax[k] - R.s[k]) / G.n[k];
    lo[k] = std::fmin(e, x);
    hi[k] = std::fmax(e, x);
  }
  R.tin = std::fmax(std::fmax(lo[0], lo[1]), lo[2]);
  R.tout = std::fmin(std::fmin(hi[0], hi[1]), hi[2]);
}

inline float model_interp(const OrcGeom& G, int k, float p) {
  float q = ((p - G.bbMin[k]) * G.bbRcp[k]) * G.dim[k];
  if (k == 2) q = q - G.zShift;
  return q - 0.5f;
}

inline int model_progression(float t0, float tout, float h, float& step, bool& ok) {
  ok = true;
  step = h;
  if (!(t0 <= tout)) return 0;
  const float t1 = t0 + h;
  step = t1 - t0;
  const float t2 = t1 + h;
  if (!(t0 > 0.0f) || t2 - t1 != step || !(step > 0.0f)) {
    ok = false;
    return 0;
  }
  int J = (int)((tout - t0) / step) + 1;
  if (J < 1) J = 1;
  while (J > 1 && t0 + (float)(J - 1) * step > tout) --J;
  while (t0 + (float)J * step <= tout) ++J;
  const float tl = t0 + (float)(J - 1) * step;
  int e0, e1;
  std::frexp(t0, &e0);
  std::frexp(tl, &e1);
  if (e0 != e1) ok = false;
  return J;
}

// one sub-ray: sum of values and of gradients; with g != nullptr, scatter w
void model_subray(const OrcGeom& G, const VolView& V, const ModelRayGeom& R, const double* d, double& sum, double& ga,
                  double& gb, double& gc, double* g, double w) {
  sum = ga = gb = gc = 0;
  const float h = G.vs[0] * 0.15f;
  float step;
  bool ok;
  const int J = model_progression(R.tin, R.tout, h, step, ok);
  if (!(R.tin <= R.tout)) return;
  auto acc = [&](double qx, double qy, double qz) {
    double v, a, b, c;
    model_sample(V, qx, qy, qz, v, a, b, c, g, w);
    sum += v;
    ga += a;
    gb += b;
    gc += c;
  };
  if (!ok) {
    float t = R.tin;
    for (int guard = 0; guard < (1 << 22) && t <= R.tout; ++guard) {
      float q[3];
      for (int k = 0; k < 3; ++k) q[k] = model_interp(G, k, std::fmaf(t, G.n[k], R.s[k]));
      acc(q[0] + d[0], q[1] + d[1], q[2] + d[2]);
      t += h;
    }
    return;
  }
  float q0[3], dq[3];
  for (int k = 0; k < 3; ++k) {
    q0[k] = model_interp(G, k, std::fmaf(R.tin, G.n[k], R.s[k]));
    dq[k] = ((step * G.n[k]) * G.bbRcp[k]) * G.dim[k];
  }
  // the GPU rounds the translated first sample to float; the flat-y test
  // is taken on that value
  const float q0y = q0[1] + (float)d[1];
  const float ylast = std::fmaf((float)(J - 1), dq[1], q0y);
  const bool flat = std::fabs(dq[1]) * (float)J < 1e-5f && std::floor(q0y) == std::floor(ylast);
  for (int j = 0; j < J; ++j)
    acc((double)q0[0] + d[0] + j * (double)dq[0], (double)q0[1] + d[1] + (flat ? 0.0 : j * (double)dq[1]),
        (double)q0[2] + d[2] + j * (double)dq[2]);
}

}  // namespace

extern "C" {

// out6 += [L, dL/ds_u, dL/ds_v, sum (dp/ds_u)^2, sum dp/ds_u dp/ds_v,
// sum (dp/ds_v)^2]; grad_vol (double, may be NULL) += dL/dx; proj_out (may
// be NULL) = A(x, s); meas may be NULL (0).
int orc_model_loss_grad(const OrcGeom* g, const float* vol, int proj_x, int proj_y, const float* meas, float shift_u,
                        float shift_v, double* grad_vol, float* proj_out, double* out6, int nthreads) {
  const OrcGeom& G = *g;
  VolView V{vol, (int)G.dim[0], (int)G.dim[1], (int)G.dim[2], 0};
  const long nvox = (long)V.nx * V.ny * V.nz;
  const double kappa = (double)(G.vs[0] * 0.15f * 0.25f);
  // translation of the interpolation coordinates per pixel of offset
  double tu[3], tv[3], d[3];
  for (int k = 0; k < 3; ++k) {
    const double S = (double)G.bbRcp[k] * G.dim[k];
    tu[k] = ((double)G.aniso[0] * G.u[k] + (double)G.aniso[3] * G.v[k]) * S;
    tv[k] = ((double)G.aniso[1] * G.u[k] + (double)G.aniso[4] * G.v[k]) * S;
    d[k] = shift_u * tu[k] + shift_v * tv[k];
  }
  const int nt = std::max(1, std::min(nthreads, proj_y));
  std::vector<ModelOut> outs(nt);
  for (auto& o : outs)
    if (grad_vol) o.grad.assign(nvox, 0.0);
  std::atomic<int> next(0);
  auto work = [&](int tid) {
    ModelOut& O = outs[tid];
    for (;;) {
      const int y = next.fetch_add(1);
      if (y >= proj_y) break;
      for (int x = 0; x < proj_x; ++x) {
        ModelRayGeom R[4];
        double sum = 0, du = 0, dv = 0;
        bool hitr[4];
        for (int sub = 0; sub < 4; ++sub) {
          const float osx = (sub & 2) ? 0.75f : 0.25f, osy = (sub & 1) ? 0.75f : 0.25f;
          model_ray_geom(G, (float)x + osx, (float)y + osy, R[sub]);
          hitr[sub] = R[sub].tout - R[sub].tin > 0.0f;
          if (!hitr[sub]) continue;
          double s, a, b, c;
          model_subray(G, V, R[sub], d, s, a, b, c, nullptr, 0.0);
          du += a * tu[0] + b * tu[1] + c * tu[2];
          dv += a * tv[0] + b * tv[1] + c * tv[2];
          sum += s;
        }
        const double p = kappa * sum;
        const size_t i = (size_t)y * proj_x + x;
        if (proj_out) proj_out[i] = (float)p;
        const double r = meas ? p - (double)meas[i] : p;
        du *= kappa;
        dv *= kappa;
        O.part[0] += 0.5 * r * r;
        O.part[1] += r * du;
        O.part[2] += r * dv;
        O.part[3] += du * du;
        O.part[4] += du * dv;
        O.part[5] += dv * dv;
        if (grad_vol && r != 0.0)
          for (int sub = 0; sub < 4; ++sub) {
            if (!hitr[sub]) continue;
            double s, a, b, c;
            model_subray(G, V, R[sub], d, s, a, b, c, O.grad.data(), r * kappa);
          }
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(work, t);
  for (auto& th : pool) th.join();
  for (auto& o : outs) {
    for (int q = 0; q < 6; ++q) out6[q] += o.part[q];
    if (grad_vol)
      for (long v = 0; v < nvox; ++v) grad_vol[v] += o.grad[v];
  }
  return 0;
}

}  // extern "C"
