// Image-space kernels of the reconstruction path: residual ("compare"),
// volume-shadow crop, pad-to-square, the Fourier-space filters other than
// the CTF (WBP weighting, band-pass, dose weighting; the CTF filters are in
// esb_ctf.cu), the fused pre/post-FFT passes of the CTF chain and volume
// storage conversions.
#include <math.h>

#include "esb_device.cuh"

namespace esb {

__device__ __forceinline__ float taper(float w) {
  if (w < 0.0f) w = 0.0f;
  return 1.0f - expf(-(w * w * 9.0f));
}

// Kernel `compare` (Compare.cu:50-130). The upper-border factors of the
// reference evaluate to w = (-y - cut)/dim <= 0, i.e. a hard zero band of
// width dim+cut; the expressions are kept as written.
__global__ void k_compare(int pw, int ph, size_t pitchE, const float* __restrict__ real, float* __restrict__ virt,
                          const float* __restrict__ dist, float realLength, float4 cut, float4 dim, float scale) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= (unsigned)pw || y >= (unsigned)ph) return;
  const size_t i = (size_t)y * pitchE + x;
  float val = dist[i];
  float error;
  if (val >= 1.0f) error = ((real[i]) - ((virt[i] / scale) / val * realLength)) / realLength * scale;
  else error = 0.0f;
  float yb = 1.f, ya = 1.f, xb = 1.f, xa = 1.f;
  const float fy = (float)y, fx = (float)x;
  if (fy < cut.z + dim.z) yb = taper((fy - cut.z) / dim.z);
  if (fy > (float)ph - dim.w - cut.w - 1.0f) ya = taper(((float)((unsigned)ph - y - 1u) - cut.w - (float)(ph - 1)) / dim.w);
  if (fx < cut.y + dim.y) xb = taper((fx - cut.y) / dim.y);
  if (fx > (float)pw - dim.x - cut.x - 1.0f) xa = taper(((float)((unsigned)pw - x - 1u) - cut.x - (float)(pw - 1)) / dim.x);
  virt[i] = xa * xb * ya * yb * error;
}

__device__ __forceinline__ float seg_dist(int2 v, int2 w, int x, int y) {  // Compare.cu:137-163
  float l2 = (float)((v.x - w.x) * (v.x - w.x) + (v.y - w.y) * (v.y - w.y));
  auto d = [](float ax, float ay, float bx, float by) { return sqrtf((ax - bx) * (ax - bx) + (ay - by) * (ay - by)); };
  if (l2 == 0.0f) return d((float)v.x, (float)v.y, (float)x, (float)y);
  float x1 = (float)(x - v.x), y1 = (float)(y - v.y), x2 = (float)(w.x - v.x), y2 = (float)(w.y - v.y);
  float t = (x1 * x2 + y1 * y2) / l2;
  if (t < 0.0f) return d((float)x, (float)y, (float)v.x, (float)v.y);
  if (t > 1.0f) return d((float)x, (float)y, (float)w.x, (float)w.y);
  float x3 = v.x + t * (w.x - v.x), y3 = v.y + t * (w.y - v.y);
  return d((float)x, (float)y, x3, y3);
}

// Mask factor of kernel `cropBorder` (Compare.cu:171-277) at pixel (x, y).
__device__ __forceinline__ float crop_factor(int pw, int ph, int x, int y, float2 cut, float2 dim, int2 p1, int2 p2,
                                             int2 p3, int2 p4) {
  float dX = 0.f, dY = 0.f;
  if ((p2.x - p1.x) * (y - p1.y) - (p2.y - p1.y) * (x - p1.x) < 0 &&
      (p3.x - p4.x) * (y - p4.y) - (p3.y - p4.y) * (x - p4.x) < 0 &&
      (p1.x - p3.x) * (y - p3.y) - (p1.y - p3.y) * (x - p3.x) < 0 &&
      (p4.x - p2.x) * (y - p2.y) - (p4.y - p2.y) * (x - p2.x) < 0) {
    dX = 1.f;
    dY = 1.f;
    float mx = 3.0f * pw, my = 3.0f * ph;
    mx = fminf(mx, seg_dist(p1, p2, x, y));
    mx = fminf(mx, seg_dist(p4, p3, x, y));
    mx = fminf(mx, (float)x);
    mx = fminf(mx, (float)(pw - x - 1));
    my = fminf(my, seg_dist(p3, p1, x, y));
    my = fminf(my, seg_dist(p2, p4, x, y));
    my = fminf(my, (float)y);
    my = fminf(my, (float)(ph - y - 1));
    if (mx < cut.x + dim.x) dX = taper((mx - cut.x) / dim.x);
    if (my < cut.y + dim.y) dY = taper((my - cut.y) / dim.y);
  }
  return dX * dY;
}

__global__ void k_crop_border(int pw, int ph, size_t pitchE, float* __restrict__ img, float2 cut, float2 dim, int2 p1,
                              int2 p2, int2 p3, int2 p4) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= pw || y >= ph) return;
  const size_t i = (size_t)y * pitchE + x;
  img[i] = crop_factor(pw, ph, x, y, cut, dim, p1, p2, p3, p4) * img[i];
}

// Kernel `makeSquare` (CopyToSquare.cu:38-92).
__global__ void k_make_square(int pw, int ph, int maxsize, size_t strideE, const float* __restrict__ in,
                              float* __restrict__ out, int bx, int by, int mirrorY, int fillZero) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= maxsize || y >= maxsize) return;
  if (fillZero) {
    float val = 0.f;
    int xi = x - bx, yi = y - by;
    if (xi >= 0 && xi < pw && yi >= 0 && yi < ph) {
      if (mirrorY) yi = ph - yi - 1;
      val = in[(size_t)yi * strideE + xi];
    }
    out[(size_t)y * maxsize + x] = val;
  } else {
    int xi = x - bx;
    if (xi < 0) xi = -xi - 1;
    if (xi >= pw) { xi = xi - pw; xi = pw - xi - 1; }
    int yi = y - by;
    if (yi < 0) yi = -yi - 1;
    if (yi >= ph) { yi = yi - ph; yi = ph - yi - 1; }
    if (mirrorY) yi = ph - yi - 1;
    out[(size_t)y * maxsize + x] = in[(size_t)yi * strideE + xi];
  }
}

// Fused cropBorder (in place on img, the reference applies it to proj_d /
// dist_d before padding) + makeSquare with zero fill (Reconstructor.cpp:566-568,
// 954-956).
__global__ void k_crop_to_square(int pw, int ph, size_t pitchE, float* __restrict__ img, int apply_crop, float2 cut,
                                 float2 dim, int2 p1, int2 p2, int2 p3, int2 p4, int maxsize, float* __restrict__ sq,
                                 int bx, int by) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= maxsize || y >= maxsize) return;
  int xi = x - bx, yi = y - by;
  float val = 0.f;
  if (xi >= 0 && xi < pw && yi >= 0 && yi < ph) {
    const size_t i = (size_t)yi * pitchE + xi;
    val = img[i];
    if (apply_crop) {
      val = crop_factor(pw, ph, xi, yi, cut, dim, p1, p2, p3, p4) * val;
      img[i] = val;
    }
  }
  sq[(size_t)y * maxsize + x] = val;
}

// Fused nppiDivC (by N*N, centred W x H window) + cropBorder + optional
// accumulation into proj (Reconstructor.cpp:578-583, 962-965).
__global__ void k_square_to_image(const float* __restrict__ sq, int maxsize, size_t shift, float inv_norm, int pw,
                                  int ph, size_t pitchE, float* __restrict__ out, float* __restrict__ accum,
                                  int apply_crop, float2 cut, float2 dim, int2 p1, int2 p2, int2 p3, int2 p4,
                                  int transpose_out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= pw || y >= ph) return;
  float v = sq[shift + (size_t)y * maxsize + x] * inv_norm;
  if (apply_crop) v = crop_factor(pw, ph, x, y, cut, dim, p1, p2, p3, p4) * v;
  const size_t i = (size_t)y * pitchE + x;
  if (out) out[transpose_out ? (size_t)x * ph + y : i] = v;
  if (accum) accum[i] += v;
}

// k_square_to_image without crop or accumulation for a stack of squares:
// square blockIdx.z to image blockIdx.z.
__global__ void k_square_to_image_batch(const float* __restrict__ sq, size_t sq_stride, int maxsize, size_t shift,
                                        float inv_norm, int pw, int ph, size_t pitchE, float* __restrict__ out,
                                        size_t out_stride, int transpose_out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= pw || y >= ph) return;
  const float v = sq[blockIdx.z * sq_stride + shift + (size_t)y * maxsize + x] * inv_norm;
  out[blockIdx.z * out_stride + (transpose_out ? (size_t)x * ph + y : (size_t)y * pitchE + x)] = v;
}

// k_crop_to_square for `count` slab inputs at once (square blockIdx.z).
// seq_crop = 0: input k is images[k] (stride img_stride), cropped in place
// when apply_crop. seq_crop = 1: every input is the one image `images`,
// cropped again for each slab, as the reference re-applies cropBorder to the
// residual before every slab (Reconstructor.cpp:954): input k is the image
// cropped k + 1 times (from `first` = slabs already applied), and the image
// is left cropped count more times.
__global__ void k_crop_to_square_batch(int pw, int ph, float* __restrict__ images, size_t img_stride, int count,
                                       int apply_crop, int seq_crop, float2 cut, float2 dim, int2 p1, int2 p2, int2 p3,
                                       int2 p4, int maxsize, float* __restrict__ sq, size_t sq_stride, int bx,
                                       int by) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= maxsize || y >= maxsize) return;
  const int xi = x - bx, yi = y - by;
  const bool inside = xi >= 0 && xi < pw && yi >= 0 && yi < ph;
  if (!seq_crop) {
    for (int k = blockIdx.z; k < count; k += gridDim.z) {
      float val = 0.f;
      if (inside) {
        float* img = images + (size_t)k * img_stride;
        const size_t i = (size_t)yi * pw + xi;
        val = img[i];
        if (apply_crop) {
          val = crop_factor(pw, ph, xi, yi, cut, dim, p1, p2, p3, p4) * val;
          img[i] = val;
        }
      }
      sq[(size_t)k * sq_stride + (size_t)y * maxsize + x] = val;
    }
    return;
  }
  if (blockIdx.z != 0) return;
  float val = 0.f, f = 1.f;
  size_t i = 0;
  if (inside) {
    i = (size_t)yi * pw + xi;
    val = images[i];
    f = crop_factor(pw, ph, xi, yi, cut, dim, p1, p2, p3, p4);
  }
  for (int k = 0; k < count; ++k) {
    if (inside) val = f * val;
    sq[(size_t)k * sq_stride + (size_t)y * maxsize + x] = val;
  }
  if (inside) images[i] = val;
}


// k_square_to_image for `count` squares: scale by inv_norm, crop, and either
// write image k (transposed or not) or add the squares to `accum` one after
// the other in slab order (the reference's per-slab accumulation).
__global__ void k_square_to_image_many(const float* __restrict__ sq, size_t sq_stride, int count, int maxsize,
                                       size_t shift, float inv_norm, int pw, int ph, float* __restrict__ out,
                                       size_t out_stride, float* __restrict__ accum, int apply_crop, float2 cut,
                                       float2 dim, int2 p1, int2 p2, int2 p3, int2 p4, int transpose_out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= pw || y >= ph) return;
  const float f = apply_crop ? crop_factor(pw, ph, x, y, cut, dim, p1, p2, p3, p4) : 1.f;
  const size_t i = (size_t)y * pw + x;
  float a = accum ? accum[i] : 0.f;
  for (int k = 0; k < count; ++k) {
    float v = sq[(size_t)k * sq_stride + shift + (size_t)y * maxsize + x] * inv_norm;
    if (apply_crop) v = f * v;
    if (out) out[(size_t)k * out_stride + (transpose_out ? (size_t)x * ph + y : i)] = v;
    if (accum) a += v;
  }
  if (accum) accum[i] = a;
}

// out[x][y] = in[y][x] for a W x H image (32x32 tiles through shared memory).
__global__ void k_transpose(const float* __restrict__ in, int w, int h, size_t pitchE, float* __restrict__ out) {
  __shared__ float tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int x = bx + threadIdx.x, y = by + j;
    if (x < w && y < h) tile[j][threadIdx.x] = in[(size_t)y * pitchE + x];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int y = by + threadIdx.x, x = bx + j;
    if (x < w && y < h) out[(size_t)x * h + y] = tile[threadIdx.x][j];
  }
}



// Kernel `wbpWeighting` (wbpWeighting.cu:50-144).
__global__ void k_wbp_weighting(float2* __restrict__ spec, int n, float s, float co, int fm) {
  const unsigned x = blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= (unsigned)(n / 2 + 1) || y >= (unsigned)n) return;
  float xp = (float)x, yp = (float)y;
  if (yp > n * 0.5f) yp = (n - yp) * -1.0f;
  float yr = s * xp + co * yp;
  float length = yr / n / 2.0f;
  float w = 1.0f;
  if (fm == 0) {
    w = fminf(fabsf(length), 1.0f);
  } else if (fm >= 2 && fm <= 4) {
    const float P[3][4] = {{1.000654227857550f, 0.006008581017124f, 0.004159659493151f, 0.000975903396538f},
                           {1.003784816598589f, 0.029016377161629f, 0.019582940715148f, 0.004559409669984f},
                           {0.999884616010943f, 0.000307646262566f, 0.004742915272196f, 0.004806551368900f}};
    const float* p = P[fm - 2];
    if (length == 0.f) w = 0.f;
    else {
      float lf = logf(fabsf(length));
      w = p[0] + p[1] * lf + p[2] * lf * lf + p[3] * lf * lf * lf;
    }
    w = fmaxf(0.f, fminf(w, 1.f));
  }
  const size_t i = (size_t)y * (n / 2 + 1) + x;
  float2 r = spec[i];
  r.x *= w;
  r.y *= w;
  spec[i] = r;
}

// Kernel `fourierFilter` (wbpWeighting.cu:148-212).
__global__ void k_fourier_filter(float2* __restrict__ spec, int n, float lp, float hp, float lps, float hps) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= n / 2 + 1 || y >= n) return;
  float mx = (float)x, my = (float)y;
  if (my > n * 0.5f) my = (n - my) * -1.0f;
  float dist = sqrtf(mx * mx + my * my);
  float fil = 0.f;
  lp = lp - lps;
  hp = hp + hps;
  if (lp > 0) { if (dist <= lp) fil = 1.f; }
  else { if (dist <= n / 2 - 1) fil = 1.f; }
  if (lps > 0) {
    float fil2 = (-fil + 1.0f) * expf(-((dist - lp) * (dist - lp) / (2 * lps * lps)));
    if (fil2 > 0.001f) fil = fil2;
  }
  if (lps > 0 && lp == 0 && hp == 0 && hps == 0) fil = expf(-((dist - lp) * (dist - lp) / (2 * lps * lps)));
  if (hp > 0) {
    float fil2 = 0.f;
    if (dist >= hp) fil2 = 1.f;
    fil *= fil2;
    if (hps > 0) {
      float fil3 = (-fil2 + 1) * expf(-((dist - hp) * (dist - hp) / (2 * hps * hps)));
      if (fil3 > 0.001f) fil = fil3;
    }
  }
  const size_t i = (size_t)y * (n / 2 + 1) + x;
  float2 r = spec[i];
  r.x *= fil;
  r.y *= fil;
  spec[i] = r;
}

// Kernel `doseWeighting` (wbpWeighting.cu:216-240).
__global__ void k_dose_weighting(float2* __restrict__ spec, int n, float dose, float pixelsize) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= n / 2 + 1 || y >= n) return;
  float mx = (float)x, my = (float)y;
  if (my > n * 0.5f) my = (n - my) * -1.0f;
  float dist = sqrtf(mx * mx + my * my);
  dist = dist / (float)(n / 2 / pixelsize);
  float fil = expf(-dose * dist);
  const size_t i = (size_t)y * (n / 2 + 1) + x;
  float2 r = spec[i];
  r.x *= fil;
  r.y *= fil;
  spec[i] = r;
}

template <int VT>
__global__ void k_convert(const void* __restrict__ vol, long n, float* __restrict__ out, float sign) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = sign * Voxel<VT>::loadrw(vol, i);
}
template <int VT>
__global__ void k_store(const float* __restrict__ in, long n, void* __restrict__ vol) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    Voxel<VT>::store(vol, i, in[i]);
}

// ------------------------------------------------- projection preparation
// Reconstructor::PrepareProjection (Reconstructor.cpp:1158-1383).

// nppiConvert_{16s,16u,32s,32u}32f / copy: input pixels to float.
template <typename T>
__global__ void k_convert_input(const T* __restrict__ in, float* __restrict__ out, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  v = 0.0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

// out[0] += sum, out[1] += sum of squares over the w x h window at (x0, y0)
// of a pitched image, in double (nppiMean_32f_C1R / nppiMean_StdDev_32f_C1R).
__global__ void k_window_stats(const float* __restrict__ img, size_t pitchE, int x0, int y0, int w, int h,
                               double* __restrict__ out) {
  const long n = (long)w * h;
  double s = 0.0, q = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double v = img[(size_t)(y0 + i / w) * pitchE + x0 + i % w];
    s += v;
    q += v * v;
  }
  s = block_sum(s);
  q = block_sum(q);
  if (threadIdx.x == 0) {
    atomicAdd(out, s);
    atomicAdd(out + 1, q);
  }
}

// nppiCompareC_32f_C1R(> threshold) + nppiSum_8u_C1R + nppiSet_32f_C1MR:
// pixels above the threshold become `value`; out[0] += their count.
__global__ void k_bad_pixels(float* __restrict__ img, long n, float threshold, float value, double* __restrict__ out) {
  double c = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    if (img[i] > threshold) {
      img[i] = value;
      c += 1.0;
    }
  }
  c = block_sum(c);
  if (threadIdx.x == 0 && c > 0.0) atomicAdd(out, c);
}

// nppiDivC_32f_C1R on the centred W x H window of the square:
// out = sq[window] / div.
__global__ void k_window_div(const float* __restrict__ sq, size_t shift, int maxsize, int pw, int ph, float div,
                             float* __restrict__ out) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= pw || y >= ph) return;
  out[(size_t)y * pw + x] = sq[shift + (size_t)y * maxsize + x] / div;
}

// nppiSubC_32f_C1R then nppiDivC_32f_C1IR(-std): out = (in - mean) / (-std).
__global__ void k_normalize(const float* __restrict__ in, float* __restrict__ out, long n, float mean, float std_) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    out[i] = (in[i] - mean) / (-std_);
}

// ----------------------------------------------------------------- launchers
static inline dim3 grid2(int w, int h, dim3 b) { return dim3((w + b.x - 1) / b.x, (h + b.y - 1) / b.y); }

cudaError_t launch_compare(int pw, int ph, size_t pitchE, const float* real, float* virt, const float* dist,
                           float realLength, float4 cut, float4 dim, float scale, cudaStream_t st) {
  dim3 b(32, 8);
  k_compare<<<grid2(pw, ph, b), b, 0, st>>>(pw, ph, pitchE, real, virt, dist, realLength, cut, dim, scale); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_crop_border(int pw, int ph, size_t pitchE, float* img, float2 cut, float2 dim, const int* p,
                               cudaStream_t st) {
  dim3 b(32, 8);
  k_crop_border<<<grid2(pw, ph, b), b, 0, st>>>(pw, ph, pitchE, img, cut, dim, make_int2(p[0], p[1]),
                                                 make_int2(p[2], p[3]), make_int2(p[4], p[5]), make_int2(p[6], p[7])); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_make_square(int pw, int ph, size_t strideE, const float* in, int maxsize, float* out, int bx,
                               int by, int mirrorY, int fillZero, cudaStream_t st) {
  dim3 b(32, 8);
  k_make_square<<<grid2(maxsize, maxsize, b), b, 0, st>>>(pw, ph, maxsize, strideE, in, out, bx, by, mirrorY, fillZero); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_crop_to_square(int pw, int ph, size_t pitchE, float* img, int apply_crop, float2 cut, float2 dim,
                                  const int* p, int maxsize, float* sq, int bx, int by, cudaStream_t st) {
  dim3 b(32, 8);
  k_crop_to_square<<<grid2(maxsize, maxsize, b), b, 0, st>>>(pw, ph, pitchE, img, apply_crop, cut, dim,
                                                            make_int2(p[0], p[1]), make_int2(p[2], p[3]),
                                                            make_int2(p[4], p[5]), make_int2(p[6], p[7]), maxsize, sq,
                                                            bx, by); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_square_to_image(const float* sq, int maxsize, size_t shift, float inv_norm, int pw, int ph,
                                   size_t pitchE, float* out, float* accum, int apply_crop, float2 cut, float2 dim,
                                   const int* p, cudaStream_t st, int transpose_out) {
  dim3 b(32, 8);
  k_square_to_image<<<grid2(pw, ph, b), b, 0, st>>>(sq, maxsize, shift, inv_norm, pw, ph, pitchE, out, accum,
                                                    apply_crop, cut, dim, make_int2(p[0], p[1]), make_int2(p[2], p[3]),
                                                    make_int2(p[4], p[5]), make_int2(p[6], p[7]), transpose_out); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

// k_square_to_image over `count` squares (stride maxsize^2) into `count`
// images (stride out_stride), one launch per 65535 squares.
cudaError_t launch_square_to_image_batch(const float* sq, int count, int maxsize, size_t shift, float inv_norm, int pw,
                                         int ph, size_t pitchE, float* out, size_t out_stride, int transpose_out,
                                         cudaStream_t st) {
  dim3 b(32, 8);
  for (int c0 = 0; c0 < count; c0 += 65535) {
    dim3 g = grid2(pw, ph, b);
    g.z = (unsigned)(count - c0 < 65535 ? count - c0 : 65535);
    k_square_to_image_batch<<<g, b, 0, st>>>(sq + (size_t)c0 * maxsize * maxsize, (size_t)maxsize * maxsize, maxsize,
                                              shift, inv_norm, pw, ph, pitchE, out + (size_t)c0 * out_stride,
                                              out_stride, transpose_out); ESB_COUNT_LAUNCH();
  }
  return cudaGetLastError();
}

cudaError_t launch_crop_to_square_batch(int pw, int ph, float* images, size_t img_stride, int count, int apply_crop,
                                        int seq_crop, float2 cut, float2 dim, const int* p, int maxsize, float* sq,
                                        size_t sq_stride, int bx, int by, cudaStream_t st) {
  dim3 b(32, 8);
  dim3 g = grid2(maxsize, maxsize, b);
  g.z = seq_crop ? 1 : (unsigned)(count < 65535 ? count : 65535);
  k_crop_to_square_batch<<<g, b, 0, st>>>(pw, ph, images, img_stride, count, apply_crop, seq_crop, cut, dim,
                                          make_int2(p[0], p[1]), make_int2(p[2], p[3]), make_int2(p[4], p[5]),
                                          make_int2(p[6], p[7]), maxsize, sq, sq_stride, bx, by);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}


cudaError_t launch_square_to_image_many(const float* sq, size_t sq_stride, int count, int maxsize, size_t shift,
                                        float inv_norm, int pw, int ph, float* out, size_t out_stride, float* accum,
                                        int apply_crop, float2 cut, float2 dim, const int* p, int transpose_out,
                                        cudaStream_t st) {
  dim3 b(32, 8);
  k_square_to_image_many<<<grid2(pw, ph, b), b, 0, st>>>(sq, sq_stride, count, maxsize, shift, inv_norm, pw, ph, out,
                                                         out_stride, accum, apply_crop, cut, dim,
                                                         make_int2(p[0], p[1]), make_int2(p[2], p[3]),
                                                         make_int2(p[4], p[5]), make_int2(p[6], p[7]), transpose_out);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_transpose(const float* in, int w, int h, size_t pitchE, float* out, cudaStream_t st) {
  dim3 b(32, 8), g((w + 31) / 32, (h + 31) / 32);
  k_transpose<<<g, b, 0, st>>>(in, w, h, pitchE, out); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

static inline int grid1(long n) {
  long b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

cudaError_t launch_convert_input(const void* in, int type, long n, float* out, cudaStream_t st) {
  switch (type) {
    case ESB_PIX_S16: k_convert_input<int16_t><<<grid1(n), 256, 0, st>>>((const int16_t*)in, out, n); break;
    case ESB_PIX_U16: k_convert_input<uint16_t><<<grid1(n), 256, 0, st>>>((const uint16_t*)in, out, n); break;
    case ESB_PIX_S32: k_convert_input<int32_t><<<grid1(n), 256, 0, st>>>((const int32_t*)in, out, n); break;
    case ESB_PIX_U32: k_convert_input<uint32_t><<<grid1(n), 256, 0, st>>>((const uint32_t*)in, out, n); break;
    default: k_convert_input<float><<<grid1(n), 256, 0, st>>>((const float*)in, out, n); break;
  }
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_window_stats(const float* img, size_t pitchE, int x0, int y0, int w, int h, double* out,
                                cudaStream_t st) {
  k_window_stats<<<grid1((long)w * h), 256, 0, st>>>(img, pitchE, x0, y0, w, h, out);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_bad_pixels(float* img, long n, float threshold, float value, double* out, cudaStream_t st) {
  k_bad_pixels<<<grid1(n), 256, 0, st>>>(img, n, threshold, value, out);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_window_div(const float* sq, size_t shift, int maxsize, int pw, int ph, float div, float* out,
                              cudaStream_t st) {
  dim3 b(32, 8);
  k_window_div<<<grid2(pw, ph, b), b, 0, st>>>(sq, shift, maxsize, pw, ph, div, out);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_normalize(const float* in, float* out, long n, float mean, float std_, cudaStream_t st) {
  k_normalize<<<grid1(n), 256, 0, st>>>(in, out, n, mean, std_);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}




cudaError_t launch_wbp_weighting(float* spec, int n, float psi_deg, int fm, cudaStream_t st) {
  dim3 b(32, 8);
  float a = -psi_deg / 180.0f * 3.14159265358979323846f;
  k_wbp_weighting<<<grid2(n / 2 + 1, n, b), b, 0, st>>>((float2*)spec, n, (float)sin((double)a), (float)cos((double)a), fm); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_fourier_filter(float* spec, int n, float lp, float hp, float lps, float hps, cudaStream_t st) {
  dim3 b(32, 8);
  k_fourier_filter<<<grid2(n / 2 + 1, n, b), b, 0, st>>>((float2*)spec, n, lp, hp, lps, hps); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_dose_weighting(float* spec, int n, float dose, float pixelsize, cudaStream_t st) {
  dim3 b(32, 8);
  k_dose_weighting<<<grid2(n / 2 + 1, n, b), b, 0, st>>>((float2*)spec, n, dose, pixelsize); ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_convert(const void* vol, int vt, long n, float* out, float sign, cudaStream_t st) {
  int blocks = (int)((n + 255) / 256 < 148 * 32 ? (n + 255) / 256 : 148 * 32);
  if (blocks < 1) blocks = 1;
  switch (vt) {
    case ESB_VOXEL_F32: k_convert<ESB_VOXEL_F32><<<blocks, 256, 0, st>>>(vol, n, out, sign); ESB_COUNT_LAUNCH(); break;
    case ESB_VOXEL_F16: k_convert<ESB_VOXEL_F16><<<blocks, 256, 0, st>>>(vol, n, out, sign); ESB_COUNT_LAUNCH(); break;
    default: k_convert<ESB_VOXEL_BF16><<<blocks, 256, 0, st>>>(vol, n, out, sign); ESB_COUNT_LAUNCH(); break;
  }
  return cudaGetLastError();
}

cudaError_t launch_store(const float* in, long n, void* vol, int vt, cudaStream_t st) {
  int blocks = (int)((n + 255) / 256 < 148 * 32 ? (n + 255) / 256 : 148 * 32);
  if (blocks < 1) blocks = 1;
  switch (vt) {
    case ESB_VOXEL_F32: k_store<ESB_VOXEL_F32><<<blocks, 256, 0, st>>>(in, n, vol); ESB_COUNT_LAUNCH(); break;
    case ESB_VOXEL_F16: k_store<ESB_VOXEL_F16><<<blocks, 256, 0, st>>>(in, n, vol); ESB_COUNT_LAUNCH(); break;
    default: k_store<ESB_VOXEL_BF16><<<blocks, 256, 0, st>>>(in, n, vol); ESB_COUNT_LAUNCH(); break;
  }
  return cudaGetLastError();
}

}  // namespace esb
