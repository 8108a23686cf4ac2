// Normalised cross-correlation displacement of EmSartRefine
// (Reconstructor::GetDisplacement, Reconstructor.cpp:1746-1960).
//
// The two N x N squares (residual and model, mirror-padded by makeSquare)
// are centred on their means and correlated through one R2C pair, the
// conjugate product (kernel conjMul, wbpWeighting.cu:244-262) and one C2R.
// The correlation is divided by N^2 sqrt(SumA SumB), its central
// (4 maxShift)^2 region is copied out fft-shifted (the reference's four
// nppiCopy calls), values farther than maxShift from the origin are zeroed
// (kernel maxShift, :266-293) and the arg-max taken. With multi-peak
// detection the local maxima of at least 0.9 of the maximum (kernel
// findPeak, :331-386) are weighted by the inverse of their distance to the
// origin (maxShiftWeighted, :296-327) and the arg-max of that map taken.
//
// The NPP reductions (nppiMean, nppiSqr + nppiSum, nppiMaxIndx) become
// double-precision grid reductions; the arg-max is one 64-bit atomicMax of
// (order-preserving bits of the value, complement of the raster index), so
// ties go to the first pixel in raster order. Arithmetic is IEEE single
// precision without contraction (the file is compiled with --fmad=false).
#include "esb_device.cuh"

namespace esb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double block_sum_d(double v) {
  __shared__ double red[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  v = 0.0;
  if (threadIdx.x < 32) {
    v = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  return v;  // valid in thread 0
}

__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v) {
  __shared__ unsigned long long red[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
    v = u > v ? u : v;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  v = 0ull;
  if (threadIdx.x < 32) {
    v = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : 0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long u = __shfl_xor_sync(0xffffffffu, v, o);
      v = u > v ? u : v;
    }
  }
  return v;  // valid in thread 0
}

// Arg-max key of value v at raster index i: larger values give larger keys,
// equal values the smaller index. NaN takes no part (key 0).
__device__ __forceinline__ unsigned long long argmax_key(float v, unsigned i) {
  if (v != v) return 0ull;
  unsigned u = __float_as_uint(v);
  u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  return ((unsigned long long)u << 32) | (unsigned long long)(0xFFFFFFFFu - i);
}

__device__ __forceinline__ float key_value(unsigned long long k) {
  if (k == 0ull) return __int_as_float(0x7fc00000);  // no value: NaN
  unsigned u = (unsigned)(k >> 32);
  u = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
  return __uint_as_float(u);
}

// Distance of pixel (x, y) of the unshifted correlation to the origin, with
// the reference's fold (maxShift, wbpWeighting.cu:276-286).
__device__ __forceinline__ float origin_dist(int x, int y, int n) {
  float mx = (float)x, my = (float)y;
  if (mx > (float)(n / 2)) mx = (float)n - mx;
  if (my > (float)(n / 2)) my = (float)n - my;
  return sqrtf(mx * mx + my * my);
}

// sums[0] += sum of x (nppiMean_32f_C1R's accumulation).
__global__ void __launch_bounds__(kThreads) k_cc_sum(const float* __restrict__ x, long n, double* __restrict__ sums) {
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) s += x[i];
  s = block_sum_d(s);
  if (threadIdx.x == 0) atomicAdd(sums, s);
}

// x -= (float)mean (nppiSubC_32f_C1IR); sums[1] += sum of the float squares
// (nppiSqr_32f_C1R + nppiSum_32f_C1R).
__global__ void __launch_bounds__(kThreads) k_cc_center(float* __restrict__ x, long n, double* __restrict__ sums) {
  const float m = (float)(sums[0] / (double)n);
  double q = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float v = x[i] - m;
    x[i] = v;
    q += (double)(v * v);
  }
  q = block_sum_d(q);
  if (threadIdx.x == 0) atomicAdd(sums + 1, q);
}

// a = conj(a) * b (conjMul).
__global__ void __launch_bounds__(kThreads) k_cc_conj_mul(float2* __restrict__ a, const float2* __restrict__ b,
                                                          long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float2 p = a[i], q = b[i];
    a[i] = make_float2(p.x * q.x + p.y * q.y, p.x * q.y - p.y * q.x);
  }
}

// Divisor of the correlation: N^2 sqrt(SumA SumB) (nppiDivC_32f_C1IR's
// argument), from the squares' sums of squares at sums[1] and sums[3];
// 1 when sums is NULL.
__device__ __forceinline__ float cc_divisor(const double* sums, int n) {
  if (!sums) return 1.0f;
  return (float)((double)n * (double)n * sqrt(sums[1] * sums[3]));
}

// map[y'][x'] = cc[(y' - 2S) mod N][(x' - 2S) mod N] / divisor over the
// (4S)^2 map (the four nppiCopy_32f_C1R quadrants); 2S <= N.
__global__ void k_cc_map(const float* __restrict__ cc, int n, int s, const double* __restrict__ sums,
                         float* __restrict__ map) {
  const int m = 4 * s;
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= m || y >= m) return;
  const int sx = x < 2 * s ? x + n - 2 * s : x - 2 * s;
  const int sy = y < 2 * s ? y + n - 2 * s : y - 2 * s;
  const float div = cc_divisor(sums, n);
  map[(size_t)y * m + x] = cc[(size_t)sy * n + sx] / div;
}

// cc = cc / divisor, zero beyond maxShift (maxShift), key = arg-max.
__global__ void __launch_bounds__(kThreads) k_cc_finish(float* __restrict__ cc, int n, int s,
                                                        const double* __restrict__ sums,
                                                        unsigned long long* __restrict__ key) {
  const float div = cc_divisor(sums, n);
  const long total = (long)n * n;
  unsigned long long best = 0ull;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % n), y = (int)(i / n);
    float v = cc[i] / div;
    if (origin_dist(x, y, n) > (float)s) v = 0.0f;
    cc[i] = v;
    const unsigned long long k = argmax_key(v, (unsigned)i);
    best = k > best ? k : best;
  }
  best = block_max_u64(best);
  if (threadIdx.x == 0 && best) atomicMax(key, best);
}

// Multi-peak map: 1 at local maxima of img of at least 0.9 x its maximum
// (findPeak with the cyclic neighbours, then nppiSet_32f_C1R(1) and
// nppiSet_32f_C1MR(0) on the non-peaks), divided by the distance to the
// origin + 1e-4 and zero beyond maxShift (maxShiftWeighted); key2 = arg-max.
__global__ void __launch_bounds__(kThreads) k_cc_peaks(const float* __restrict__ img, float* __restrict__ out, int n,
                                                       int s, const unsigned long long* __restrict__ key,
                                                       unsigned long long* __restrict__ key2) {
  const float thr = key_value(*key) * 0.9f;
  const long total = (long)n * n;
  unsigned long long best = 0ull;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int x = (int)(i % n), y = (int)(i / n);
    const int xm = x - 1 < 0 ? n - 1 : x - 1, xp = x + 1 >= n ? 0 : x + 1;
    const int ym = y - 1 < 0 ? n - 1 : y - 1, yp = y + 1 >= n ? 0 : y + 1;
    const float* rM = img + (size_t)ym * n;
    const float* r0 = img + (size_t)y * n;
    const float* rP = img + (size_t)yp * n;
    const float val = r0[x];
    const bool peak = r0[xm] < val && r0[xp] < val && rM[x] < val && rP[x] < val && rM[xm] <= val &&
                      rP[xm] < val && rM[xp] <= val && rP[xp] < val && val >= thr;
    const float d = origin_dist(x, y, n);
    float v = peak ? 1.0f : 0.0f;
    if (d > (float)s) v = 0.0f;
    else v = v / (d + 0.0001f);
    out[i] = v;
    const unsigned long long k = argmax_key(v, (unsigned)i);
    best = k > best ? k : best;
  }
  best = block_max_u64(best);
  if (threadIdx.x == 0 && best) atomicMax(key2, best);
}

inline int grid_for(long n) {
  long g = (n + kThreads - 1) / kThreads;
  return (int)(g < 1 ? 1 : (g > 148 * 8 ? 148 * 8 : g));
}

}  // namespace

cudaError_t launch_cc_center(float* sq, long n, double* sums, cudaStream_t st) {
  k_cc_sum<<<grid_for(n), kThreads, 0, st>>>(sq, n, sums);
  ESB_COUNT_LAUNCH();
  k_cc_center<<<grid_for(n), kThreads, 0, st>>>(sq, n, sums);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_cc_conj_mul(float* a, const float* b, long n_complex, cudaStream_t st) {
  k_cc_conj_mul<<<grid_for(n_complex), kThreads, 0, st>>>((float2*)a, (const float2*)b, n_complex);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_cc_map(const float* cc, int n, int s, const double* sums, float* map, cudaStream_t st) {
  dim3 b(32, 8), g((4 * s + 31) / 32, (4 * s + 7) / 8);
  k_cc_map<<<g, b, 0, st>>>(cc, n, s, sums, map);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_cc_finish(float* cc, int n, int s, const double* sums, unsigned long long* key, cudaStream_t st) {
  k_cc_finish<<<grid_for((long)n * n), kThreads, 0, st>>>(cc, n, s, sums, key);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_cc_peaks(const float* img, float* out, int n, int s, const unsigned long long* key,
                            unsigned long long* key2, cudaStream_t st) {
  k_cc_peaks<<<grid_for((long)n * n), kThreads, 0, st>>>(img, out, n, s, key, key2);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace esb
