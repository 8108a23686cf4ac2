// Host-CPU execution shim for the reference's CUDA kernel sources
// (TEST INFRASTRUCTURE).
//
// The reference's device code (src/EmSART/cuda_kernels/*.cu) no longer builds
// with nvcc 12.9: it uses texture and surface references, which CUDA 12
// removed. To run the reference's own kernel source on the same inputs as
// the oracle, oracle/ref_build.py compiles those .cu files, unmodified and
// where they lie, with g++ for the host. The CUDA headers they include are
// replaced by this shim, which emulates:
//  - the execution model: __global__/__device__/__constant__ as plain
//    functions and globals, blockIdx/threadIdx/blockDim/gridDim as
//    thread-local variables set by a grid loop (oracle/ref_shim/ref_launch.h);
//    __shared__ memory is thread-local (the kernels used here do not
//    communicate between threads);
//  - texture objects/references with linear or point filtering, clamp
//    addressing and unnormalised coordinates (texel centres at +0.5), written
//    from the published description of texture filtering (optionally with
//    the 8-bit weight fraction);
//  - surfaces (byte-addressed x) and the half-precision conversions.
// Arithmetic is IEEE host arithmetic without contraction (-ffp-contract=off):
// the reference itself was built with --use_fast_math and FMA contraction,
// so this is the reference's code evaluated in exact IEEE float.
#pragma once

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cmath>
#include <cstdlib>

using std::abs;
using std::atan2;
using std::ceil;
using std::cos;
using std::floor;
using std::sin;
using std::sqrt;

#define __global__
#define __device__
#define __host__
#define __constant__
#define __shared__ thread_local
#define __forceinline__ inline
#define __device_builtin__
#define __align__(n) alignas(n)
#define CUDART_VERSION 12090

typedef unsigned int uint;
typedef unsigned short ushort;

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct alignas(16) float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct alignas(16) int4 { int x, y, z, w; };
struct uint2 { unsigned int x, y; };
struct uint3 { unsigned int x, y, z; };
struct alignas(16) uint4 { unsigned int x, y, z, w; };
struct ushort4 { unsigned short x, y, z, w; };
struct double3 { double x, y, z; };
struct dim3 {
  unsigned int x, y, z;
  dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};

inline float2 make_float2(float x, float y) { return float2{x, y}; }
inline float3 make_float3(float x, float y, float z) { return float3{x, y, z}; }
inline float4 make_float4(float x, float y, float z, float w) { return float4{x, y, z, w}; }
inline int2 make_int2(int x, int y) { return int2{x, y}; }
inline int3 make_int3(int x, int y, int z) { return int3{x, y, z}; }
inline int4 make_int4(int x, int y, int z, int w) { return int4{x, y, z, w}; }
inline uint2 make_uint2(unsigned x, unsigned y) { return uint2{x, y}; }
inline uint3 make_uint3(unsigned x, unsigned y, unsigned z) { return uint3{x, y, z}; }
inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { return uint4{x, y, z, w}; }

// CUDA's device math under the names the kernels call
inline float rsqrtf(float x) { return 1.0f / sqrtf(x); }
inline float __sinf(float x) { return sinf(x); }
inline float __cosf(float x) { return cosf(x); }
inline float __expf(float x) { return expf(x); }
inline float max(float a, float b) { return fmaxf(a, b); }
inline float min(float a, float b) { return fminf(a, b); }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline void __syncthreads() {}

// execution-model indices, set per emulated thread by the grid loop
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

// driver / runtime names used in signatures
typedef unsigned long long CUtexObject;
typedef unsigned long long cudaTextureObject_t;
typedef int CUresult;
enum cudaTextureReadMode { cudaReadModeElementType = 0, cudaReadModeNormalizedFloat = 1 };
#define cudaSurfaceType3D 0x03
typedef float2 cuComplex;
typedef float2 cufftComplex;
typedef float cufftReal;

// ---------------------------------------------------------------- textures
// Software texture with unnormalised coordinates and clamp addressing.
struct EsbSoftTexture {
  const void* data = nullptr;
  int dims = 2;
  int nx = 0, ny = 0, nz = 1;
  size_t pitch_elems = 0;  // row pitch (2-D) in elements
  int half_storage = 0;    // data holds IEEE half values
  int linear = 1;          // linear filtering (else point)
  int weight8 = 0;         // 8-bit fixed-point filter weights
};

float esb_half_to_float(unsigned short h);
unsigned short esb_float_to_half_rn(float f);

inline float esb_tex_fetch(const EsbSoftTexture& t, long x, long y, long z) {
  auto cl = [](long v, int n) { return v < 0 ? 0 : (v > n - 1 ? n - 1 : v); };
  x = cl(x, t.nx);
  y = cl(y, t.ny);
  z = cl(z, t.nz);
  long i = t.dims == 2 ? y * (long)t.pitch_elems + x : (z * (long)t.ny + y) * (long)t.nx + x;
  if (t.half_storage) return esb_half_to_float(((const unsigned short*)t.data)[i]);
  return ((const float*)t.data)[i];
}

inline float esb_weight(float f, int w8) { return w8 ? floorf(f * 256.0f + 0.5f) / 256.0f : f; }

inline long esb_floor_l(float v) {
  if (!(v > -1e18f)) return -1000000000L;  // NaN and -inf clamp to the first texel
  if (v > 1e18f) return 1000000000L;
  return (long)floorf(v);
}

inline float esb_tex2d(const EsbSoftTexture& t, float x, float y) {
  if (!t.linear) return esb_tex_fetch(t, esb_floor_l(x), esb_floor_l(y), 0);
  float xb = x - 0.5f, yb = y - 0.5f;
  long ix = esb_floor_l(xb), iy = esb_floor_l(yb);
  float a = esb_weight(xb - floorf(xb), t.weight8), b = esb_weight(yb - floorf(yb), t.weight8);
  float t00 = esb_tex_fetch(t, ix, iy, 0), t10 = esb_tex_fetch(t, ix + 1, iy, 0);
  float t01 = esb_tex_fetch(t, ix, iy + 1, 0), t11 = esb_tex_fetch(t, ix + 1, iy + 1, 0);
  return (1.0f - b) * ((1.0f - a) * t00 + a * t10) + b * ((1.0f - a) * t01 + a * t11);
}

inline float esb_tex3d(const EsbSoftTexture& t, float x, float y, float z) {
  float xb = x - 0.5f, yb = y - 0.5f, zb = z - 0.5f;
  long ix = esb_floor_l(xb), iy = esb_floor_l(yb), iz = esb_floor_l(zb);
  float a = esb_weight(xb - floorf(xb), t.weight8), b = esb_weight(yb - floorf(yb), t.weight8),
        c = esb_weight(zb - floorf(zb), t.weight8);
  float ia = 1.0f - a, ib = 1.0f - b, ic = 1.0f - c;
  return ic * (ib * (ia * esb_tex_fetch(t, ix, iy, iz) + a * esb_tex_fetch(t, ix + 1, iy, iz)) +
               b * (ia * esb_tex_fetch(t, ix, iy + 1, iz) + a * esb_tex_fetch(t, ix + 1, iy + 1, iz))) +
         c * (ib * (ia * esb_tex_fetch(t, ix, iy, iz + 1) + a * esb_tex_fetch(t, ix + 1, iy, iz + 1)) +
              b * (ia * esb_tex_fetch(t, ix, iy + 1, iz + 1) + a * esb_tex_fetch(t, ix + 1, iy + 1, iz + 1)));
}

// texture references (bound by the launcher before the grid runs)
template <class T, int dim, int mode = 0>
struct texture {
  const EsbSoftTexture* bound = nullptr;
};

template <class T, int dim, int mode>
inline float tex2D(const texture<T, dim, mode>& t, float x, float y) {
  return esb_tex2d(*t.bound, x, y);
}
template <class T, int dim, int mode>
inline float tex3D(const texture<T, dim, mode>& t, float x, float y, float z) {
  return esb_tex3d(*t.bound, x, y, z);
}
// texture objects: the handle is the address of an EsbSoftTexture
template <class T>
inline T tex3D(CUtexObject obj, float x, float y, float z) {
  return (T)esb_tex3d(*(const EsbSoftTexture*)(uintptr_t)obj, x, y, z);
}

// surfaces: x in bytes
template <class T, int kind>
struct surface {
  void* data = nullptr;
  int nx_bytes = 0, ny = 0, nz = 0;
};
template <class V, class S>
inline void surf3Dread(V* out, const S& s, int xbytes, int y, int z) {
  memcpy(out, (const char*)s.data + ((long)z * s.ny + y) * (long)s.nx_bytes + xbytes, sizeof(V));
}
template <class V, class S>
inline void surf3Dwrite(V v, const S& s, int xbytes, int y, int z) {
  memcpy((char*)s.data + ((long)z * s.ny + y) * (long)s.nx_bytes + xbytes, &v, sizeof(V));
}

// IEEE half conversions under CUDA's names (half as its bit pattern)
inline float __half2float(unsigned short h) { return esb_half_to_float(h); }
inline unsigned short __float2half_rn(float f) { return esb_float_to_half_rn(f); }
