// Thread-local CUDA indices and IEEE half conversions of the shim
// (TEST INFRASTRUCTURE).
#include <cstring>

#include "esb_ref_shim.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

float esb_half_to_float(unsigned short h) {
  unsigned sign = (h >> 15) & 1u, ex = (h >> 10) & 0x1fu, man = h & 0x3ffu;
  float v;
  if (ex == 0) v = ldexpf((float)man, -24);
  else if (ex == 31) v = man ? NAN : INFINITY;
  else v = ldexpf((float)(man | 0x400u), (int)ex - 25);
  return sign ? -v : v;
}

unsigned short esb_float_to_half_rn(float f) {
  unsigned x;
  memcpy(&x, &f, 4);
  unsigned sign = (x >> 16) & 0x8000u, ax = x & 0x7fffffffu;
  if (ax >= 0x7f800000u) return (unsigned short)(sign | (ax > 0x7f800000u ? 0x7e00u : 0x7c00u));
  if (ax >= 0x477ff000u) return (unsigned short)(sign | 0x7c00u);
  int e = (int)(ax >> 23) - 127;
  if (e < -25) return (unsigned short)sign;
  unsigned m = (ax & 0x7fffffu) | 0x800000u;
  int shift;
  unsigned base;
  if (e >= -14) {
    shift = 13;
    base = (unsigned)(e + 15) << 10;
    m &= 0x7fffffu;
  } else {
    shift = 13 + (-14 - e);
    base = 0;
  }
  unsigned q = m >> shift, rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
  if (rem > half || (rem == half && (q & 1u))) q += 1;
  return (unsigned short)(sign | (base + q));
}
