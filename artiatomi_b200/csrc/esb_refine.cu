// Volume rotation of the shift refinement (EmSartRefine's rotated
// references).
//
// RotKernel::operator() launches `rot3d` (wbpWeighting.cu:389-405) over the
// size^3 output: voxel p takes the input at c + R^T (p - c), c = size / 2
// (integer division), read through a 3-D texture with linear filtering and
// clamp addressing at the sample position + 0.5, i.e. trilinear
// interpolation with texel centres at integer coordinates. Here the same
// interpolation runs in FP32 from global memory (the texture unit's 8-bit
// filter weights are not reproduced).
#include "esb_ray_core.cuh"

namespace esb {

namespace {

__global__ void __launch_bounds__(512) k_rot3d(const float* __restrict__ in, float* __restrict__ out, int size,
                                               float3 r0, float3 r1, float3 r2) {
  const int x = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = (int)(blockIdx.y * blockDim.y + threadIdx.y);
  const int z = (int)(blockIdx.z * blockDim.z + threadIdx.z);
  if (x >= size || y >= size || z >= size) return;
  const float c = (float)(size / 2);
  const float vx = (float)x - c, vy = (float)y - c, vz = (float)z - c;
  // rows r0, r1, r2 of R: the sample is c + R^T v
  const float px = c + r0.x * vx + r1.x * vy + r2.x * vz;
  const float py = c + r0.y * vx + r1.y * vy + r2.y * vz;
  const float pz = c + r0.z * vx + r1.z * vy + r2.z * vz;
  const long n = size;
  raycore::Cell<ESB_VOXEL_F32> C{in, size, size, size, n, n * n};
  out[((long)z * n + y) * n + x] = raycore::trilinear<ESB_VOXEL_F32>(C, px, py, pz);
}

}  // namespace

cudaError_t launch_rotate_volume(const float* in, float* out, int size, const float rot[9], cudaStream_t st) {
  dim3 blk(8, 8, 8), grd((size + 7) / 8, (size + 7) / 8, (size + 7) / 8);
  k_rot3d<<<grd, blk, 0, st>>>(in, out, size, make_float3(rot[0], rot[1], rot[2]), make_float3(rot[3], rot[4], rot[5]),
                               make_float3(rot[6], rot[7], rot[8]));
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace esb
