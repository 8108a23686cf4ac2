// Grid loop and shared definitions of the host-compiled reference kernels
// (TEST INFRASTRUCTURE; see esb_ref_shim.h).
#pragma once

#include <atomic>
#include <thread>
#include <vector>

#include "esb_ref_shim.h"

// Same layout as the oracle's OrcGeom (oracle/esb_oracle.cpp): the values the
// reference's SetConstantValues writes into the kernels' constant memory.
struct RefGeom {
  float det[3], u[3], v[3], n[3];
  float detMat[16];
  float bbMin[3], bbMax[3], bbRcp[3], dim[3], vs[3];
  float zShift;
  int dimXQuarter;
  float aniso[9], anisoInv[9];
};

inline float3 ref_f3(const float* a) { return make_float3(a[0], a[1], a[2]); }

// Runs body() once per thread of a grid x block launch, blocks spread over
// nthreads host threads; each host thread owns its blockIdx/threadIdx.
template <class F>
void esb_grid(dim3 grid, dim3 block, int nthreads, F body) {
  const long nblocks = (long)grid.x * grid.y * grid.z;
  std::atomic<long> next(0);
  auto worker = [&]() {
    for (;;) {
      long b = next.fetch_add(1);
      if (b >= nblocks) break;
      gridDim = grid;
      blockDim = block;
      blockIdx = make_uint3((unsigned)(b % grid.x), (unsigned)((b / grid.x) % grid.y),
                            (unsigned)(b / ((long)grid.x * grid.y)));
      for (unsigned z = 0; z < block.z; ++z)
        for (unsigned y = 0; y < block.y; ++y)
          for (unsigned x = 0; x < block.x; ++x) {
            threadIdx = make_uint3(x, y, z);
            body();
          }
    }
  };
  int nt = nthreads < 1 ? 1 : nthreads;
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
}

// Kernel constants of DeviceVariables.cuh:13-34 as SetConstantValues writes
// them (Kernels.cpp:949-1101); NS is the namespace holding one kernel file.
#define ESB_REF_SET_CONSTANTS(NS, g, for_bp)                                   \
  do {                                                                         \
    NS::c_projNorm = ref_f3((g).n);                                            \
    NS::c_detektor = ref_f3((g).det);                                          \
    NS::c_uPitch = ref_f3((g).u);                                              \
    NS::c_vPitch = ref_f3((g).v);                                              \
    NS::c_volumeBBoxRcp = ref_f3((g).bbRcp);                                   \
    NS::c_bBoxMin = ref_f3((g).bbMin);                                         \
    NS::c_bBoxMax = ref_f3((g).bbMax);                                         \
    NS::c_volumeDim = ref_f3((g).dim);                                         \
    NS::c_voxelSize = ref_f3((g).vs);                                          \
    NS::c_zShiftForPartialVolume = (for_bp) ? (g).zShift : 0.0f;               \
    NS::c_volumeDim_x_quarter = (g).dimXQuarter;                               \
    memcpy(&NS::c_DetectorMatrix, (g).detMat, sizeof(float) * 16);             \
    memcpy(&NS::c_magAniso, (g).aniso, sizeof(float) * 9);                     \
    memcpy(&NS::c_magAnisoInv, (g).anisoInv, sizeof(float) * 9);               \
  } while (0)

// The reference's cutil_math.h adds one-argument overloads of make_float2
// and friends. Inside a kernel file's namespace those would hide the shim's
// constructors, so each namespace re-exports them first.
#define ESB_REF_USING                                                                                     \
  using ::make_float2; using ::make_float3; using ::make_float4; using ::make_int2; using ::make_int3;    \
  using ::make_int4; using ::make_uint2; using ::make_uint3; using ::make_uint4; using ::max; using ::min; \
  using ::fminf; using ::fmaxf; using ::floorf; using ::fmodf; using ::fabs; using ::abs; using ::rsqrtf;
