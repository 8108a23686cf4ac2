// The z-slab SART of EmSart's MPI runs (EmSart.cpp:579-675 on rank `rank`
// of `world`, Volume.cpp:82-114) through libesb with an NCCL all-reduce: the
// code of INTEGRATION.md's multi-GPU section, compiled here (to an object
// only: running it needs one process per GPU, and the communicator comes
// from the caller's launcher). tests/test_cpp_caller.py compiles it and
// checks that INTEGRATION.md shows this block.
#include <cstdio>

#include <cuda_runtime.h>

// --- begin: z-slab SART with NCCL
#include <nccl.h>
#include "esb.h"

// esb_allreduce_fn: sum `count` floats at `buf` over the ranks, ordered on `stream`
static int nccl_sum(float* buf, size_t count, void* stream, void* user) {
  ncclComm_t comm = (ncclComm_t)user;
  return ncclAllReduce(buf, buf, count, ncclFloat, ncclSum, comm, (cudaStream_t)stream) == ncclSuccess ? 0 : 1;
}
// --- end ---

int zslab_sart(esb_reconstructor* rec, ncclComm_t comm, int rank, int world, const int dims[3],
               const float voxel_size[3], const float volume_shift[3], float* vol_slab_d, const float* projections_d,
               const int* index_list, int proj_count, int iterations, int sirt_count) {
  // --- begin: z-slab SART call
  // rank r of `world`: slab r of the volume, the same projections and index list on every rank
  esb_vol_geom slab;
  esb_volume_geometry(dims, world, rank, voxel_size, volume_shift, &slab);
  int empty = 1;
  if (esb_sart_run_zslab(rec, &slab, vol_slab_d, ESB_VOXEL_F32, projections_d, index_list, proj_count,
                         iterations, sirt_count, &empty, nccl_sum, comm) != ESB_OK)
    fprintf(stderr, "%s\n", esb_last_error());
  // --- end ---
  return empty;
}
