// Host interface of the batched sub-volume back-projection (esb_subvolume.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <vector>

#include "esb_device.cuh"

namespace esb {

// f(i) for i in [0, n) on the host cores (chunks of consecutive i per
// thread; serial below `serial_below` items).
template <class F>
void host_parallel_for(long n, F f, long serial_below = 4096) {
  const unsigned hw = std::thread::hardware_concurrency();
  const long nt = std::min<long>(std::max(1u, std::min(hw, 32u)), (n + serial_below - 1) / std::max(serial_below, 1L));
  if (nt <= 1) {
    for (long i = 0; i < n; ++i) f(i);
    return;
  }
  std::vector<std::thread> pool;
  const long chunk = (n + nt - 1) / nt;
  for (long t = 0; t < nt; ++t)
    pool.emplace_back([=, &f]() {
      const long e = std::min(n, (t + 1) * chunk);
      for (long i = t * chunk; i < e; ++i) f(i);
    });
  for (auto& th : pool) th.join();
}

// Device tables of one batched call: the work list (blocks of 128 voxel
// quads of one particle), the particles' boxes and the kernel constants of
// every (particle, list position) pair. Kept by the reconstructor and grown
// on demand, so that repeated calls allocate nothing.
struct SubvolBatch {
  void* dev = nullptr;
  size_t cap = 0;
  unsigned char* host = nullptr;  // pinned staging copy of the tables
  size_t host_cap = 0;
  cudaEvent_t copied = nullptr;   // the last copy of the staging buffer to the device
  size_t off_parts = 0, off_pairs = 0;
  int n_work = 0;
  int n_list = 0;
  int n_particles = 0;
  int all_axis = 0;  // every pair takes the single-axis sums
  // CTF patches (subvol_patch_plan): per pair the part of its tilt's slab
  // images that the box's quads read, gathered into one buffer
  void* pdev = nullptr;  // patch table, slab tables, miss counter
  size_t pcap = 0;
  std::vector<unsigned char> phost;
  size_t off_slabs = 0, off_miss = 0;
  float* patches = nullptr;
  size_t patches_cap = 0;  // floats
};

// True when every box can be updated with aligned float4 accesses (x extent a
// multiple of 4, 16-byte aligned pointer): the batched kernel's layout.
bool subvol_batchable(int n_particles, float* const* boxes, const KConst* consts, int n_list);

// consts/active: [n_particles][n_list] for the list positions of one call;
// active may be NULL (all pairs active).
cudaError_t subvol_batch_build(SubvolBatch& b, int n_particles, float* const* boxes, const KConst* consts,
                               const unsigned char* active, int n_list, int os, cudaStream_t st);

// Adds list positions [t0, t0 + nt) to every box. Without slabs
// (slabs.count == 0) position t reads image imgs + (t - t0) * img_stride;
// with slabs each quad reads the image of its slab. Images are transposed
// ([x][y]).
cudaError_t subvol_batch_launch(const SubvolBatch& b, int t0, int nt, const float* imgs, size_t img_stride,
                                const SlabTable& slabs, int pw, int ph, int os, int linear, cudaStream_t st);

// With CTF: plans, for every (particle, list position) pair, the patch of
// the position's slab images (slabs[t], images transposed, pw x ph) that the
// particle's quads read: the slabs its depth range meets, and the detector
// rectangle of its box's shadow with a margin, out-of-image texels held as
// their clamped values. ok is false (nothing planned) when some pair does
// not take the single-axis sums or the patches exceed max_bytes.
cudaError_t subvol_patch_plan(SubvolBatch& b, const SlabTable* slabs, int pw, int ph, size_t max_bytes,
                              cudaStream_t st, bool& ok);

// Copies list position t's patches out of its slab images.
cudaError_t subvol_patch_gather(const SubvolBatch& b, int t, const float* imgs, size_t img_stride, int pw, int ph,
                                cudaStream_t st);

// Adds every list position to every box in one persistent launch, reading
// the patches.
cudaError_t subvol_patch_launch(const SubvolBatch& b, int pw, int ph, int os, int linear, cudaStream_t st);

// Number of (quad, position) pairs whose samples the plan did not cover
// (skipped, so nothing was read outside the patches); synchronises.
cudaError_t subvol_patch_misses(const SubvolBatch& b, cudaStream_t st, unsigned long long& misses);

void subvol_batch_free(SubvolBatch& b);

}  // namespace esb
