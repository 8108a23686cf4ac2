// Batched sub-volume weighted back-projection (EmSARTSubVolumes).
//
// The reference reconstructs particles in batches. For every tilt it binds
// each particle's 3-D array to the surface reference and launches the
// back-projection once per particle (Reconstructor.cpp:893-914), and once per
// particle per defocus slab with CTF (:975-1033). At 2000 particles x 61
// tilts that is 122k mostly small launches, most of which cannot fill the
// GPU (a 48^3 box is 216 blocks of 128 quads).
//
// Here one persistent launch processes every particle, of mixed box sizes.
// The work list holds blocks of 128 consecutive voxel quads of one particle.
// The launch also loops over all tilts: each thread keeps its quad in
// registers, adds the tilts in list order and writes the quad once. Without
// CTF it reads the tilts' images. With CTF the slab images of all tilts do
// not fit the device (61 tilts x ~25 slabs x 4096^2), so after each tilt's
// CTF chain a gather copies, for every particle, the patch of the slab images
// its quads read (the slabs its depth range meets, the rectangle of its
// box's shadow with a margin; texels beyond the image edge stored as their
// clamped values) into one patch buffer of a few GB; the persistent launch
// then reads each quad's slab from its patch. Reads from a patch equal the
// clamped reads from the slab image, so both give the per-tilt result bit
// for bit. (Pairs whose geometry does not take the single-axis sums, or
// patches beyond the buffer cap, fall back to one launch per tilt.) The per-voxel sums are those of the single-volume fast
// back-projector (esb_bp_core.cuh: the single-axis sums for projections
// without a y component of the beam, the general chords otherwise), added in
// the same order, so batched and per-particle results agree to float
// rounding.
#include <string.h>

#include <cmath>

#include "esb_bp_core.cuh"
#include "esb_subvolume.cuh"

namespace esb {

using namespace bpcore;

namespace {

constexpr int kQuadsPerItem = 128;

struct SubvolWork {
  int particle;
  int quad0;  // first quad of the block within the particle
};

struct SubvolParticle {
  float* box;
  int nqx, ny, nquads;
  int pad;
};

// Kernel constants of one (particle, list position) pair.
struct PairConst {
  KConst k;
  BpGeom g;
  AxisGeom a;  // single-axis sums (axis_sums) when axis != 0
  int axis;
  int active;
};

// AXIS: every pair of the call takes the single-axis sums.
template <bool AXIS>
__global__ void __launch_bounds__(kQuadsPerItem, 5) k_subvol_batch(const SubvolWork* __restrict__ work, int n_work,
                                                                const SubvolParticle* __restrict__ parts,
                                                                const PairConst* __restrict__ pairs, int n_list,
                                                                int t0, int nt, const float* __restrict__ imgs,
                                                                size_t img_stride, SlabTable slabs, int pw, int ph,
                                                                int os, float inv, int linear) {
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    const SubvolWork item = work[w];
    const SubvolParticle P = parts[item.particle];
    const int q = item.quad0 + (int)threadIdx.x;
    if (q >= P.nquads) continue;
    const int qx = q % P.nqx, y = (q / P.nqx) % P.ny, z = q / (P.nqx * P.ny);
    const int x = 4 * qx;
    float4* cell = (float4*)(P.box + ((size_t)z * P.ny + y) * (size_t)(4 * P.nqx) + x);
    float4 v = *cell;
    bool touched = false;
#pragma unroll 1
    for (int t = t0; t < t0 + nt; ++t) {
      const PairConst& pc = pairs[(size_t)item.particle * n_list + t];
      if (!pc.active) continue;
      float depth;
      int pbx, pby, pbz, pbw;
      if (AXIS && !pc.a.clips) {  // the rectangle from its affine form (macro_rect)
        depth = macro_depth(pc.k, x, y, z);
        macro_rect(pc.a, x, y, z, pw, ph, pbx, pby, pbz, pbw);
      } else {
        macro_footprint(pc.k, x, y, z, pw, ph, depth, pbx, pby, pbz, pbw);
      }
      const float* img;
      if (slabs.count > 0) {
        if (!(depth >= slabs.bound[0] && depth < slabs.bound[slabs.count])) continue;
        int s = 0;
        while (s + 1 < slabs.count && depth >= slabs.bound[s + 1]) ++s;
        img = imgs + (size_t)s * img_stride;
      } else {
        if (!(depth >= 0.0f && depth < 9999999999999.0f)) continue;
        img = imgs + (size_t)(t - t0) * img_stride;
      }
      float acc[4], dacc[4];
      if (AXIS) {
        const AxisGeom& ag = pc.a;
        const float cy = pc.k.bbMin.y + ((float)y + 0.5f) * pc.k.vs.y;
        const float cz = pc.k.bbMin.z + ((float)z + 0.5f) * pc.k.vs.z;
        const float uyz = ag.U.y * cy + ag.U.z * cz + ag.U0, vyz = ag.V.y * cy + ag.V.z * cz + ag.V0;
        const bool lin = linear != 0;
        const bool interior = !lin || (pbx >= 1 && pbz >= 1);
        auto read = [&](int mu, int mv) -> float {
          const float px = ((float)mu + 0.5f) * inv, py = ((float)mv + 0.5f) * inv;
          return interior ? sample_interior(img, (size_t)ph, 1, px, py, lin)
                          : sample_image(img, pw, ph, (size_t)pw, px, py, lin, true);
        };
        const bool patch = os == 2 && lin && interior;
        const float cx0 = pc.k.bbMin.x + ((float)x + 0.5f) * pc.k.vs.x;
        const RowAnchor anchor(ag, y, ag.U.x * cx0 + uyz, ag.V.x * cx0 + vyz, (float)os);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float cx = pc.k.bbMin.x + ((float)(x + i) + 0.5f) * pc.k.vs.x;
          const float uc = ag.U.x * cx + uyz, vc = ag.V.x * cx + vyz;
          if (!(patch && axis_sums_os2(ag, uc, vc, inv * ag.wv, anchor, pbx * 2, pby * 2 - 1, pbz * 2,
                                       pbw * 2 - 1, img, (size_t)ph, 1, pw, ph, acc[i], dacc[i])))
            axis_sums(ag, uc, vc, (float)os, inv, inv * ag.wv, anchor, pbx * os, pby * os - 1, pbz * os,
                            pbw * os - 1, read, acc[i], dacc[i]);
        }
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          voxel_sums(pc.k, pc.g, img, pw, ph, (size_t)pw, os, inv, linear != 0, true, x + i, y, z, pbx, pby, pbz,
                     pbw, acc[i], dacc[i]);
      }
      // lambda = 1 (weighted back-projection): v += 1 * acc / dacc
      if (dacc[0] > 0.f) v.x += 1.0f * acc[0] / dacc[0];
      if (dacc[1] > 0.f) v.y += 1.0f * acc[1] / dacc[1];
      if (dacc[2] > 0.f) v.z += 1.0f * acc[2] / dacc[2];
      if (dacc[3] > 0.f) v.w += 1.0f * acc[3] / dacc[3];
      touched = true;
    }
    if (touched) *cell = v;
  }
}

// One (particle, list position) pair's patches: ns slab patches of pw x ph
// texels ([x][y], ph floats per column), patch texel (i, j) = slab image
// texel (clamp(ox + i), clamp(oy + j)).
struct PatchInfo {
  long long off;  // first float in the patch buffer
  int ox, oy;
  int pw, ph;
  int s0, ns;     // slabs s0 .. s0 + ns - 1 (ns = 0: no quad of the pair in a slab)
};
static_assert(sizeof(PatchInfo) == 32, "PatchInfo layout");

__global__ void __launch_bounds__(256) k_patch_gather(const PatchInfo* __restrict__ info, int n_particles, int n_list,
                                                      int t, const float* __restrict__ imgs, size_t img_stride,
                                                      int pw, int ph, float* __restrict__ patches) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  for (int p = blockIdx.x; p < n_particles; p += gridDim.x) {
    const PatchInfo pi = info[(size_t)p * n_list + t];
    const int cols = pi.ns * pi.pw;
    for (int col = warp; col < cols; col += nwarps) {
      const int sl = col / pi.pw, i = col - sl * pi.pw;
      const int gx = min(max(pi.ox + i, 0), pw - 1);
      const float* src = imgs + (size_t)(pi.s0 + sl) * img_stride + (size_t)gx * ph;
      float* dst = patches + pi.off + (long long)col * pi.ph;
      for (int j = lane; j < pi.ph; j += 32) dst[j] = __ldg(src + min(max(pi.oy + j, 0), ph - 1));
    }
  }
}

// k_subvol_batch over all list positions with CTF, each quad reading its
// slab from the pair's patch (single-axis sums only). Samples outside the
// planned patch (none, by the plan's margins) are counted in *misses and
// skipped.
__global__ void __launch_bounds__(kQuadsPerItem, 5) k_subvol_patches(
    const SubvolWork* __restrict__ work, int n_work, const SubvolParticle* __restrict__ parts,
    const PairConst* __restrict__ pairs, const PatchInfo* __restrict__ info, const SlabTable* __restrict__ slabs,
    int n_list, const float* __restrict__ patches, int pw, int ph, int os, float inv, int linear,
    unsigned long long* __restrict__ misses) {
  for (int w = blockIdx.x; w < n_work; w += gridDim.x) {
    const SubvolWork item = work[w];
    const SubvolParticle P = parts[item.particle];
    const int q = item.quad0 + (int)threadIdx.x;
    if (q >= P.nquads) continue;
    const int qx = q % P.nqx, y = (q / P.nqx) % P.ny, z = q / (P.nqx * P.ny);
    const int x = 4 * qx;
    float4* cell = (float4*)(P.box + ((size_t)z * P.ny + y) * (size_t)(4 * P.nqx) + x);
    float4 v = *cell;
    bool touched = false;
#pragma unroll 1
    for (int t = 0; t < n_list; ++t) {
      const PairConst& pc = pairs[(size_t)item.particle * n_list + t];
      if (!pc.active) continue;
      float depth;
      int pbx, pby, pbz, pbw;
      if (!pc.a.clips) {
        depth = macro_depth(pc.k, x, y, z);
        macro_rect(pc.a, x, y, z, pw, ph, pbx, pby, pbz, pbw);
      } else {
        macro_footprint(pc.k, x, y, z, pw, ph, depth, pbx, pby, pbz, pbw);
      }
      const SlabTable& T = slabs[t];
      const int nsl = T.count;
      if (!(depth >= T.bound[0] && depth < T.bound[nsl])) continue;
      int s = 0;
      while (s + 1 < nsl && depth >= T.bound[s + 1]) ++s;
      const PatchInfo pi = info[(size_t)item.particle * n_list + t];
      if (s < pi.s0 || s >= pi.s0 + pi.ns || pbx < pi.ox + 1 || pby > pi.ox + pi.pw - 2 || pbz < pi.oy + 1 ||
          pbw > pi.oy + pi.ph - 2) {
        atomicAdd(misses, 1ull);
        continue;
      }
      // the patch addressed in detector texels: texel (gx, gy) at img + gx * sx + gy
      const size_t sx = (size_t)pi.ph;
      const float* img =
          patches + (pi.off + (long long)(s - pi.s0) * pi.pw * pi.ph - (long long)pi.ox * pi.ph - pi.oy);
      const AxisGeom& ag = pc.a;
      const float cy = pc.k.bbMin.y + ((float)y + 0.5f) * pc.k.vs.y;
      const float cz = pc.k.bbMin.z + ((float)z + 0.5f) * pc.k.vs.z;
      const float uyz = ag.U.y * cy + ag.U.z * cz + ag.U0, vyz = ag.V.y * cy + ag.V.z * cz + ag.V0;
      const bool lin = linear != 0;
      const bool interior = !lin || (pbx >= 1 && pbz >= 1);
      auto read = [&](int mu, int mv) -> float {
        const float px = ((float)mu + 0.5f) * inv, py = ((float)mv + 0.5f) * inv;
        return sample_interior(img, sx, 1, px, py, lin);
      };
      const bool patch = os == 2 && lin && interior;
      const float cx0 = pc.k.bbMin.x + ((float)x + 0.5f) * pc.k.vs.x;
      const RowAnchor anchor(ag, y, ag.U.x * cx0 + uyz, ag.V.x * cx0 + vyz, (float)os);
      float acc[4], dacc[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float cx = pc.k.bbMin.x + ((float)(x + i) + 0.5f) * pc.k.vs.x;
        const float uc = ag.U.x * cx + uyz, vc = ag.V.x * cx + vyz;
        if (!(patch && axis_sums_os2(ag, uc, vc, inv * ag.wv, anchor, pbx * 2, pby * 2 - 1, pbz * 2, pbw * 2 - 1,
                                     img, sx, 1, pw, ph, acc[i], dacc[i])))
          axis_sums(ag, uc, vc, (float)os, inv, inv * ag.wv, anchor, pbx * os, pby * os - 1, pbz * os,
                    pbw * os - 1, read, acc[i], dacc[i]);
      }
      if (dacc[0] > 0.f) v.x += 1.0f * acc[0] / dacc[0];
      if (dacc[1] > 0.f) v.y += 1.0f * acc[1] / dacc[1];
      if (dacc[2] > 0.f) v.z += 1.0f * acc[2] / dacc[2];
      if (dacc[3] > 0.f) v.w += 1.0f * acc[3] / dacc[3];
      touched = true;
    }
    if (touched) *cell = v;
  }
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

}  // namespace

bool subvol_batchable(int n_particles, float* const* boxes, const KConst* consts, int n_list) {
  for (int p = 0; p < n_particles; ++p) {
    const KConst& k = consts[(size_t)p * n_list];
    if (((uintptr_t)boxes[p] & 15) != 0) return false;
    if ((int)k.dim.x != 4 * k.dimXQuarter) return false;
  }
  return true;
}

cudaError_t subvol_batch_build(SubvolBatch& b, int n_particles, float* const* boxes, const KConst* consts,
                               const unsigned char* active, int n_list, int os, cudaStream_t st) {
  std::vector<SubvolWork> work;
  std::vector<SubvolParticle> parts((size_t)n_particles);
  for (int p = 0; p < n_particles; ++p) {
    const KConst& k = consts[(size_t)p * n_list];
    SubvolParticle& P = parts[p];
    P.box = boxes[p];
    P.nqx = k.dimXQuarter;
    P.ny = (int)k.dim.y;
    P.nquads = P.nqx * P.ny * (int)k.dim.z;
    P.pad = 0;
    bool any = false;
    for (int t = 0; t < n_list && !any; ++t) any = !active || active[(size_t)p * n_list + t];
    if (!any) continue;
    for (int q0 = 0; q0 < P.nquads; q0 += kQuadsPerItem) work.push_back(SubvolWork{p, q0});
  }
  const size_t n_pairs = (size_t)n_particles * n_list;
  b.off_parts = align256(work.size() * sizeof(SubvolWork));
  b.off_pairs = b.off_parts + align256(parts.size() * sizeof(SubvolParticle));
  const size_t bytes = b.off_pairs + n_pairs * sizeof(PairConst);
  cudaError_t e;
  // the staging buffer is pinned (the copy runs asynchronously): wait for
  // the previous call's copy before writing it again
  if (b.copied && (e = cudaEventSynchronize(b.copied)) != cudaSuccess) return e;
  if (!b.copied && (e = cudaEventCreateWithFlags(&b.copied, cudaEventDisableTiming)) != cudaSuccess) return e;
  if (bytes > b.host_cap) {
    cudaFreeHost(b.host);
    b.host = nullptr;
    b.host_cap = 0;
    if ((e = cudaHostAlloc((void**)&b.host, bytes, cudaHostAllocDefault)) != cudaSuccess) return e;
    b.host_cap = bytes;
  }
  memcpy(b.host, work.data(), work.size() * sizeof(SubvolWork));
  memcpy(b.host + b.off_parts, parts.data(), parts.size() * sizeof(SubvolParticle));
  PairConst* pc = (PairConst*)(b.host + b.off_pairs);
  // per-pair constants on the host cores (the tables of 2000 particles x 61
  // tilts are 1.2e5 pairs)
  host_parallel_for((long)n_pairs, [&](long i) {
    PairConst& q = pc[i];
    q.k = consts[i];
    q.g = make_geom(consts[i], os);
    q.axis = axis_eligible(consts[i], q.g) ? 1 : 0;
    if (q.axis) q.a = make_axis_geom(consts[i], q.g, os);
    q.active = !active || active[i];
  });
  b.all_axis = 1;
  for (size_t i = 0; i < n_pairs; ++i)
    if (!pc[i].axis) b.all_axis = 0;
  if (bytes > b.cap) {
    e = cudaStreamSynchronize(st);  // the old tables may be in use
    if (e != cudaSuccess) return e;
    cudaFree(b.dev);
    b.dev = nullptr;
    b.cap = 0;
    if ((e = cudaMalloc(&b.dev, bytes)) != cudaSuccess) return e;
    b.cap = bytes;
  }
  b.n_work = (int)work.size();
  b.n_list = n_list;
  b.n_particles = n_particles;
  if ((e = cudaMemcpyAsync(b.dev, b.host, bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  return cudaEventRecord(b.copied, st);
}

cudaError_t subvol_batch_launch(const SubvolBatch& b, int t0, int nt, const float* imgs, size_t img_stride,
                                const SlabTable& slabs, int pw, int ph, int os, int linear, cudaStream_t st) {
  if (b.n_work <= 0 || nt <= 0) return cudaSuccess;
  int dev = 0, n_sm = 0, per_sm = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
           &per_sm, b.all_axis ? k_subvol_batch<true> : k_subvol_batch<false>, kQuadsPerItem, 0)) != cudaSuccess)
    return e;
  // persistent grid: every resident block slot of every SM, looping over the
  // work list
  long blocks = (long)n_sm * (per_sm > 0 ? per_sm : 1);
  if (blocks > b.n_work) blocks = b.n_work;
  const char* base = (const char*)b.dev;
  auto kern = b.all_axis ? k_subvol_batch<true> : k_subvol_batch<false>;
  kern<<<(unsigned)blocks, kQuadsPerItem, 0, st>>>((const SubvolWork*)base, b.n_work,
                                                   (const SubvolParticle*)(base + b.off_parts),
                                                   (const PairConst*)(base + b.off_pairs), b.n_list, t0, nt, imgs,
                                                   img_stride, slabs, pw, ph, os, 1.0f / (float)os, linear);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t subvol_patch_plan(SubvolBatch& b, const SlabTable* slabs, int pw, int ph, size_t max_bytes,
                              cudaStream_t st, bool& ok) {
  ok = false;
  if (!b.all_axis || b.n_work <= 0 || b.n_list <= 0) return cudaSuccess;
  const int np = b.n_particles, nl = b.n_list;
  const SubvolParticle* parts = (const SubvolParticle*)(b.host + b.off_parts);
  const PairConst* pcs = (const PairConst*)(b.host + b.off_pairs);
  std::vector<PatchInfo> info((size_t)np * nl);
  host_parallel_for((long)np * nl, [&](long i) {
    const int p = (int)(i / nl), t = (int)(i % nl);
    PatchInfo& pi = info[i];
    pi = PatchInfo{0, 0, 0, 1, 1, 0, 0};
    const PairConst& q = pcs[i];
    const SubvolParticle& P = parts[p];
    const SlabTable& T = slabs[t];
    if (!q.active || P.nquads <= 0 || T.count <= 0) return;
    const KConst& k = q.k;
    const int nz = P.nquads / (P.nqx * P.ny);
    // depth range of the quads' first corners (macro_depth), and the shadow
    // of the box (x extended by the last quad's 5-voxel macro cell)
    const double n[3] = {k.n.x, k.n.y, k.n.z};
    const double ndet = -(n[0] * k.det.x + n[1] * k.det.y + n[2] * k.det.z);
    const double bmin[3] = {k.bbMin.x, k.bbMin.y, k.bbMin.z}, vs[3] = {k.vs.x, k.vs.y, k.vs.z};
    const double qlast[3] = {4.0 * (P.nqx - 1), (double)(P.ny - 1), (double)(nz - 1)};
    const double ext[3] = {(double)(4 * P.nqx + 1), (double)P.ny, (double)nz};
    const double U[3] = {q.a.U.x, q.a.U.y, q.a.U.z}, V[3] = {q.a.V.x, q.a.V.y, q.a.V.z};
    double dlo = 1e300, dhi = -1e300, tlo = 1e300, thi = -1e300;
    double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
    for (int c = 0; c < 8; ++c) {
      double tq = ndet, u = q.a.U0, v = q.a.V0;
      for (int j = 0; j < 3; ++j) {
        const int hi = (c >> j) & 1;
        tq += n[j] * (bmin[j] + (hi ? qlast[j] : 0.0) * vs[j]);
        const double pj = bmin[j] + (hi ? ext[j] : 0.0) * vs[j];
        u += U[j] * pj;
        v += V[j] * pj;
      }
      tlo = std::min(tlo, tq), thi = std::max(thi, tq);
      umin = std::min(umin, u), umax = std::max(umax, u);
      vmin = std::min(vmin, v), vmax = std::max(vmax, v);
    }
    if (tlo >= 0.0) dlo = tlo, dhi = thi;
    else if (thi <= 0.0) dlo = -thi, dhi = -tlo;
    else dlo = 0.0, dhi = std::max(-tlo, thi);
    const double eps = 1e-2 + 1e-5 * dhi;
    if (dhi + eps < T.bound[0] || dlo - eps >= T.bound[T.count]) return;  // no quad in a slab
    auto slab_of = [&](double d) {
      int s = 0;
      while (s + 1 < T.count && d >= T.bound[s + 1]) ++s;
      return s;
    };
    const int s0 = slab_of(dlo - eps), s1 = slab_of(dhi + eps);
    const int m = 3;  // texels of margin around the shadow
    auto clampi = [](int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); };
    const int bx0 = clampi((int)std::floor(umin) - m, 0, pw - 1), bx1 = clampi((int)std::ceil(umax) + m, 0, pw - 1);
    const int by0 = clampi((int)std::floor(vmin) - m, 0, ph - 1), by1 = clampi((int)std::ceil(vmax) + m, 0, ph - 1);
    pi.ox = bx0 - 1;
    pi.pw = bx1 - bx0 + 3;
    pi.oy = by0 - 1;
    pi.ph = by1 - by0 + 3;
    pi.s0 = s0;
    pi.ns = s1 - s0 + 1;
  });
  size_t total = 0;
  for (PatchInfo& pi : info) {
    pi.off = (long long)total;
    total += (size_t)pi.ns * pi.pw * pi.ph;
  }
  if (total * sizeof(float) > max_bytes) return cudaSuccess;
  cudaError_t e;
  if (total > b.patches_cap) {
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    cudaFree(b.patches);
    b.patches = nullptr;
    b.patches_cap = 0;
    if ((e = cudaMalloc(&b.patches, std::max<size_t>(total, 1) * sizeof(float))) != cudaSuccess) return e;
    b.patches_cap = total;
  }
  b.off_slabs = align256(info.size() * sizeof(PatchInfo));
  b.off_miss = b.off_slabs + align256((size_t)nl * sizeof(SlabTable));
  const size_t bytes = b.off_miss + sizeof(unsigned long long);
  if (bytes > b.pcap) {
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
    cudaFree(b.pdev);
    b.pdev = nullptr;
    b.pcap = 0;
    if ((e = cudaMalloc(&b.pdev, bytes)) != cudaSuccess) return e;
    b.pcap = bytes;
  }
  // pageable source: the copy is staged before cudaMemcpyAsync returns, but
  // a previous call's copy may still read the vector; wait for the stream
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  b.phost.assign(bytes, 0);
  memcpy(b.phost.data(), info.data(), info.size() * sizeof(PatchInfo));
  memcpy(b.phost.data() + b.off_slabs, slabs, (size_t)nl * sizeof(SlabTable));
  if ((e = cudaMemcpyAsync(b.pdev, b.phost.data(), bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
  ok = true;
  return cudaSuccess;
}

cudaError_t subvol_patch_gather(const SubvolBatch& b, int t, const float* imgs, size_t img_stride, int pw, int ph,
                                cudaStream_t st) {
  if (b.n_particles <= 0) return cudaSuccess;
  const unsigned blocks = (unsigned)std::min(b.n_particles, 148 * 8);
  k_patch_gather<<<blocks, 256, 0, st>>>((const PatchInfo*)b.pdev, b.n_particles, b.n_list, t, imgs, img_stride, pw,
                                         ph, b.patches);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t subvol_patch_launch(const SubvolBatch& b, int pw, int ph, int os, int linear, cudaStream_t st) {
  if (b.n_work <= 0) return cudaSuccess;
  int dev = 0, n_sm = 0, per_sm = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_subvol_patches, kQuadsPerItem, 0)) != cudaSuccess)
    return e;
  long blocks = (long)n_sm * (per_sm > 0 ? per_sm : 1);
  if (blocks > b.n_work) blocks = b.n_work;
  const char* base = (const char*)b.dev;
  const char* pbase = (const char*)b.pdev;
  unsigned long long* miss = (unsigned long long*)(pbase + b.off_miss);
  if ((e = cudaMemsetAsync(miss, 0, sizeof(unsigned long long), st)) != cudaSuccess) return e;
  k_subvol_patches<<<(unsigned)blocks, kQuadsPerItem, 0, st>>>(
      (const SubvolWork*)base, b.n_work, (const SubvolParticle*)(base + b.off_parts),
      (const PairConst*)(base + b.off_pairs), (const PatchInfo*)pbase, (const SlabTable*)(pbase + b.off_slabs),
      b.n_list, b.patches, pw, ph, os, 1.0f / (float)os, linear, miss);
  ESB_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t subvol_patch_misses(const SubvolBatch& b, cudaStream_t st, unsigned long long& misses) {
  misses = 0;
  if (!b.pdev) return cudaSuccess;
  cudaError_t e = cudaMemcpyAsync(&misses, (const char*)b.pdev + b.off_miss, sizeof(misses), cudaMemcpyDeviceToHost,
                                  st);
  if (e != cudaSuccess) return e;
  return cudaStreamSynchronize(st);
}

void subvol_batch_free(SubvolBatch& b) {
  cudaFree(b.pdev);
  b.pdev = nullptr;
  b.pcap = 0;
  cudaFree(b.patches);
  b.patches = nullptr;
  b.patches_cap = 0;
  cudaFree(b.dev);
  b.dev = nullptr;
  b.cap = 0;
  if (b.copied) cudaEventSynchronize(b.copied);
  cudaFreeHost(b.host);
  b.host = nullptr;
  b.host_cap = 0;
  if (b.copied) cudaEventDestroy(b.copied);
  b.copied = nullptr;
}

}  // namespace esb
