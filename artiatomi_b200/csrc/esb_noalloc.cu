// SART projection update that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host application whose device memory
// is owned by its own allocator and budgeted up front, a process that
// forbids allocations after start-up so that it cannot fail late for lack of
// memory, or a loop that must not pay cudaMalloc's implicit device
// synchronisation. esb_sart_projection_update_noalloc serves them: its two
// scratch images (forward projection and ray lengths, the reconstructor's
// proj_d and dist_d) live in the file-scope array below instead of in buffers
// the reconstructor allocates.
#include <cuda.h>

#include <mutex>

#include "esb_device.cuh"
#include "esb_internal.h"

namespace esb {
cudaError_t launch_march(const KConst& c, const void* vol, int vt, float* proj, float* dist, size_t pitchE, int x0,
                         int y0, int x1, int y1, cudaStream_t st);
cudaError_t launch_travlen(const KConst& c, float* dist, size_t pitchE, int x0, int y0, int x1, int y1, cudaStream_t st);
cudaError_t launch_bp(const KConst& c, void* vol, int vt, const float* img, int pw, int ph, size_t pitchE, float lambda,
                      int os, float distMin, float distMax, int linear, cudaStream_t st);
cudaError_t launch_compare(int pw, int ph, size_t pitchE, const float* real, float* virt, const float* dist,
                           float realLength, float4 cut, float4 dim, float scale, cudaStream_t st);
cudaError_t launch_crop_border(int pw, int ph, size_t pitchE, float* img, float2 cut, float2 dim, const int* p,
                               cudaStream_t st);
cudaError_t launch_project_fast(const KConst& c, const void* vol, int vt, int mode, float* proj, float* dist,
                                size_t pitchE, float tmin, float tmax, int x0, int y0, int x1, int y1,
                                cudaStream_t st, int nw);
cudaError_t launch_bp_fast(const KConst& k, void* vol, int vt, const float* img, int pw, int ph, size_t pitchE,
                           float lambda, int os, float distMin, float distMax, int linear, cudaStream_t st);
}  // namespace esb

using namespace esb;

// Two W x H float images of at most ESB_NOALLOC_MAX_PIXELS pixels each
// (32 MiB). The array stays resident until the process exits on every GPU
// that loads this module of the library (no later than the entry point's
// first call on that GPU).
static __device__ __align__(256) float g_noalloc_scratch[2 * (size_t)ESB_NOALLOC_MAX_PIXELS];

namespace {
std::mutex g_setup_mutex;
// Device address of the array per device ordinal, and the context it was
// looked up in: a device reset (cudaDeviceReset) or a new primary context
// loads the module again, possibly at another address, so the address is
// looked up again when the device's current context changes.
float* g_scratch_of_device[128] = {nullptr};
void* g_context_of_device[128] = {nullptr};
typedef CUresult (*CtxGetCurrent)(CUcontext*);
CtxGetCurrent g_ctx_get_current = nullptr;
bool g_ctx_resolved = false;
}  // namespace

// Device address of the scratch array on the current device. In host code
// g_noalloc_scratch only names a host-side stand-in, so the address is looked
// up (cudaGetSymbolAddress) with the device current, once per device and
// context, and cached. cuCtxGetCurrent is reached through the runtime's
// driver entry point table, so the library does not link libcuda.
static int scratch_on_current_device(float** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(ESB_ERR_CUDA, std::string("esb_sart_projection_update_noalloc: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= 128) return fail(ESB_ERR_UNSUPPORTED, "esb_sart_projection_update_noalloc: device ordinal >= 128");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_ctx_resolved) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = (CtxGetCurrent)fn;
    g_ctx_resolved = true;
  }
  auto current_context = [&]() -> void* {
    CUcontext c = nullptr;
    if (g_ctx_get_current && g_ctx_get_current(&c) == CUDA_SUCCESS) return (void*)c;
    return nullptr;
  };
  if (!g_scratch_of_device[dev] || current_context() != g_context_of_device[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the runtime's context current
    if (e != cudaSuccess || !p)
      return fail(ESB_ERR_CUDA, std::string("esb_sart_projection_update_noalloc: scratch set-up failed: ") +
                                    cudaGetErrorString(e));
    g_scratch_of_device[dev] = (float*)p;
    g_context_of_device[dev] = current_context();
  }
  *out = g_scratch_of_device[dev];
  return ESB_OK;
}

extern "C" int esb_sart_projection_update_noalloc(const esb_recon_config* cfg, const esb_proj_geom* pg,
                                                  const esb_vol_geom* vg, const float mag_aniso[9],
                                                  const float mag_aniso_inv[9], void* vol, int voxel_type,
                                                  const float* real, float sirt_count, int volume_is_empty,
                                                  void* stream) {
  const char* where = "esb_sart_projection_update_noalloc";
  if (!cfg || !pg || !vg || !vol || !real)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": NULL argument");
  if (voxel_type != ESB_VOXEL_F32 && voxel_type != ESB_VOXEL_F16 && voxel_type != ESB_VOXEL_BF16)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": unknown voxel type");
  if (cfg->ctf_mode)
    return fail(ESB_ERR_UNSUPPORTED, std::string(where) + ": CTF mode needs FFT plans, which allocate; use the reconstructor");
  const int W = cfg->proj_x, H = cfg->proj_y;
  if (W <= 0 || H <= 0 || cfg->oversampling < 1 || !(sirt_count > 0))
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": invalid size, oversampling or sirt_count");
  if ((long long)W * H > (long long)ESB_NOALLOC_MAX_PIXELS)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": projection of " + std::to_string(W) + " x " +
                                              std::to_string(H) + " pixels exceeds the scratch limit of " +
                                              std::to_string(ESB_NOALLOC_MAX_PIXELS) + " pixels");
  if (cfg->variant != ESB_VARIANT_FAITHFUL && cfg->variant != ESB_VARIANT_FAST)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": unknown kernel variant");
  float* scratch = nullptr;
  int rc = scratch_on_current_device(&scratch);
  if (rc != ESB_OK) return rc;
  float* proj = scratch;
  float* dist = scratch + (size_t)ESB_NOALLOC_MAX_PIXELS;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t img = (size_t)W * H * sizeof(float);

  esb_constants cf, cb;
  int p[8];
  if ((rc = esb_set_constant_values(pg, vg, mag_aniso, mag_aniso_inv, 0, &cf)) != ESB_OK ||
      (rc = esb_set_constant_values(pg, vg, mag_aniso, mag_aniso_inv, 1, &cb)) != ESB_OK ||
      (rc = esb_compute_hit_points(pg, vg, p)) != ESB_OK)
    return rc;
  const KConst kf = to_kconst(cf), kb = to_kconst(cb);
  const bool fast = cfg->variant == ESB_VARIANT_FAST;
  cudaError_t e;
  // The array keeps the previous call's images: clear both (ResetProjectionsDevice).
  if ((e = cudaMemsetAsync(proj, 0, img, st)) != cudaSuccess || (e = cudaMemsetAsync(dist, 0, img, st)) != cudaSuccess)
    return fail(ESB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  // Forward projection (Reconstructor.cpp:429-438, 465-470)
  // (FAST: the closed-form projector at its default launch shape, 4 warps
  // per block: the reconstructor's launch-shape trials write scratch buffers,
  // and the shape does not change the result)
  if (volume_is_empty)
    e = launch_travlen(kf, dist, W, 0, 0, W, H, st);
  else if (fast)
    e = launch_project_fast(kf, vol, voxel_type, 0, proj, dist, W, 0.f, 0.f, 0, 0, W, H, st, 4);
  else
    e = launch_march(kf, vol, voxel_type, proj, dist, W, 0, 0, W, H, st);
  if (e != cudaSuccess) return fail(ESB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  // Compare (Reconstructor.cpp:1386-1405)
  const float DIST = -10000.0f;
  const float zdir = pg->proj_norm[2];
  const float len = fabsf((DIST - vg->full_bbox_min[2]) / zdir - (DIST - vg->full_bbox_max[2]) / zdir);
  e = launch_compare(W, H, W, real, proj, dist, len, make_float4(cfg->crop[0], cfg->crop[1], cfg->crop[2], cfg->crop[3]),
                     make_float4(cfg->crop_dim[0], cfg->crop_dim[1], cfg->crop_dim[2], cfg->crop_dim[3]),
                     cfg->projection_scale_factor, st);
  if (e != cudaSuccess) return fail(ESB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  // Back-projection of the residual (Reconstructor.cpp:871-887)
  e = launch_crop_border(W, H, W, proj, make_float2(cfg->cut_length[0], cfg->cut_length[1]),
                         make_float2(cfg->dim_length[0], cfg->dim_length[1]), p, st);
  if (e != cudaSuccess) return fail(ESB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  // (FAST: the per-voxel-shadow back-projector reading the residual image
  // directly; the reconstructor first copies it transposed and pre-sampled
  // into buffers it owns, which gives the same sums)
  const float lam = cfg->lambda / sirt_count;
  e = fast ? launch_bp_fast(kb, vol, voxel_type, proj, W, H, W, lam, cfg->oversampling, 0.0f, 9999999999999.0f, 0, st)
           : launch_bp(kb, vol, voxel_type, proj, W, H, W, lam, cfg->oversampling, 0.0f, 9999999999999.0f, 0, st);
  if (e != cudaSuccess) return fail(ESB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
  return ESB_OK;
}
