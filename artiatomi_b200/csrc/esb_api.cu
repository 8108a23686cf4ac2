// C ABI of libesb: argument checking and launches of the kernel entry points,
// and the Reconstructor (buffers, cuFFT plans, CTF slab loops, SART driver
// loop, sub-volume back-projection).
#include <cufft.h>
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "esb_device.cuh"
#include "esb_internal.h"
#include "esb_subvolume.cuh"

namespace esb {

cudaError_t launch_march(const KConst& c, const void* vol, int vt, float* proj, float* dist, size_t pitchE, int x0,
                         int y0, int x1, int y1, cudaStream_t st);
cudaError_t launch_slicer(const KConst& c, const void* vol, int vt, float* proj, size_t pitchE, float tmin, float tmax,
                          int x0, int y0, int x1, int y1, cudaStream_t st);
cudaError_t launch_travlen(const KConst& c, float* dist, size_t pitchE, int x0, int y0, int x1, int y1, cudaStream_t st);
cudaError_t launch_bp(const KConst& c, void* vol, int vt, const float* img, int pw, int ph, size_t pitchE, float lambda,
                      int os, float distMin, float distMax, int linear, cudaStream_t st);
cudaError_t launch_project_fast(const KConst& c, const void* vol, int vt, int mode, float* proj, float* dist,
                                size_t pitchE, float tmin, float tmax, int x0, int y0, int x1, int y1, cudaStream_t st, int nw = 4);
cudaError_t launch_bp_fast(const KConst& k, void* vol, int vt, const float* img, int pw, int ph, size_t pitchE,
                           float lambda, int os, float distMin, float distMax, int linear, cudaStream_t st);
cudaError_t launch_bp_fast_slabs(const KConst& k, void* vol, int vt, const float* imgs, size_t img_stride,
                                 const SlabTable& slabs, int pw, int ph, size_t pitchE, float lambda, int os,
                                 float distMin, float distMax, int linear, cudaStream_t st, int transposed,
                                 const float2* ups = nullptr, size_t up_stride = 0, const BpShape* shape = nullptr);
cudaError_t launch_upsample(const KConst& k, const float* imgs, size_t img_stride, int count, int pw, int ph, int os,
                            int linear, float2* up, size_t up_stride, cudaStream_t st);
bool bp_can_upsample(const KConst& k, int os);
bool bp_uses_axis(const KConst& k, int os);
bool bp_set_eligible(const KConst& k, int os, int nslab);
cudaError_t launch_bp_axis_set(const KConst* ks, const float2* const* ups, const SlabTable* slabs, int count,
                               size_t up_stride, void* vol, int vt, int pw, int ph, float lambda, int os,
                               const BpShape* shape, cudaStream_t st);
cudaError_t launch_slicer_fused(const KConst& c, const void* vol, int vt, float* imgs, size_t img_stride,
                                size_t pitchE, const SlabTable& slabs, int x0, int y0, int x1, int y1, cudaStream_t st, int nw = 4);
cudaError_t launch_compare(int pw, int ph, size_t pitchE, const float* real, float* virt, const float* dist,
                           float realLength, float4 cut, float4 dim, float scale, cudaStream_t st);
cudaError_t launch_crop_border(int pw, int ph, size_t pitchE, float* img, float2 cut, float2 dim, const int* p,
                               cudaStream_t st);
cudaError_t launch_make_square(int pw, int ph, size_t strideE, const float* in, int maxsize, float* out, int bx, int by,
                               int mirrorY, int fillZero, cudaStream_t st);
cudaError_t launch_crop_to_square(int pw, int ph, size_t pitchE, float* img, int apply_crop, float2 cut, float2 dim,
                                  const int* p, int maxsize, float* sq, int bx, int by, cudaStream_t st);
cudaError_t launch_square_to_image(const float* sq, int maxsize, size_t shift, float inv_norm, int pw, int ph,
                                   size_t pitchE, float* out, float* accum, int apply_crop, float2 cut, float2 dim,
                                   const int* p, cudaStream_t st, int transpose_out);
cudaError_t launch_transpose(const float* in, int w, int h, size_t pitchE, float* out, cudaStream_t st);
cudaError_t launch_square_to_image_batch(const float* sq, int count, int maxsize, size_t shift, float inv_norm, int pw,
                                         int ph, size_t pitchE, float* out, size_t out_stride, int transpose_out,
                                         cudaStream_t st);
cudaError_t launch_ctf_slabs(const float* in, float* out, size_t out_stride, int n, const CtfConst& k,
                             const CtfSlabs& slabs_nm, float angle_deg, int applyForFP, int phaseFlip, float wiener,
                             float4 beta, cudaStream_t st);
cudaError_t launch_fp_adjoint(const KConst& c, float* grad, const float* img, size_t pitchE, float sx, float sy, int w,
                              int h, cudaStream_t st);
cudaError_t launch_loss_grad(const KConst& c, const void* vol, int vt, const float* meas, size_t pitchE, float sx,
                             float sy, float* grad, float* proj_out, double* out, int w, int h, cudaStream_t st,
                             const int* roi = nullptr);
cudaError_t launch_rotate_volume(const float* in, float* out, int size, const float rot[9], cudaStream_t st);
cudaError_t launch_cc_center(float* sq, long n, double* sums, cudaStream_t st);
cudaError_t launch_cc_conj_mul(float* a, const float* b, long n_complex, cudaStream_t st);
cudaError_t launch_cc_map(const float* cc, int n, int s, const double* sums, float* map, cudaStream_t st);
cudaError_t launch_cc_finish(float* cc, int n, int s, const double* sums, unsigned long long* key, cudaStream_t st);
cudaError_t launch_cc_peaks(const float* img, float* out, int n, int s, const unsigned long long* key,
                            unsigned long long* key2, cudaStream_t st);
cudaError_t launch_convert_input(const void* in, int type, long n, float* out, cudaStream_t st);
cudaError_t launch_window_stats(const float* img, size_t pitchE, int x0, int y0, int w, int h, double* out,
                                cudaStream_t st);
cudaError_t launch_bad_pixels(float* img, long n, float threshold, float value, double* out, cudaStream_t st);
cudaError_t launch_window_div(const float* sq, size_t shift, int maxsize, int pw, int ph, float div, float* out,
                              cudaStream_t st);
cudaError_t launch_normalize(const float* in, float* out, long n, float mean, float std_, cudaStream_t st);
cudaError_t launch_crop_to_square_batch(int pw, int ph, float* images, size_t img_stride, int count, int apply_crop,
                                        int seq_crop, float2 cut, float2 dim, const int* p, int maxsize, float* sq,
                                        size_t sq_stride, int bx, int by, cudaStream_t st);
cudaError_t launch_ctf_batch(float* spec, size_t spec_stride, int n, const CtfConst& k, const CtfSlabs& slabs_nm,
                             float angle_deg, int applyForFP, int phaseFlip, float wiener, float4 beta,
                             cudaStream_t st);
cudaError_t launch_square_to_image_many(const float* sq, size_t sq_stride, int count, int maxsize, size_t shift,
                                        float inv_norm, int pw, int ph, float* out, size_t out_stride, float* accum,
                                        int apply_crop, float2 cut, float2 dim, const int* p, int transpose_out,
                                        cudaStream_t st);
CtfConst make_ctf_const(int n, float cs_mm, float voltage_kv, float amp_contrast, float pixel_size_nm);
cudaError_t launch_ctf(float* spec, int n, const CtfConst& k, float d0_nm, float d1_nm, float angle_deg, int applyForFP,
                       int phaseFlip, float wiener, float4 beta, cudaStream_t st);
cudaError_t launch_wbp_weighting(float* spec, int n, float psi_deg, int fm, cudaStream_t st);
cudaError_t launch_fourier_filter(float* spec, int n, float lp, float hp, float lps, float hps, cudaStream_t st);
cudaError_t launch_dose_weighting(float* spec, int n, float dose, float pixelsize, cudaStream_t st);
cudaError_t launch_convert(const void* vol, int vt, long n, float* out, float sign, cudaStream_t st);
cudaError_t launch_store(const float* in, long n, void* vol, int vt, cudaStream_t st);

static thread_local std::string g_last_error;
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
static void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void set_error(const std::string& msg) { g_last_error = msg; }
int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

static int cuda_fail(cudaError_t e, const char* where) {
  cudaGetLastError();  // a non-sticky error must not resurface in the next call
  return fail(ESB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

}  // namespace esb

using namespace esb;

#define ESB_CK(call, where)                       \
  do {                                            \
    cudaError_t e_ = (call);                      \
    if (e_ != cudaSuccess) return cuda_fail(e_, where); \
  } while (0)

#define ESB_FFT(call, where)                                                         \
  do {                                                                               \
    cufftResult r_ = (call);                                                         \
    if (r_ != CUFFT_SUCCESS)                                                         \
      return fail(ESB_ERR_CUFFT, std::string(where) + ": cuFFT error " + std::to_string((int)r_)); \
  } while (0)

static inline cudaStream_t as_stream(void* s) { return (cudaStream_t)s; }
static inline bool valid_vt(int vt) { return vt == ESB_VOXEL_F32 || vt == ESB_VOXEL_F16 || vt == ESB_VOXEL_BF16; }

static int check_image(int pw, int ph, size_t pitch, const char* where) {
  if (pw <= 0 || ph <= 0) return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": image size must be positive");
  if (pitch < (size_t)pw * sizeof(float) || pitch % sizeof(float) != 0)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": pitch must be a multiple of 4 and >= width*4");
  return ESB_OK;
}

static int check_constants(const esb_constants* c, const char* where) {
  if (!c) return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": constants are NULL");
  for (int k = 0; k < 3; ++k)
    if (!(c->volume_dim[k] >= 1.0f) || c->volume_dim[k] != floorf(c->volume_dim[k]))
      return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": volume_dim must be positive integers");
  return ESB_OK;
}

extern "C" {

const char* esb_last_error(void) { return g_last_error.c_str(); }
int esb_version(void) { return 100; }
unsigned long long esb_kernel_launches(void) { return g_launches.load(std::memory_order_relaxed); }

int esb_fp(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj, float* dist,
           size_t pitch, int roi_x0, int roi_y0, int roi_x1, int roi_y1, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_fp")) || (r = check_image(proj_x, proj_y, pitch, "esb_fp"))) return r;
  if (!vol || !proj || !dist || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_fp: invalid argument");
  roi_x0 = roi_x0 < 0 ? 0 : roi_x0;
  roi_y0 = roi_y0 < 0 ? 0 : roi_y0;
  roi_x1 = roi_x1 > proj_x ? proj_x : roi_x1;
  roi_y1 = roi_y1 > proj_y ? proj_y : roi_y1;
  ESB_CK(launch_march(to_kconst(*c), vol, voxel_type, proj, dist, pitch / 4, roi_x0, roi_y0, roi_x1, roi_y1,
                      as_stream(stream)), "esb_fp");
  return ok();
}

int esb_fp_slicer(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj,
                  size_t pitch, float tmin, float tmax, int roi_x0, int roi_y0, int roi_x1, int roi_y1, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_fp_slicer")) || (r = check_image(proj_x, proj_y, pitch, "esb_fp_slicer"))) return r;
  if (!vol || !proj || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_fp_slicer: invalid argument");
  roi_x0 = roi_x0 < 0 ? 0 : roi_x0;
  roi_y0 = roi_y0 < 0 ? 0 : roi_y0;
  roi_x1 = roi_x1 > proj_x ? proj_x : roi_x1;
  roi_y1 = roi_y1 > proj_y ? proj_y : roi_y1;
  ESB_CK(launch_slicer(to_kconst(*c), vol, voxel_type, proj, pitch / 4, tmin, tmax, roi_x0, roi_y0, roi_x1, roi_y1,
                       as_stream(stream)), "esb_fp_slicer");
  return ok();
}

int esb_vol_traversal_length(const esb_constants* c, int proj_x, int proj_y, float* dist, size_t pitch, int roi_x0,
                             int roi_y0, int roi_x1, int roi_y1, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_vol_traversal_length")) ||
      (r = check_image(proj_x, proj_y, pitch, "esb_vol_traversal_length")))
    return r;
  if (!dist) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_vol_traversal_length: dist is NULL");
  roi_x0 = roi_x0 < 0 ? 0 : roi_x0;
  roi_y0 = roi_y0 < 0 ? 0 : roi_y0;
  roi_x1 = roi_x1 > proj_x ? proj_x : roi_x1;
  roi_y1 = roi_y1 > proj_y ? proj_y : roi_y1;
  ESB_CK(launch_travlen(to_kconst(*c), dist, pitch / 4, roi_x0, roi_y0, roi_x1, roi_y1, as_stream(stream)),
         "esb_vol_traversal_length");
  return ok();
}

int esb_compare(int proj_x, int proj_y, size_t pitch, const float* real, float* virt, const float* dist,
                float real_length, const float crop[4], const float crop_dim[4], float proj_val_scale, void* stream) {
  int r;
  if ((r = check_image(proj_x, proj_y, pitch, "esb_compare"))) return r;
  if (!real || !virt || !dist || !crop || !crop_dim) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_compare: NULL argument");
  ESB_CK(launch_compare(proj_x, proj_y, pitch / 4, real, virt, dist, real_length,
                        make_float4(crop[0], crop[1], crop[2], crop[3]),
                        make_float4(crop_dim[0], crop_dim[1], crop_dim[2], crop_dim[3]), proj_val_scale,
                        as_stream(stream)), "esb_compare");
  return ok();
}

int esb_crop_border(int proj_x, int proj_y, size_t pitch, float* img, const float cut_length[2],
                    const float dim_length[2], const int p[8], void* stream) {
  int r;
  if ((r = check_image(proj_x, proj_y, pitch, "esb_crop_border"))) return r;
  if (!img || !cut_length || !dim_length || !p) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_crop_border: NULL argument");
  ESB_CK(launch_crop_border(proj_x, proj_y, pitch / 4, img, make_float2(cut_length[0], cut_length[1]),
                            make_float2(dim_length[0], dim_length[1]), p, as_stream(stream)), "esb_crop_border");
  return ok();
}

int esb_bp(const esb_constants* c, void* vol, int voxel_type, int proj_x, int proj_y, const float* img, size_t pitch,
           float lambda, int oversampling, float dist_min, float dist_max, int linear_filter, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_bp")) || (r = check_image(proj_x, proj_y, pitch, "esb_bp"))) return r;
  if (!vol || !img || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_bp: invalid argument");
  if (oversampling < 1) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_bp: oversampling must be >= 1");
  if (4 * c->volume_dim_x_quarter > (int)c->volume_dim[0])
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_bp: volume_dim_x_quarter exceeds volume_dim.x / 4");
  ESB_CK(launch_bp(to_kconst(*c), vol, voxel_type, img, proj_x, proj_y, pitch / 4, lambda, oversampling, dist_min,
                   dist_max, linear_filter, as_stream(stream)), "esb_bp");
  return ok();
}

int esb_fp_fast(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj,
                float* dist, size_t pitch, int roi_x0, int roi_y0, int roi_x1, int roi_y1, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_fp_fast")) || (r = check_image(proj_x, proj_y, pitch, "esb_fp_fast"))) return r;
  if (!vol || !proj || !dist || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_fp_fast: invalid argument");
  roi_x0 = roi_x0 < 0 ? 0 : roi_x0;
  roi_y0 = roi_y0 < 0 ? 0 : roi_y0;
  roi_x1 = roi_x1 > proj_x ? proj_x : roi_x1;
  roi_y1 = roi_y1 > proj_y ? proj_y : roi_y1;
  ESB_CK(launch_project_fast(to_kconst(*c), vol, voxel_type, 0, proj, dist, pitch / 4, 0.f, 0.f, roi_x0, roi_y0, roi_x1,
                             roi_y1, as_stream(stream)), "esb_fp_fast");
  return ok();
}

int esb_fp_slicer_fast(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj,
                       size_t pitch, float tmin, float tmax, int roi_x0, int roi_y0, int roi_x1, int roi_y1,
                       void* stream) {
  int r;
  if ((r = check_constants(c, "esb_fp_slicer_fast")) || (r = check_image(proj_x, proj_y, pitch, "esb_fp_slicer_fast")))
    return r;
  if (!vol || !proj || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_fp_slicer_fast: invalid argument");
  roi_x0 = roi_x0 < 0 ? 0 : roi_x0;
  roi_y0 = roi_y0 < 0 ? 0 : roi_y0;
  roi_x1 = roi_x1 > proj_x ? proj_x : roi_x1;
  roi_y1 = roi_y1 > proj_y ? proj_y : roi_y1;
  ESB_CK(launch_project_fast(to_kconst(*c), vol, voxel_type, 1, proj, nullptr, pitch / 4, tmin, tmax, roi_x0, roi_y0,
                             roi_x1, roi_y1, as_stream(stream)), "esb_fp_slicer_fast");
  return ok();
}

int esb_bp_fast(const esb_constants* c, void* vol, int voxel_type, int proj_x, int proj_y, const float* img,
                size_t pitch, float lambda, int oversampling, float dist_min, float dist_max, int linear_filter,
                void* stream) {
  int r;
  if ((r = check_constants(c, "esb_bp_fast")) || (r = check_image(proj_x, proj_y, pitch, "esb_bp_fast"))) return r;
  if (!vol || !img || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_bp_fast: invalid argument");
  if (oversampling < 1) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_bp_fast: oversampling must be >= 1");
  if (4 * c->volume_dim_x_quarter > (int)c->volume_dim[0])
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_bp_fast: volume_dim_x_quarter exceeds volume_dim.x / 4");
  ESB_CK(launch_bp_fast(to_kconst(*c), vol, voxel_type, img, proj_x, proj_y, pitch / 4, lambda, oversampling, dist_min,
                        dist_max, linear_filter, as_stream(stream)), "esb_bp_fast");
  return ok();
}

int esb_fp_adjoint(const esb_constants* c, float* grad_vol, int proj_x, int proj_y, const float* img, size_t pitch,
                   float shift_u, float shift_v, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_fp_adjoint")) || (r = check_image(proj_x, proj_y, pitch, "esb_fp_adjoint"))) return r;
  if (!grad_vol || !img) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_fp_adjoint: NULL argument");
  ESB_CK(launch_fp_adjoint(to_kconst(*c), grad_vol, img, pitch / 4, shift_u, shift_v, proj_x, proj_y, as_stream(stream)),
         "esb_fp_adjoint");
  return ok();
}

int esb_projection_loss_grad(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y,
                             const float* measured, size_t pitch, float shift_u, float shift_v, float* grad_vol,
                             float* proj_out, double* out6, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_projection_loss_grad")) ||
      (r = check_image(proj_x, proj_y, pitch, "esb_projection_loss_grad")))
    return r;
  if (!vol || !out6 || !valid_vt(voxel_type))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_projection_loss_grad: invalid argument");
  ESB_CK(launch_loss_grad(to_kconst(*c), vol, voxel_type, measured, pitch / 4, shift_u, shift_v, grad_vol, proj_out,
                          out6, proj_x, proj_y, as_stream(stream)), "esb_projection_loss_grad");
  return ok();
}

int esb_projection_loss_grad_roi(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y,
                                 const float* measured, size_t pitch, float shift_u, float shift_v, const int roi[4],
                                 float* grad_vol, float* proj_out, double* out8, void* stream) {
  int r;
  if ((r = check_constants(c, "esb_projection_loss_grad_roi")) ||
      (r = check_image(proj_x, proj_y, pitch, "esb_projection_loss_grad_roi")))
    return r;
  if (!vol || !out8 || !roi || !valid_vt(voxel_type))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_projection_loss_grad_roi: invalid argument");
  const int box[4] = {std::max(roi[0], 0), std::max(roi[1], 0), std::min(roi[2], proj_x), std::min(roi[3], proj_y)};
  ESB_CK(launch_loss_grad(to_kconst(*c), vol, voxel_type, measured, pitch / 4, shift_u, shift_v, grad_vol, proj_out,
                          out8, proj_x, proj_y, as_stream(stream), box), "esb_projection_loss_grad_roi");
  return ok();
}

int esb_rotate_volume(const float* in, float* out, int size, const float rot[9], void* stream) {
  if (!in || !out || !rot || size <= 0 || size > 2048)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rotate_volume: invalid argument");
  const size_t bytes = (size_t)size * size * size * sizeof(float);
  if ((const char*)in < (const char*)out + bytes && (const char*)out < (const char*)in + bytes)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rotate_volume: in and out overlap");
  ESB_CK(launch_rotate_volume(in, out, size, rot, as_stream(stream)), "esb_rotate_volume");
  return ok();
}

int esb_make_square(int proj_x, int proj_y, size_t pitch, const float* in, int maxsize, float* out, int border_x,
                    int border_y, int mirror_y, int fill_zero, void* stream) {
  int r;
  if ((r = check_image(proj_x, proj_y, pitch, "esb_make_square"))) return r;
  if (!in || !out || maxsize <= 0) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_make_square: invalid argument");
  if (!fill_zero && (maxsize - border_x > 2 * proj_x || maxsize - border_y > 2 * proj_y || border_x > proj_x ||
                     border_y > proj_y))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_make_square: mirror padding wider than the image");
  ESB_CK(launch_make_square(proj_x, proj_y, pitch / 4, in, maxsize, out, border_x, border_y, mirror_y, fill_zero,
                            as_stream(stream)), "esb_make_square");
  return ok();
}

int esb_ctf(float* spectrum, int n, float defocus_min_nm, float defocus_max_nm, float angle_deg, int apply_for_fp,
            int phase_flip_only, float wiener_noise_level, const float beta_fac[4], float cs_mm, float voltage_kv,
            float amp_contrast, float pixel_size_nm, void* stream) {
  if (!spectrum || n <= 1 || !beta_fac || pixel_size_nm <= 0)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_ctf: invalid argument");
  CtfConst k = make_ctf_const(n, cs_mm, voltage_kv, amp_contrast, pixel_size_nm);
  ESB_CK(launch_ctf(spectrum, n, k, defocus_min_nm, defocus_max_nm, angle_deg, apply_for_fp, phase_flip_only,
                    wiener_noise_level, make_float4(beta_fac[0], beta_fac[1], beta_fac[2], beta_fac[3]),
                    as_stream(stream)), "esb_ctf");
  return ok();
}

int esb_wbp_weighting(float* spectrum, int n, float psi_deg, int filter, void* stream) {
  if (!spectrum || n <= 1 || filter < 0 || filter > 4)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_wbp_weighting: invalid argument");
  ESB_CK(launch_wbp_weighting(spectrum, n, psi_deg, filter, as_stream(stream)), "esb_wbp_weighting");
  return ok();
}

int esb_fourier_filter(float* spectrum, int n, float lp, float hp, float lps, float hps, void* stream) {
  if (!spectrum || n <= 1) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_fourier_filter: invalid argument");
  ESB_CK(launch_fourier_filter(spectrum, n, lp, hp, lps, hps, as_stream(stream)), "esb_fourier_filter");
  return ok();
}

int esb_dose_weighting(float* spectrum, int n, float dose, float pixel_size_a, void* stream) {
  if (!spectrum || n <= 1 || pixel_size_a <= 0) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_dose_weighting: invalid argument");
  ESB_CK(launch_dose_weighting(spectrum, n, dose, pixel_size_a, as_stream(stream)), "esb_dose_weighting");
  return ok();
}

int esb_convert_volume(const void* vol, int voxel_type, long n_voxels, float* out, int negate, void* stream) {
  if (!vol || !out || n_voxels < 0 || !valid_vt(voxel_type))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_convert_volume: invalid argument");
  if (n_voxels == 0) return ok();
  ESB_CK(launch_convert(vol, voxel_type, n_voxels, out, negate ? -1.0f : 1.0f, as_stream(stream)), "esb_convert_volume");
  return ok();
}

int esb_store_volume(const float* in, long n_voxels, void* vol, int voxel_type, void* stream) {
  if (!vol || !in || n_voxels < 0 || !valid_vt(voxel_type))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_store_volume: invalid argument");
  if (n_voxels == 0) return ok();
  ESB_CK(launch_store(in, n_voxels, vol, voxel_type, as_stream(stream)), "esb_store_volume");
  return ok();
}

}  // extern "C"

// ===================================================================== Reconstructor

// Pool of event pairs for one timing phase.
struct PhaseTimer {
  std::vector<cudaEvent_t> start, stop;
  size_t used = 0;
  cudaError_t begin(cudaStream_t s) {
    if (used == start.size()) {
      cudaEvent_t a, b;
      cudaError_t e = cudaEventCreate(&a);
      if (e != cudaSuccess) return e;
      e = cudaEventCreate(&b);
      if (e != cudaSuccess) return e;
      start.push_back(a);
      stop.push_back(b);
    }
    return cudaEventRecord(start[used], s);
  }
  cudaError_t end(cudaStream_t s) { return cudaEventRecord(stop[used++], s); }
  void destroy() {
    for (auto e : start) cudaEventDestroy(e);
    for (auto e : stop) cudaEventDestroy(e);
    start.clear();
    stop.clear();
    used = 0;
  }
};

struct esb_reconstructor {
  esb_recon_config cfg;
  std::vector<esb_proj_geom> geoms;
  std::vector<float> tilt;
  std::vector<float> defocus;  // [n][3]: min nm, max nm, astigmatism angle deg
  float aniso[9], anisoInv[9];
  int N = 0;
  int borderX = 0, borderY = 0;
  size_t squareShift = 0;
  float *proj_d = nullptr, *dist_d = nullptr, *real_d = nullptr;
  float* square_d = nullptr;
  float* fft_d = nullptr;
  std::vector<float*> sirt_d;  // residual images of one ordered subset
  bool plans = false;
  cufftHandle r2c = 0, c2r = 0;
  cudaStream_t stream = nullptr;
  CtfConst ctfk;
  bool timing = false;
  PhaseTimer timers[4];
  float* slab_imgs = nullptr;  // per-slab images of the fused CTF paths
  size_t slab_cap = 0;         // capacity in images
  float2* up_imgs = nullptr;   // the slab images pre-sampled on the sub-pixel grid, with sample rows
  size_t up_cap = 0;           // capacity in floats
  void* tune_scratch = nullptr;  // the autotuner's trial outputs
  size_t tune_cap = 0;           // capacity in bytes
  SubvolBatch batch;           // tables of the batched sub-volume launch
  // filtered spectra and squares of a chunk of CTF slabs, with a batched
  // C2R plan per chunk size
  float* spec_batch = nullptr;
  float* sq_batch = nullptr;
  int batch_slabs = 0;
  cufftHandle c2r_many[ESB_CTF_SLAB_BATCH + 1] = {};
  bool c2r_many_ok[ESB_CTF_SLAB_BATCH + 1] = {};
  cufftHandle r2c_many[ESB_CTF_SLAB_BATCH + 1] = {};
  bool r2c_many_ok[ESB_CTF_SLAB_BATCH + 1] = {};
  bool graphs = false;                   // replay SART iterations from a captured graph
  int fuse_subsets = -1;                 // subset back-projection in one volume pass: 1 on, 0 off, -1 half volumes
  bool subvol_patches = false;           // sub-volume WBP with CTF: all tilts in one launch from gathered patches
  cudaGraphExec_t sart_exec = nullptr;   // the last captured iteration
  // inputs the captured iteration was recorded with (it replays only for the
  // same ones) and the library kernels it launches
  struct {
    const void* vol = nullptr;
    int voxel_type = -1;
    const float* projections = nullptr;
    esb_vol_geom vg{};
    std::vector<int> index_list;
    int sirt_count = 0;
  } sart_key;
  unsigned long long sart_graph_launches = 0;
  cudaStream_t capture_stream = nullptr;  // private stream the capture records on
  // projection preparation: square, spectrum and plans when CTF is off,
  // the converted / windowed image and the statistics
  float* prep_sq = nullptr;
  float* prep_fft = nullptr;
  float* prep_img = nullptr;
  double* prep_stats = nullptr;
  cufftHandle prep_r2c = 0, prep_c2r = 0;
  bool prep_plans = false;
  // cross-correlation displacement: two squares, two spectra, the sums of
  // both squares (4 doubles) and two arg-max keys
  float* cc_sq = nullptr;
  float* cc_spec = nullptr;
  void* cc_red = nullptr;
};

// Brackets a phase of launches with events when timing is enabled.
struct PhaseScope {
  esb_reconstructor* r;
  int phase;
  PhaseScope(esb_reconstructor* r_, int p) : r(r_), phase(p) {
    if (r->timing) r->timers[phase].begin(r->stream);
  }
  ~PhaseScope() {
    if (r->timing) r->timers[phase].end(r->stream);
  }
};

static int rec_alloc(esb_reconstructor* r) {
  const size_t img = (size_t)r->cfg.proj_x * r->cfg.proj_y * sizeof(float);
  // the projection and the ray-length image are one buffer (projection
  // first), so that a z-slab run sums both over ranks in one collective
  ESB_CK(cudaMalloc(&r->proj_d, 2 * img), "esb_reconstructor_create");
  r->dist_d = r->proj_d + (size_t)r->cfg.proj_x * r->cfg.proj_y;
  ESB_CK(cudaMalloc(&r->real_d, img), "esb_reconstructor_create");
  ESB_CK(cudaMemset(r->proj_d, 0, img), "esb_reconstructor_create");
  ESB_CK(cudaMemset(r->dist_d, 0, img), "esb_reconstructor_create");
  if (r->cfg.ctf_mode) {
    const int N = r->N;
    ESB_CK(cudaMalloc(&r->square_d, (size_t)N * N * sizeof(float)), "esb_reconstructor_create");
    ESB_CK(cudaMalloc(&r->fft_d, (size_t)(N / 2 + 1) * N * 2 * sizeof(float)), "esb_reconstructor_create");
    ESB_FFT(cufftPlan2d(&r->r2c, N, N, CUFFT_R2C), "esb_reconstructor_create");
    ESB_FFT(cufftPlan2d(&r->c2r, N, N, CUFFT_C2R), "esb_reconstructor_create");
    r->plans = true;
  }
  return ESB_OK;
}

static void rec_free(esb_reconstructor* r) {
  cudaFree(r->proj_d);  // with dist_d
  cudaFree(r->real_d);
  cudaFree(r->square_d);
  cudaFree(r->fft_d);
  for (float* p : r->sirt_d) cudaFree(p);
  r->sirt_d.clear();
  if (r->plans) {
    cufftDestroy(r->r2c);
    cufftDestroy(r->c2r);
  }
  for (auto& t : r->timers) t.destroy();
  cudaFree(r->slab_imgs);
  r->slab_imgs = nullptr;
  r->slab_cap = 0;
  cudaFree(r->up_imgs);
  cudaFree(r->tune_scratch);
  r->up_imgs = nullptr;
  r->up_cap = 0;
  subvol_batch_free(r->batch);
  if (r->sart_exec) {
    cudaStreamSynchronize(r->stream);
    cudaGraphExecDestroy(r->sart_exec);
    r->sart_exec = nullptr;
  }
  if (r->capture_stream) {
    cudaStreamDestroy(r->capture_stream);
    r->capture_stream = nullptr;
  }
  cudaFree(r->prep_sq);
  cudaFree(r->prep_fft);
  cudaFree(r->prep_img);
  cudaFree(r->prep_stats);
  r->prep_sq = r->prep_fft = r->prep_img = nullptr;
  r->prep_stats = nullptr;
  if (r->prep_plans) {
    cufftDestroy(r->prep_r2c);
    cufftDestroy(r->prep_c2r);
    r->prep_plans = false;
  }
  cudaFree(r->cc_sq);
  cudaFree(r->cc_spec);
  cudaFree(r->cc_red);
  r->cc_sq = r->cc_spec = nullptr;
  r->cc_red = nullptr;
  cudaFree(r->spec_batch);
  cudaFree(r->sq_batch);
  r->spec_batch = r->sq_batch = nullptr;
  r->batch_slabs = 0;
  for (int i = 0; i <= ESB_CTF_SLAB_BATCH; ++i) {
    if (r->c2r_many_ok[i]) {
      cufftDestroy(r->c2r_many[i]);
      r->c2r_many_ok[i] = false;
    }
    if (r->r2c_many_ok[i]) {
      cufftDestroy(r->r2c_many[i]);
      r->r2c_many_ok[i] = false;
    }
  }
}

extern "C" {

int esb_reconstructor_create(const esb_recon_config* cfg, const esb_proj_geom* geoms, const float* tilt_deg,
                             const float* defocus, const float mag_aniso[9], const float mag_aniso_inv[9],
                             esb_reconstructor** out) {
  if (!cfg || !geoms || !tilt_deg || !out)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_create: NULL argument");
  if (cfg->proj_x <= 0 || cfg->proj_y <= 0 || cfg->n_proj <= 0 || cfg->oversampling < 1)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_create: invalid sizes");
  if (cfg->ctf_mode && (!defocus || cfg->pixel_size_nm <= 0 || cfg->ctf_slice_thickness_nm <= 0))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_create: CTF mode needs defocus, pixel size and slab thickness");
  esb_reconstructor* r = new esb_reconstructor();
  r->cfg = *cfg;
  r->geoms.assign(geoms, geoms + cfg->n_proj);
  r->tilt.assign(tilt_deg, tilt_deg + cfg->n_proj);
  if (defocus) r->defocus.assign(defocus, defocus + 3 * (size_t)cfg->n_proj);
  static const float ident[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  memcpy(r->aniso, mag_aniso ? mag_aniso : ident, sizeof(r->aniso));
  memcpy(r->anisoInv, mag_aniso_inv ? mag_aniso_inv : ident, sizeof(r->anisoInv));
  // Reconstructor::Reconstructor (Reconstructor.cpp:340-347): square image
  // of the larger side, image centred in it.
  r->N = cfg->proj_x > cfg->proj_y ? cfg->proj_x : cfg->proj_y;
  size_t shx = (r->N - cfg->proj_x) / 2, shy = (size_t)((r->N - cfg->proj_y) / 2) * r->N;
  r->squareShift = shx + shy;
  r->borderX = (r->N - cfg->proj_x) / 2;
  r->borderY = (r->N - cfg->proj_y) / 2;
  if (cfg->ctf_mode) r->ctfk = make_ctf_const(r->N, cfg->cs_mm, cfg->voltage_kv, cfg->amp_contrast, cfg->pixel_size_nm);
  int rc = rec_alloc(r);
  if (rc != ESB_OK) {
    std::string msg = esb_last_error();
    rec_free(r);
    delete r;
    return fail(rc, msg);
  }
  *out = r;
  return ok();
}

int esb_reconstructor_destroy(esb_reconstructor* rec) {
  if (!rec) return ok();
  rec_free(rec);
  delete rec;
  return ok();
}

int esb_reconstructor_set_stream(esb_reconstructor* rec, void* stream) {
  if (!rec) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_set_stream: NULL reconstructor");
  rec->stream = (cudaStream_t)stream;
  if (rec->plans) {
    ESB_FFT(cufftSetStream(rec->r2c, rec->stream), "esb_reconstructor_set_stream");
    ESB_FFT(cufftSetStream(rec->c2r, rec->stream), "esb_reconstructor_set_stream");
    for (int i = 0; i <= ESB_CTF_SLAB_BATCH; ++i) {
      if (rec->c2r_many_ok[i]) ESB_FFT(cufftSetStream(rec->c2r_many[i], rec->stream), "esb_reconstructor_set_stream");
      if (rec->r2c_many_ok[i]) ESB_FFT(cufftSetStream(rec->r2c_many[i], rec->stream), "esb_reconstructor_set_stream");
    }
  }
  return ok();
}

int esb_reconstructor_buffers(esb_reconstructor* rec, float** proj_d, float** dist_d, float** real_d) {
  if (!rec) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_buffers: NULL reconstructor");
  if (proj_d) *proj_d = rec->proj_d;
  if (dist_d) *dist_d = rec->dist_d;
  if (real_d) *real_d = rec->real_d;
  return ok();
}

int esb_reconstructor_enable_timing(esb_reconstructor* rec, int enable) {
  if (!rec) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_enable_timing: NULL reconstructor");
  rec->timing = enable != 0;
  for (auto& t : rec->timers) t.used = 0;
  return ok();
}

int esb_reconstructor_enable_graphs(esb_reconstructor* rec, int enable) {
  if (!rec) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_enable_graphs: NULL reconstructor");
  rec->graphs = enable != 0;
  return ok();
}

int esb_reconstructor_fuse_subsets(esb_reconstructor* rec, int enable) {
  if (!rec) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_fuse_subsets: NULL reconstructor");
  rec->fuse_subsets = enable < 0 ? -1 : (enable != 0);
  return ok();
}

int esb_reconstructor_subvolume_patches(esb_reconstructor* rec, int enable) {
  if (!rec) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_subvolume_patches: NULL reconstructor");
  rec->subvol_patches = enable != 0;
  return ok();
}

int esb_reconstructor_timing(esb_reconstructor* rec, double out_ms[4], int counts[4]) {
  if (!rec || !out_ms || !counts) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_reconstructor_timing: NULL argument");
  ESB_CK(cudaStreamSynchronize(rec->stream), "esb_reconstructor_timing");
  for (int p = 0; p < 4; ++p) {
    double sum = 0;
    PhaseTimer& t = rec->timers[p];
    for (size_t i = 0; i < t.used; ++i) {
      float ms = 0;
      ESB_CK(cudaEventElapsedTime(&ms, t.start[i], t.stop[i]), "esb_reconstructor_timing");
      sum += ms;
    }
    out_ms[p] = sum;
    counts[p] = (int)t.used;
    t.used = 0;
  }
  return ok();
}

int esb_rec_reset_projections(esb_reconstructor* r) {
  if (!r) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_reset_projections: NULL reconstructor");
  PhaseScope ps(r, 3);
  const size_t img = (size_t)r->cfg.proj_x * r->cfg.proj_y * sizeof(float);
  ESB_CK(cudaMemsetAsync(r->proj_d, 0, img, r->stream), "esb_rec_reset_projections");
  ESB_CK(cudaMemsetAsync(r->dist_d, 0, img, r->stream), "esb_rec_reset_projections");
  return ok();
}

}  // extern "C"

// ------------------------------------------------------------ autotuning
// Launch shapes that do not change results (every thread does the same work
// under every shape) are picked per GPU and problem shape the first time a
// reconstructor launches the kernel outside stream capture: each candidate
// is timed with CUDA events on the reconstructor's stream (one warm-up
// launch, two timed ones) and the fastest is cached for the process.
// Projector candidates read the real volume and write scratch images;
// back-projection candidates run on a scratch slab of up to 32 planes from
// the middle of the volume, so the caller's volume is never written by a
// trial; the scratch is released once the trials are done. During
// capture, or when tuning is off, the cached or the default shape is taken.
namespace {
struct TuneKey {
  int kernel, dev, sms, vt, w, h, dx, dy, dz, os, ctf;
  auto tie() const { return std::tie(kernel, dev, sms, vt, w, h, dx, dy, dz, os, ctf); }
  bool operator<(const TuneKey& o) const { return tie() < o.tie(); }
};
std::mutex g_tune_mu;
std::map<TuneKey, int> g_tune;
std::atomic<int> g_tune_on{1};
std::atomic<int> g_tune_force{-1};  // >= 0: every tuned kernel takes this candidate (tests)
// back-projection shapes (quads x rows per block), candidate index -> shape
const int kBpShapes[][2] = {{32, 4}, {32, 2}, {16, 8}, {64, 2}, {32, 1}};
const int kNBpShapes = 5;
const char* kTuneNames[] = {"fp_slicer_fused", "fp_march", "bp_axis"};
}  // namespace

static TuneKey tune_key(esb_reconstructor* r, int kernel, int vt, const KConst& c, int ctf) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return TuneKey{kernel, dev, sms, vt, r->cfg.proj_x, r->cfg.proj_y, (int)c.dim.x, (int)c.dim.y, (int)c.dim.z,
                 r->cfg.oversampling, ctf};
}

static void* rec_tune_scratch(esb_reconstructor* r, size_t bytes) {
  if (bytes <= r->tune_cap) return r->tune_scratch;
  if (cudaStreamSynchronize(r->stream) != cudaSuccess) return nullptr;
  cudaFree(r->tune_scratch);
  r->tune_scratch = nullptr;
  r->tune_cap = 0;
  if (cudaMalloc(&r->tune_scratch, bytes) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  r->tune_cap = bytes;
  return r->tune_scratch;
}

// The cached choice for key, else candidates[0..n) timed with run(choice)
// (a trial that fails excludes its candidate); def when nothing is measured.
template <class Run>
static int rec_tuned(esb_reconstructor* r, const TuneKey& key, int n, int def, Run run) {
  const int forced = g_tune_force.load();
  if (forced >= 0) return std::min(forced, n - 1);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  if (!g_tune_on.load()) return def;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(r->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {
    cudaGetLastError();
    return def;
  }
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return def;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return def;
  }
  int best = def;
  float best_ms = FLT_MAX;
  for (int i = 0; i < n; ++i) {
    if (run(i) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    cudaEventRecord(e0, r->stream);
    cudaError_t e = run(i);
    if (e == cudaSuccess) e = run(i);
    cudaEventRecord(e1, r->stream);
    float ms = FLT_MAX;
    if (e == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
    cudaGetLastError();
    if (ms < best_ms) {
      best_ms = ms;
      best = i;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the trials are done (synchronised above): release their scratch
  cudaFree(r->tune_scratch);
  r->tune_scratch = nullptr;
  r->tune_cap = 0;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune[key] = best;
  return best;
}

static const int kNw[3] = {4, 2, 8};  // warps per projector block; index 0 is the default

extern "C" int esb_autotune(int enable) {
  if (enable < -1) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_autotune: enable must be >= -1");
  if (enable == -1) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune.clear();
  } else if (enable >= 2) {
    g_tune_force.store(enable - 2);
  } else {
    g_tune_force.store(-1);
    g_tune_on.store(enable);
  }
  return ok();
}

extern "C" int esb_autotune_report(char* buf, size_t len, size_t* needed) {
  if (!buf && len) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_autotune_report: buf is NULL");
  std::string text;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (const auto& kv : g_tune) {
      const TuneKey& k = kv.first;
      char line[256];
      if (k.kernel == 2)
        snprintf(line, sizeof line, "%s dev=%d sms=%d voxel=%d detector=%dx%d volume=%dx%dx%d os=%d ctf=%d block=%dx%d\n",
                 kTuneNames[k.kernel], k.dev, k.sms, k.vt, k.w, k.h, k.dx, k.dy, k.dz, k.os, k.ctf,
                 kBpShapes[kv.second][0], kBpShapes[kv.second][1]);
      else
        snprintf(line, sizeof line, "%s dev=%d sms=%d voxel=%d detector=%dx%d volume=%dx%dx%d os=%d ctf=%d warps=%d\n",
                 kTuneNames[k.kernel], k.dev, k.sms, k.vt, k.w, k.h, k.dx, k.dy, k.dz, k.os, k.ctf, kNw[kv.second]);
      text += line;
    }
  }
  if (needed) *needed = text.size() + 1;
  if (len) {
    const size_t n = std::min(len - 1, text.size());
    memcpy(buf, text.data(), n);
    buf[n] = 0;
  }
  return ok();
}

// Warps per block of the fused slicer for this problem.
static int rec_slicer_nw(esb_reconstructor* r, const KConst& c, const void* vol, int vt, size_t img,
                         const SlabTable& T) {
  const int W = r->cfg.proj_x, H = r->cfg.proj_y;
  const int i = rec_tuned(r, tune_key(r, 0, vt, c, 1), 3, 0, [&](int k) {
    return launch_slicer_fused(c, vol, vt, r->slab_imgs, img, W, T, 0, 0, W, H, r->stream, kNw[k]);
  });
  return kNw[i];
}

// Warps per block of the march projector (trials write scratch images: the
// projection accumulates into proj_d).
static int rec_march_nw(esb_reconstructor* r, const KConst& c, const void* vol, int vt) {
  const int W = r->cfg.proj_x, H = r->cfg.proj_y;
  const size_t img = (size_t)W * H;
  const int i = rec_tuned(r, tune_key(r, 1, vt, c, 0), 3, 0, [&](int k) {
    float* s = (float*)rec_tune_scratch(r, 2 * img * sizeof(float));
    if (!s) return cudaErrorMemoryAllocation;
    return launch_project_fast(c, vol, vt, 0, s, s + img, W, 0.f, 0.f, 0, 0, W, H, r->stream, kNw[k]);
  });
  return kNw[i];
}

// Block shape of the single-axis back-projection for this problem; trials on
// a scratch slab of up to 32 planes from the middle of the volume.
static BpShape rec_bp_shape(esb_reconstructor* r, const KConst& c, int vt, const float* imgs, size_t img_stride,
                            const SlabTable& T, int linear, const float2* up, size_t up_stride) {
  const int W = r->cfg.proj_x, H = r->cfg.proj_y, os = r->cfg.oversampling;
  BpShape s{kBpShapes[0][0], kBpShapes[0][1], 0, 0};
  if (!bp_uses_axis(c, os)) return s;
  const int nz = (int)c.dim.z, planes = std::min(nz, 32);
  const size_t plane = (size_t)c.dim.x * (size_t)c.dim.y * (vt == ESB_VOXEL_F32 ? 4 : 2);
  const int i = rec_tuned(r, tune_key(r, 2, vt, c, T.count > 0), kNBpShapes, 0, [&](int k) {
    void* slab = rec_tune_scratch(r, plane * planes);
    if (!slab) return cudaErrorMemoryAllocation;
    const BpShape t{kBpShapes[k][0], kBpShapes[k][1], std::max(0, nz / 2 - planes / 2), planes};
    return launch_bp_fast_slabs(c, slab, vt, imgs, img_stride, T, W, H, W, 0.0f, os, 0.0f, 9999999999999.0f, linear,
                                r->stream, 1, up, up_stride, &t);
  });
  s.bx = kBpShapes[i][0];
  s.by = kBpShapes[i][1];
  return s;
}

// Kernel variant of the reconstructor (faithful or fast).
// roi: detector region [roi[0], roi[2]) x [roi[1], roi[3]) (the reference's
// roiMin / roiMax), already clipped to the image.
static cudaError_t rec_march(esb_reconstructor* r, const KConst& c, const void* vol, int vt, const int* roi) {
  const int W = r->cfg.proj_x;
  if (r->cfg.variant == ESB_VARIANT_FAST)
    return launch_project_fast(c, vol, vt, 0, r->proj_d, r->dist_d, W, 0.f, 0.f, roi[0], roi[1], roi[2], roi[3],
                               r->stream, rec_march_nw(r, c, vol, vt));
  return launch_march(c, vol, vt, r->proj_d, r->dist_d, W, roi[0], roi[1], roi[2], roi[3], r->stream);
}
static cudaError_t rec_slicer(esb_reconstructor* r, const KConst& c, const void* vol, int vt, float* out, float t0,
                              float t1, const int* roi) {
  const int W = r->cfg.proj_x;
  if (r->cfg.variant == ESB_VARIANT_FAST)
    return launch_project_fast(c, vol, vt, 1, out, nullptr, W, t0, t1, roi[0], roi[1], roi[2], roi[3], r->stream);
  return launch_slicer(c, vol, vt, out, W, t0, t1, roi[0], roi[1], roi[2], roi[3], r->stream);
}
static cudaError_t rec_bp(esb_reconstructor* r, const KConst& c, void* vol, int vt, const float* img, float lambda,
                          float dmin, float dmax, int linear) {
  const int W = r->cfg.proj_x, H = r->cfg.proj_y;
  if (r->cfg.variant == ESB_VARIANT_FAST)
    return launch_bp_fast(c, vol, vt, img, W, H, W, lambda, r->cfg.oversampling, dmin, dmax, linear, r->stream);
  return launch_bp(c, vol, vt, img, W, H, W, lambda, r->cfg.oversampling, dmin, dmax, linear, r->stream);
}

static int rec_check(esb_reconstructor* r, const esb_vol_geom* vg, int index, const char* where) {
  if (!r || !vg) return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": NULL argument");
  if (index < 0 || index >= r->cfg.n_proj) return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": index out of range");
  return ESB_OK;
}

static KConst rec_const(esb_reconstructor* r, const esb_proj_geom& g, const esb_vol_geom& vg, int for_bp) {
  esb_constants c;
  esb_set_constant_values(&g, &vg, r->aniso, r->anisoInv, for_bp, &c);
  return to_kconst(c);
}

// CTF chain of one slab on `img` (W x H): optional in-place crop, pad to the
// N x N square, R2C, CTF (FP or Wiener BP), C2R, scale 1/N^2, crop, and write
// to `out` and/or accumulate into `accum` (Reconstructor.cpp:559-583, 952-965).
static int rec_ctf_chain(esb_reconstructor* r, float* img, int crop_in, const int* p_in, int index, float dmin,
                         float dmax, int for_fp, float* out, float* accum, int crop_out, const int* p_out,
                         int transpose_out = 0) {
  const esb_recon_config& cf = r->cfg;
  const int W = cf.proj_x, H = cf.proj_y, N = r->N;
  PhaseScope ps(r, 2);
  float2 cut = make_float2(cf.cut_length[0], cf.cut_length[1]);
  float2 dim = make_float2(cf.dim_length[0], cf.dim_length[1]);
  ESB_CK(launch_crop_to_square(W, H, W, img, crop_in, cut, dim, p_in, N, r->square_d, r->borderX, r->borderY, r->stream),
         "ctf chain");
  ESB_FFT(cufftExecR2C(r->r2c, (cufftReal*)r->square_d, (cufftComplex*)r->fft_d), "ctf chain R2C");
  float4 beta = make_float4(cf.ctf_beta_fac[0], cf.ctf_beta_fac[1], cf.ctf_beta_fac[2], cf.ctf_beta_fac[3]);
  ESB_CK(launch_ctf(r->fft_d, N, r->ctfk, dmin, dmax, r->defocus[3 * index + 2], for_fp, cf.phase_flip_only,
                    cf.wiener_noise_level, beta, r->stream), "ctf chain");
  ESB_FFT(cufftExecC2R(r->c2r, (cufftComplex*)r->fft_d, (cufftReal*)r->square_d), "ctf chain C2R");
  ESB_CK(launch_square_to_image(r->square_d, N, r->squareShift, 1.0f / ((float)N * (float)N), W, H, W, out, accum,
                                crop_out, cut, dim, p_out, r->stream, transpose_out), "ctf chain");
  return ESB_OK;
}

// Slab boundaries of projection `index`: the reference's loop
// for (ray = t_in; ray < t_out; ray += thickness/pixelsize) with its float
// recurrence (Reconstructor.cpp:515, 935).
static int rec_slab_table(esb_reconstructor* r, const esb_vol_geom* vg, int index, SlabTable& T) {
  float t_in, t_out;
  esb_defocus_distances(&r->geoms[index], vg, r->cfg.proj_x, r->cfg.proj_y, &t_in, &t_out);
  const float step = r->cfg.ctf_slice_thickness_nm / r->cfg.pixel_size_nm;
  int K = 0;
  float ray = t_in;
  for (; ray < t_out; ray += step) {
    if (K >= ESB_MAX_SLABS) return fail(ESB_ERR_UNSUPPORTED, "more than 256 CTF slabs in one projection");
    T.bound[K++] = ray;
  }
  T.bound[K] = ray;  // = bound[K-1] + step, the last slab's upper limit
  T.count = K;
  return ESB_OK;
}

static int rec_slab_capacity(esb_reconstructor* r, int count) {
  if ((size_t)count <= r->slab_cap) return ESB_OK;
  cudaFree(r->slab_imgs);
  r->slab_imgs = nullptr;
  r->slab_cap = 0;
  const size_t bytes = (size_t)count * r->cfg.proj_x * r->cfg.proj_y * sizeof(float);
  ESB_CK(cudaMalloc(&r->slab_imgs, bytes), "slab images");
  r->slab_cap = count;
  return ESB_OK;
}

// Chunk buffers of the batched CTF chains: `want` spectra and squares.
static int rec_batch_buffers(esb_reconstructor* r, int want) {
  const int N = r->N;
  if (want <= r->batch_slabs) return ESB_OK;
  const size_t spec = (size_t)(N / 2 + 1) * N * 2, sq = (size_t)N * N;
  ESB_CK(cudaStreamSynchronize(r->stream), "CTF slab buffers");
  cudaFree(r->spec_batch);
  cudaFree(r->sq_batch);
  r->spec_batch = r->sq_batch = nullptr;
  r->batch_slabs = 0;
  ESB_CK(cudaMalloc(&r->spec_batch, (size_t)want * spec * sizeof(float)), "CTF slab buffers");
  ESB_CK(cudaMalloc(&r->sq_batch, (size_t)want * sq * sizeof(float)), "CTF slab buffers");
  r->batch_slabs = want;
  return ESB_OK;
}

// Batched N x N transforms of `cnt` squares / spectra (one plan per count).
static int rec_fft_many(esb_reconstructor* r, int cnt, bool forward) {
  const int N = r->N;
  cufftHandle* plans = forward ? r->r2c_many : r->c2r_many;
  bool* ok = forward ? r->r2c_many_ok : r->c2r_many_ok;
  if (!ok[cnt]) {
    int dims[2] = {N, N};
    ESB_FFT(cufftPlanMany(&plans[cnt], 2, dims, nullptr, 1, 0, nullptr, 1, 0, forward ? CUFFT_R2C : CUFFT_C2R, cnt),
            "CTF slab plan");
    ok[cnt] = true;
    ESB_FFT(cufftSetStream(plans[cnt], r->stream), "CTF slab plan");
  }
  if (forward)
    ESB_FFT(cufftExecR2C(plans[cnt], (cufftReal*)r->sq_batch, (cufftComplex*)r->spec_batch), "CTF slab R2C");
  else
    ESB_FFT(cufftExecC2R(plans[cnt], (cufftComplex*)r->spec_batch, (cufftReal*)r->sq_batch), "CTF slab C2R");
  return ESB_OK;
}

// The CTF chain of rec_ctf_chain for every slab of table T, ESB_CTF_SLAB_BATCH
// slabs per batched transform. Inputs: the slab images (seq_crop = 0,
// images + k * img, cropped in place when crop_in) or one image cropped again
// before every slab (seq_crop = 1, the back-projection's residual). Outputs:
// image k written to out + k * img (transposed when transpose_out) and/or
// all slabs added to accum in slab order.
static int rec_ctf_chain_slabs(esb_reconstructor* r, const SlabTable& T, int index, float* images, int seq_crop,
                               int crop_in, const int* p_in, int for_fp, float* out, float* accum, int crop_out,
                               const int* p_out, int transpose_out) {
  const esb_recon_config& cf = r->cfg;
  const int W = cf.proj_x, H = cf.proj_y, N = r->N;
  const size_t img = (size_t)W * H, spec = (size_t)(N / 2 + 1) * N * 2, sq = (size_t)N * N;
  int rc;
  if ((rc = rec_batch_buffers(r, std::min(T.count, ESB_CTF_SLAB_BATCH)))) return rc;
  const float2 cut = make_float2(cf.cut_length[0], cf.cut_length[1]);
  const float2 dim = make_float2(cf.dim_length[0], cf.dim_length[1]);
  const float4 beta = make_float4(cf.ctf_beta_fac[0], cf.ctf_beta_fac[1], cf.ctf_beta_fac[2], cf.ctf_beta_fac[3]);
  PhaseScope ps(r, 2);
  for (int c0 = 0; c0 < T.count; c0 += ESB_CTF_SLAB_BATCH) {
    const int cnt = std::min(ESB_CTF_SLAB_BATCH, T.count - c0);
    CtfSlabs S;
    S.count = cnt;
    for (int j = 0; j < cnt; ++j)
      esb_defocus_min_max(T.bound[c0 + j], r->defocus[3 * index], r->defocus[3 * index + 1], r->tilt[index],
                          cf.add_tilt_angle, cf.pixel_size_nm, cf.ctf_slice_thickness_nm, cf.volume_shift[2],
                          cf.ignore_z_shift_for_ctf, cf.switch_ctf_direction, &S.d0[j], &S.d1[j]);
    ESB_CK(launch_crop_to_square_batch(W, H, seq_crop ? images : images + (size_t)c0 * img, img, cnt, crop_in, seq_crop,
                                       cut, dim, p_in, N, r->sq_batch, sq, r->borderX, r->borderY, r->stream),
           "CTF slab chain");
    if ((rc = rec_fft_many(r, cnt, true))) return rc;
    ESB_CK(launch_ctf_batch(r->spec_batch, spec, N, r->ctfk, S, r->defocus[3 * index + 2], for_fp,
                            cf.phase_flip_only, cf.wiener_noise_level, beta, r->stream), "CTF slab chain");
    if ((rc = rec_fft_many(r, cnt, false))) return rc;
    ESB_CK(launch_square_to_image_many(r->sq_batch, sq, cnt, N, r->squareShift, 1.0f / ((float)N * (float)N), W, H,
                                       out ? out + (size_t)c0 * img : nullptr, img, accum, crop_out, cut, dim, p_out,
                                       transpose_out, r->stream), "CTF slab chain");
  }
  return ESB_OK;
}

// Wiener-filtered slab images of prepared projection `index` for the
// sub-volume paths, into slab_imgs (transposed). The reference pads,
// transforms, filters and transforms back the same projection once per slab
// (Reconstructor.cpp:975-1004, no crop). Here the projection is padded and
// transformed once; each chunk of up to ESB_CTF_SLAB_BATCH slabs gets its
// filtered spectra in one launch, one batched C2R and one batched
// scale + window + transpose.
static int rec_subvol_slab_images(esb_reconstructor* r, const esb_vol_geom* full_vol, const float* proj, int index,
                                  SlabTable& T) {
  const esb_recon_config& cf = r->cfg;
  const int W = cf.proj_x, H = cf.proj_y, N = r->N;
  int rc;
  if ((rc = rec_slab_table(r, full_vol, index, T))) return rc;
  if ((rc = rec_slab_capacity(r, T.count))) return rc;
  if ((rc = rec_batch_buffers(r, std::min(T.count, ESB_CTF_SLAB_BATCH)))) return rc;
  const size_t spec = (size_t)(N / 2 + 1) * N * 2;
  static const int none[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const size_t img = (size_t)W * H;
  PhaseScope ps(r, 2);
  ESB_CK(launch_crop_to_square(W, H, W, const_cast<float*>(proj), 0, make_float2(0.f, 0.f), make_float2(0.f, 0.f), none,
                               N, r->square_d, r->borderX, r->borderY, r->stream), "CTF slab images");
  ESB_FFT(cufftExecR2C(r->r2c, (cufftReal*)r->square_d, (cufftComplex*)r->fft_d), "CTF slab images R2C");
  const float4 beta = make_float4(cf.ctf_beta_fac[0], cf.ctf_beta_fac[1], cf.ctf_beta_fac[2], cf.ctf_beta_fac[3]);
  for (int c0 = 0; c0 < T.count; c0 += ESB_CTF_SLAB_BATCH) {
    const int cnt = std::min(ESB_CTF_SLAB_BATCH, T.count - c0);
    CtfSlabs S;
    S.count = cnt;
    for (int j = 0; j < cnt; ++j)
      esb_defocus_min_max(T.bound[c0 + j], r->defocus[3 * index], r->defocus[3 * index + 1], r->tilt[index],
                          cf.add_tilt_angle, cf.pixel_size_nm, cf.ctf_slice_thickness_nm, cf.volume_shift[2],
                          cf.ignore_z_shift_for_ctf, cf.switch_ctf_direction, &S.d0[j], &S.d1[j]);
    ESB_CK(launch_ctf_slabs(r->fft_d, r->spec_batch, spec, N, r->ctfk, S, r->defocus[3 * index + 2], 0,
                            cf.phase_flip_only, cf.wiener_noise_level, beta, r->stream), "CTF slab images");
    if ((rc = rec_fft_many(r, cnt, false))) return rc;
    ESB_CK(launch_square_to_image_batch(r->sq_batch, cnt, N, r->squareShift, 1.0f / ((float)N * (float)N), W, H, W,
                                        r->slab_imgs + (size_t)c0 * img, img, 1, r->stream), "CTF slab images");
  }
  return ESB_OK;
}

// Pre-samples `count` transposed slab images for the back-projection
// (launch_upsample); returns NULL when the geometry does not allow it
// (oversampling not a power of two, magnification anisotropy) or the
// images would exceed 8 GiB, and the back-projection then filters the slab
// images itself. `up_stride` receives the (value, row) pairs per image.
static const float2* rec_upsample(esb_reconstructor* r, const KConst& c, int count, int linear, size_t& up_stride) {
  const esb_recon_config& cf = r->cfg;
  const int os = cf.oversampling;
  up_stride = (size_t)cf.proj_x * os * (size_t)cf.proj_y * os;
  const size_t need = up_stride * (size_t)count;
  if (!bp_can_upsample(c, os) || need * sizeof(float2) > ((size_t)8 << 30)) return nullptr;
  if (need > r->up_cap) {
    if (cudaStreamSynchronize(r->stream) != cudaSuccess) return nullptr;
    cudaFree(r->up_imgs);
    r->up_imgs = nullptr;
    r->up_cap = 0;
    if (cudaMalloc(&r->up_imgs, need * sizeof(float2)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    r->up_cap = need;
  }
  const size_t img = (size_t)cf.proj_x * cf.proj_y;
  if (launch_upsample(c, r->slab_imgs, img, count, cf.proj_x, cf.proj_y, os, linear, r->up_imgs, up_stride,
                      r->stream) != cudaSuccess)
    return nullptr;
  return r->up_imgs;
}

// ForwardProjection / ForwardProjectionROI (Reconstructor.cpp:428-644,
// 649-859): rays of the detector region roi (NULL: the whole detector) are
// projected and added to proj_d; dist_d gets their traversal lengths. With
// CTF every slab image is filtered over the whole detector.
static int rec_forward(esb_reconstructor* r, const esb_vol_geom* vg, const void* vol, int voxel_type, int index,
                       int volume_is_empty, const int* roi_in, const char* where) {
  int rc;
  if ((rc = rec_check(r, vg, index, where))) return rc;
  if (!vol || !valid_vt(voxel_type)) return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": invalid volume");
  const esb_recon_config& cf = r->cfg;
  const int W = cf.proj_x, H = cf.proj_y;
  int roi[4] = {0, 0, W, H};
  if (roi_in) {
    roi[0] = std::max(roi_in[0], 0);
    roi[1] = std::max(roi_in[1], 0);
    roi[2] = std::min(roi_in[2], W);
    roi[3] = std::min(roi_in[3], H);
    if (roi[2] <= roi[0] || roi[3] <= roi[1]) return ok();  // no ray in the region
  }
  KConst c = rec_const(r, r->geoms[index], *vg, 0);
  if (volume_is_empty) {  // Reconstructor.cpp:465-470 / 622-627
    PhaseScope ps(r, 0);
    ESB_CK(launch_travlen(c, r->dist_d, W, roi[0], roi[1], roi[2], roi[3], r->stream), where);
    return ok();
  }
  if (!cf.ctf_mode) {  // ForwardProjectionNoCTF (Reconstructor.cpp:429-438)
    PhaseScope ps(r, 0);
    ESB_CK(rec_march(r, c, vol, voxel_type, roi), where);
    return ok();
  }
  // ForwardProjectionCTF (Reconstructor.cpp:496-590)
  float t_in, t_out;
  esb_defocus_distances(&r->geoms[index], vg, W, H, &t_in, &t_out);
  const float step = cf.ctf_slice_thickness_nm / cf.pixel_size_nm;
  const int full[8] = {0, H - 1, W - 1, H - 1, 0, 0, W - 1, 0};  // pA, pB, pC, pD (Reconstructor.cpp:559-566)
  if (cf.variant == ESB_VARIANT_FAST) {
    // all slabs in one slicer launch, then the CTF chain per slab image
    SlabTable T;
    if ((rc = rec_slab_table(r, vg, index, T))) return rc;
    if ((rc = rec_slab_capacity(r, T.count))) return rc;
    const size_t img = (size_t)W * H;
    {
      PhaseScope ps(r, 3);
      ESB_CK(cudaMemsetAsync(r->slab_imgs, 0, (size_t)T.count * img * sizeof(float), r->stream),
             where);
    }
    {
      PhaseScope ps(r, 0);
      const int nw = rec_slicer_nw(r, c, vol, voxel_type, img, T);
      ESB_CK(launch_slicer_fused(c, vol, voxel_type, r->slab_imgs, img, W, T, roi[0], roi[1], roi[2], roi[3],
                                 r->stream, nw),
             where);
    }
    // each slab image through the CTF, added to proj_d in slab order
    if ((rc = rec_ctf_chain_slabs(r, T, index, r->slab_imgs, 0, 1, full, 1, nullptr, r->proj_d, 1, full, 0))) return rc;
  }
  for (float ray = t_in; cf.variant != ESB_VARIANT_FAST && ray < t_out; ray += step) {
    float dmin, dmax;
    esb_defocus_min_max(ray, r->defocus[3 * index], r->defocus[3 * index + 1], r->tilt[index], cf.add_tilt_angle,
                        cf.pixel_size_nm, cf.ctf_slice_thickness_nm, cf.volume_shift[2], cf.ignore_z_shift_for_ctf,
                        cf.switch_ctf_direction, &dmin, &dmax);
    {
      PhaseScope ps(r, 3);
      ESB_CK(cudaMemsetAsync(r->dist_d, 0, (size_t)W * H * sizeof(float), r->stream), where);
    }
    {
      PhaseScope ps(r, 0);
      ESB_CK(rec_slicer(r, c, vol, voxel_type, r->dist_d, ray, ray + step, roi), where);
    }
    if ((rc = rec_ctf_chain(r, r->dist_d, 1, full, index, dmin, dmax, 1, nullptr, r->proj_d, 1, full))) return rc;
  }
  {
    PhaseScope ps(r, 3);
    ESB_CK(cudaMemsetAsync(r->dist_d, 0, (size_t)W * H * sizeof(float), r->stream), where);
  }
  PhaseScope ps(r, 0);
  ESB_CK(launch_travlen(c, r->dist_d, W, roi[0], roi[1], roi[2], roi[3], r->stream), where);
  return ok();
}

extern "C" {

int esb_rec_forward_projection(esb_reconstructor* r, const esb_vol_geom* vg, const void* vol, int voxel_type, int index,
                               int volume_is_empty) {
  return rec_forward(r, vg, vol, voxel_type, index, volume_is_empty, nullptr, "esb_rec_forward_projection");
}

int esb_rec_forward_projection_roi(esb_reconstructor* r, const esb_vol_geom* vg, const void* vol, int voxel_type,
                                   int index, int volume_is_empty, const int roi[4]) {
  if (!roi) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_forward_projection_roi: roi is NULL");
  return rec_forward(r, vg, vol, voxel_type, index, volume_is_empty, roi, "esb_rec_forward_projection_roi");
}

int esb_rec_compare(esb_reconstructor* r, const esb_vol_geom* vg, const float* real, int index) {
  int rc;
  if ((rc = rec_check(r, vg, index, "esb_rec_compare"))) return rc;
  if (!real) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_compare: real is NULL");
  const esb_recon_config& cf = r->cfg;
  // Reconstructor::Compare (Reconstructor.cpp:1386-1405)
  const float DIST = -10000.0f;
  float zdir = r->geoms[index].proj_norm[2];
  float zmin = vg->full_bbox_min[2], zmax = vg->full_bbox_max[2];
  float len = fabsf((DIST - zmin) / zdir - (DIST - zmax) / zdir);
  PhaseScope ps(r, 3);
  ESB_CK(launch_compare(cf.proj_x, cf.proj_y, cf.proj_x, real, r->proj_d, r->dist_d, len,
                        make_float4(cf.crop[0], cf.crop[1], cf.crop[2], cf.crop[3]),
                        make_float4(cf.crop_dim[0], cf.crop_dim[1], cf.crop_dim[2], cf.crop_dim[3]),
                        cf.projection_scale_factor, r->stream), "esb_rec_compare");
  return ok();
}

}  // extern "C"

// BackProjection of image `img` (Reconstructor.cpp:871-887 and 920-969).
static int rec_back_project_image(esb_reconstructor* r, const esb_vol_geom* vg, void* vol, int voxel_type, int index,
                                  float sirt_count, float* img) {
  const esb_recon_config& cf = r->cfg;
  const int W = cf.proj_x, H = cf.proj_y;
  int p[8];
  esb_compute_hit_points(&r->geoms[index], vg, p);
  KConst c = rec_const(r, r->geoms[index], *vg, 1);
  const float lambda = cf.lambda / sirt_count;
  if (!cf.ctf_mode) {
    {
      PhaseScope ps(r, 3);
      ESB_CK(launch_crop_border(W, H, W, img, make_float2(cf.cut_length[0], cf.cut_length[1]),
                                make_float2(cf.dim_length[0], cf.dim_length[1]), p, r->stream), "back projection");
    }
    if (cf.variant == ESB_VARIANT_FAST) {
      int rc2;
      if ((rc2 = rec_slab_capacity(r, 1))) return rc2;
      {
        PhaseScope ps(r, 3);
        ESB_CK(launch_transpose(img, W, H, W, r->slab_imgs, r->stream), "back projection");
      }
      SlabTable none;
      none.count = 0;
      PhaseScope ps(r, 1);
      size_t up_stride = 0;
      const float2* up = rec_upsample(r, c, 1, 0, up_stride);
      ESB_CK(cudaGetLastError(), "back projection");
      const BpShape shape = rec_bp_shape(r, c, voxel_type, r->slab_imgs, 0, none, 0, up, up_stride);
      ESB_CK(launch_bp_fast_slabs(c, vol, voxel_type, r->slab_imgs, 0, none, W, H, W, lambda, cf.oversampling, 0.0f,
                                  9999999999999.0f, 0, r->stream, 1, up, up_stride, &shape), "back projection");
      return ESB_OK;
    }
    PhaseScope ps(r, 1);
    ESB_CK(rec_bp(r, c, vol, voxel_type, img, lambda, 0.0f, 9999999999999.0f, 0), "back projection");
    return ESB_OK;
  }
  float t_in, t_out;
  esb_defocus_distances(&r->geoms[index], vg, W, H, &t_in, &t_out);
  const float step = cf.ctf_slice_thickness_nm / cf.pixel_size_nm;
  int rc;
  if (cf.variant == ESB_VARIANT_FAST) {
    // Wiener-filtered image per slab, then one back-projection launch that
    // picks each quad's slab image by its first-corner depth
    SlabTable T;
    if ((rc = rec_slab_table(r, vg, index, T))) return rc;
    if ((rc = rec_slab_capacity(r, T.count))) return rc;
    // cropBorder(proj_d) is re-applied to the residual on every slab (:954)
    if ((rc = rec_ctf_chain_slabs(r, T, index, img, 1, 1, p, 0, r->slab_imgs, nullptr, 1, p, 1))) return rc;
    PhaseScope ps(r, 1);
    size_t up_stride = 0;
    const float2* up = rec_upsample(r, c, T.count, 1, up_stride);
    ESB_CK(cudaGetLastError(), "back projection");
    const BpShape shape = rec_bp_shape(r, c, voxel_type, r->slab_imgs, (size_t)W * H, T, 1, up, up_stride);
    ESB_CK(launch_bp_fast_slabs(c, vol, voxel_type, r->slab_imgs, (size_t)W * H, T, W, H, W, lambda, cf.oversampling,
                                0.f, 0.f, 1, r->stream, 1, up, up_stride, &shape), "back projection");
    return ESB_OK;
  }
  for (float ray = t_in; ray < t_out; ray += step) {
    float dmin, dmax;
    esb_defocus_min_max(ray, r->defocus[3 * index], r->defocus[3 * index + 1], r->tilt[index], cf.add_tilt_angle,
                        cf.pixel_size_nm, cf.ctf_slice_thickness_nm, cf.volume_shift[2], cf.ignore_z_shift_for_ctf,
                        cf.switch_ctf_direction, &dmin, &dmax);
    // cropBorder(proj_d) is re-applied to the residual on every slab (:954)
    if ((rc = rec_ctf_chain(r, img, 1, p, index, dmin, dmax, 0, r->dist_d, nullptr, 1, p))) return rc;
    PhaseScope ps(r, 1);
    ESB_CK(rec_bp(r, c, vol, voxel_type, r->dist_d, lambda, ray, ray + step, 1), "back projection");
  }
  return ESB_OK;
}

// The back-projections of one ordered subset (EmSart.cpp:649-673) in one
// pass over the volume per chunk (launch_bp_axis_set): each projection's
// residual is cropped or CTF-filtered per slab and pre-sampled exactly as
// rec_back_project_image does it, into its own part of the pre-sampled image
// buffer; a chunk is as many consecutive projections as fit ESB_BP_SET_MAX and
// the buffer cap. `done` stays false (nothing launched) when a projection
// cannot join (faithful kernels, geometry without the single-axis kernel or
// pre-sampling, too many slabs); the caller then back-projects each one.
static int rec_back_project_subset(esb_reconstructor* r, const esb_vol_geom* vg, void* vol, int voxel_type,
                                   const int* indices, int n, float sirt_count, float* const* imgs, bool& done) {
  done = false;
  const esb_recon_config& cf = r->cfg;
  const bool on = r->fuse_subsets > 0 || (r->fuse_subsets < 0 && voxel_type != ESB_VOXEL_F32);
  if (!on || cf.variant != ESB_VARIANT_FAST || n < 2) return ESB_OK;
  const int W = cf.proj_x, H = cf.proj_y, os = cf.oversampling;
  const size_t img = (size_t)W * H, up_stride = (size_t)W * os * (size_t)H * os;
  const size_t cap_images = std::max<size_t>(1, ((size_t)16 << 30) / (up_stride * sizeof(float2)));
  std::vector<KConst> ks(n);
  std::vector<SlabTable> T(n);
  std::vector<int> cnt(n);
  int rc;
  for (int j = 0; j < n; ++j) {
    ks[j] = rec_const(r, r->geoms[indices[j]], *vg, 1);
    T[j].count = 0;
    if (cf.ctf_mode && (rc = rec_slab_table(r, vg, indices[j], T[j]))) return rc;
    cnt[j] = cf.ctf_mode ? T[j].count : 1;
    if (!bp_set_eligible(ks[j], os, T[j].count) || (size_t)cnt[j] > cap_images) return ESB_OK;
  }
  // chunks of consecutive projections: [first, first + size)
  std::vector<std::pair<int, int>> chunks;
  size_t most = 0;
  for (int j = 0; j < n;) {
    int m = 0;
    size_t tot = 0;
    while (j + m < n && m < ESB_BP_SET_MAX && tot + cnt[j + m] <= cap_images) tot += cnt[j + m++];
    chunks.emplace_back(j, m);
    most = std::max(most, tot);
    j += m;
  }
  const size_t need = most * up_stride;
  if (need > r->up_cap) {
    ESB_CK(cudaStreamSynchronize(r->stream), "subset back projection");
    cudaFree(r->up_imgs);
    r->up_imgs = nullptr;
    r->up_cap = 0;
    ESB_CK(cudaMalloc(&r->up_imgs, need * sizeof(float2)), "subset back projection");
    r->up_cap = need;
  }
  done = true;
  const float lambda = cf.lambda / sirt_count;
  for (const auto& ch : chunks) {
    const float2* ups[ESB_BP_SET_MAX];
    size_t off = 0;
    for (int j = ch.first; j < ch.first + ch.second; ++j) {
      const int index = indices[j];
      int p[8];
      esb_compute_hit_points(&r->geoms[index], vg, p);
      float2* up = r->up_imgs + off * up_stride;
      if (cf.ctf_mode) {
        if ((rc = rec_slab_capacity(r, T[j].count))) return rc;
        // cropBorder(proj_d) is re-applied to the residual on every slab (:954)
        if ((rc = rec_ctf_chain_slabs(r, T[j], index, imgs[j], 1, 1, p, 0, r->slab_imgs, nullptr, 1, p, 1))) return rc;
        PhaseScope ps(r, 1);
        ESB_CK(launch_upsample(ks[j], r->slab_imgs, img, T[j].count, W, H, os, 1, up, up_stride, r->stream),
               "subset back projection");
      } else {
        if ((rc = rec_slab_capacity(r, 1))) return rc;
        PhaseScope ps(r, 3);
        ESB_CK(launch_crop_border(W, H, W, imgs[j], make_float2(cf.cut_length[0], cf.cut_length[1]),
                                  make_float2(cf.dim_length[0], cf.dim_length[1]), p, r->stream),
               "subset back projection");
        ESB_CK(launch_transpose(imgs[j], W, H, W, r->slab_imgs, r->stream), "subset back projection");
        ESB_CK(launch_upsample(ks[j], r->slab_imgs, img, 1, W, H, os, 0, up, up_stride, r->stream),
               "subset back projection");
      }
      ups[j - ch.first] = up;
      off += cnt[j];
    }
    PhaseScope ps(r, 1);
    const int f = ch.first;
    const BpShape shape =
        rec_bp_shape(r, ks[f], voxel_type, r->slab_imgs, img, T[f], cf.ctf_mode ? 1 : 0, ups[0], up_stride);
    ESB_CK(launch_bp_axis_set(&ks[f], ups, &T[f], ch.second, up_stride, vol, voxel_type, W, H, lambda, os, &shape,
                              r->stream),
           "subset back projection");
  }
  return ESB_OK;
}

extern "C" {

int esb_rec_back_projection(esb_reconstructor* r, const esb_vol_geom* vg, void* vol, int voxel_type, int index,
                            float sirt_count) {
  int rc;
  if ((rc = rec_check(r, vg, index, "esb_rec_back_projection"))) return rc;
  if (!vol || !valid_vt(voxel_type) || !(sirt_count > 0))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_back_projection: invalid argument");
  return rec_back_project_image(r, vg, vol, voxel_type, index, sirt_count, r->proj_d);
}

}  // extern "C"

// One SART iteration of EmSart.cpp:579-675: ordered subsets of sirt_count
// projections, {FP, compare} for each, then {BP} for each.
static int sart_iteration(esb_reconstructor* r, const esb_vol_geom* vg, void* vol, int voxel_type,
                          const float* projections, const int* index_list, int proj_count, int sirt_count,
                          int* volume_is_empty) {
  const size_t img = (size_t)r->cfg.proj_x * r->cfg.proj_y;
  int rc;
  const int steps = (proj_count + sirt_count - 1) / sirt_count;
  for (int s = 0; s < steps; ++s) {
    for (int i = 0; i < sirt_count; ++i) {
      if (s * sirt_count + i >= proj_count) continue;
      const int index = index_list[s * sirt_count + i];
      if ((rc = esb_rec_reset_projections(r))) return rc;
      if ((rc = esb_rec_forward_projection(r, vg, vol, voxel_type, index, *volume_is_empty))) return rc;
      if ((rc = esb_rec_compare(r, vg, projections + (size_t)index * img, index))) return rc;
      ESB_CK(cudaMemcpyAsync(r->sirt_d[i], r->proj_d, img * sizeof(float), cudaMemcpyDeviceToDevice, r->stream),
             "esb_sart_run");
    }
    const int in_subset = std::min(sirt_count, proj_count - s * sirt_count);
    bool fused = false;
    if ((rc = rec_back_project_subset(r, vg, vol, voxel_type, index_list + s * sirt_count, in_subset,
                                      (float)sirt_count, r->sirt_d.data(), fused)))
      return rc;
    if (fused) *volume_is_empty = 0;
    for (int i = 0; i < sirt_count && !fused; ++i) {
      if (s * sirt_count + i >= proj_count) continue;
      *volume_is_empty = 0;
      const int index = index_list[s * sirt_count + i];
      if ((rc = rec_back_project_image(r, vg, vol, voxel_type, index, (float)sirt_count, r->sirt_d[i]))) return rc;
    }
  }
  return ESB_OK;
}

extern "C" {

int esb_prepare_projection(esb_reconstructor* r, const esb_prepare_config* pc, const void* in, float* out,
                           float* mean_out, float* std_out, int* bad_out) {
  if (!r || !pc || !in || !out) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_prepare_projection: NULL argument");
  if (pc->input_type < ESB_PIX_F32 || pc->input_type > ESB_PIX_U32 || pc->normalization < ESB_PNM_MEAN ||
      pc->normalization > ESB_PNM_NONE || pc->wbp_filter < 0 || pc->wbp_filter > 4)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_prepare_projection: invalid mode");
  const int W = r->cfg.proj_x, H = r->cfg.proj_y, N = r->N;
  const long npx = (long)W * H, nsq = (long)N * N;
  cudaStream_t st = r->stream;
  // buffers (the CTF configuration already owns a square, a spectrum and plans)
  if (!r->prep_img) ESB_CK(cudaMalloc(&r->prep_img, npx * sizeof(float)), "esb_prepare_projection");
  if (!r->prep_stats) ESB_CK(cudaMalloc(&r->prep_stats, 4 * sizeof(double)), "esb_prepare_projection");
  float* sq = r->square_d;
  float* spec = r->fft_d;
  cufftHandle r2c = r->r2c, c2r = r->c2r;
  if (!r->plans) {
    if (!r->prep_sq) ESB_CK(cudaMalloc(&r->prep_sq, nsq * sizeof(float)), "esb_prepare_projection");
    if (!r->prep_fft) ESB_CK(cudaMalloc(&r->prep_fft, (size_t)(N / 2 + 1) * N * 2 * sizeof(float)), "esb_prepare_projection");
    if (!r->prep_plans) {
      ESB_FFT(cufftPlan2d(&r->prep_r2c, N, N, CUFFT_R2C), "esb_prepare_projection");
      ESB_FFT(cufftPlan2d(&r->prep_c2r, N, N, CUFFT_C2R), "esb_prepare_projection");
      r->prep_plans = true;
    }
    sq = r->prep_sq;
    spec = r->prep_fft;
    r2c = r->prep_r2c;
    c2r = r->prep_c2r;
  }
  ESB_FFT(cufftSetStream(r2c, st), "esb_prepare_projection");
  ESB_FFT(cufftSetStream(c2r, st), "esb_prepare_projection");
  double h[4];
  auto stats = [&](const float* img, size_t pitchE, int x0, int y0, int w, int hh) -> int {
    ESB_CK(cudaMemsetAsync(r->prep_stats, 0, 2 * sizeof(double), st), "esb_prepare_projection");
    ESB_CK(launch_window_stats(img, pitchE, x0, y0, w, hh, r->prep_stats, st), "esb_prepare_projection");
    ESB_CK(cudaMemcpyAsync(h, r->prep_stats, 2 * sizeof(double), cudaMemcpyDeviceToHost, st), "esb_prepare_projection");
    ESB_CK(cudaStreamSynchronize(st), "esb_prepare_projection");
    return ESB_OK;
  };
  int rc;
  // convert, pad (cts with fillZero = false, mirrorY for DM4: Reconstructor.cpp:1192-1204)
  ESB_CK(launch_convert_input(in, pc->input_type, npx, out, st), "esb_prepare_projection");
  ESB_CK(launch_make_square(W, H, W, out, N, sq, r->borderX, r->borderY, pc->mirror_y, 0, st), "esb_prepare_projection");
  if ((rc = stats(sq, N, 0, 0, N, N))) return rc;
  float meanValue = (float)(h[0] / (double)nsq);
  // bad pixels (:1212-1227)
  int bad = 0;
  if (pc->correct_bad_pixels) {
    ESB_CK(cudaMemsetAsync(r->prep_stats + 2, 0, sizeof(double), st), "esb_prepare_projection");
    ESB_CK(launch_bad_pixels(sq, nsq, pc->bad_pixel_value * meanValue, meanValue, r->prep_stats + 2, st),
           "esb_prepare_projection");
    ESB_CK(cudaMemcpyAsync(h + 2, r->prep_stats + 2, sizeof(double), cudaMemcpyDeviceToHost, st),
           "esb_prepare_projection");
    ESB_CK(cudaStreamSynchronize(st), "esb_prepare_projection");
    bad = (int)h[2];
  }
  float stdValue = 0.f;
  auto mean_std = [&](double s, double q, double n, float& m, float& sd) {
    const double mu = s / n;
    double var = q / n - mu * mu;
    m = (float)mu;
    sd = (float)sqrt(var > 0.0 ? var : 0.0);
  };
  if (pc->wbp) {  // statistics of the raw window (:1231-1270)
    ESB_CK(launch_window_div(sq, r->squareShift, N, W, H, 1.0f, r->prep_img, st), "esb_prepare_projection");
    if ((rc = stats(r->prep_img, W, 0, 0, W, H))) return rc;
    mean_std(h[0], h[1], (double)npx, meanValue, stdValue);
    float std_hf = stdValue, mean_hf = meanValue;
    if (pc->normalization == ESB_PNM_MEAN) std_hf = meanValue;
    if (pc->normalization == ESB_PNM_NONE) {
      std_hf = 1;
      mean_hf = 0;
    }
    if (pc->down_weight_tilts) std_hf /= cosf(fabsf(pc->tilt_deg) / 180.0f * (float)M_PI);
    ESB_CK(launch_normalize(r->prep_img, out, npx, mean_hf, std_hf, st), "esb_prepare_projection");
    ESB_CK(launch_make_square(W, H, W, out, N, sq, r->borderX, r->borderY, 0, 0, st), "esb_prepare_projection");
  }
  float normVal = 1.0f;
  if (!pc->skip_filter || pc->wbp) {  // (:1274-1310)
    ESB_FFT(cufftExecR2C(r2c, (cufftReal*)sq, (cufftComplex*)spec), "esb_prepare_projection R2C");
    if (!pc->skip_filter)
      ESB_CK(launch_fourier_filter(spec, N, pc->lp, pc->hp, pc->lps, pc->hps, st), "esb_prepare_projection");
    if (pc->dose_weighting)
      ESB_CK(launch_dose_weighting(spec, N, pc->accumulated_dose, pc->pixel_size_nm * 10.0f, st),
             "esb_prepare_projection");
    if (pc->wbp) ESB_CK(launch_wbp_weighting(spec, N, pc->psi_deg, pc->wbp_filter, st), "esb_prepare_projection");
    ESB_FFT(cufftExecC2R(c2r, (cufftComplex*)spec, (cufftReal*)sq), "esb_prepare_projection C2R");
    normVal = (float)N * (float)N;
  }
  // normalise from the FFT (:1315-1316)
  ESB_CK(launch_window_div(sq, r->squareShift, N, W, H, normVal, r->prep_img, st), "esb_prepare_projection");
  if (!pc->wbp) {  // SART: statistics of the filtered window (:1320-1372)
    if (pc->normalization == ESB_PNM_NONE) {
      if ((rc = stats(r->prep_img, W, W / 4, H / 4, W / 2, H / 2))) return rc;
      mean_std(h[0], h[1], (double)(W / 2) * (double)(H / 2), meanValue, stdValue);
    } else {
      if ((rc = stats(r->prep_img, W, 0, 0, W, H))) return rc;
      mean_std(h[0], h[1], (double)npx, meanValue, stdValue);
    }
    float std_hf = stdValue, mean_hf = meanValue;
    if (pc->normalization == ESB_PNM_MEAN) std_hf = meanValue;
    if (pc->normalization == ESB_PNM_NONE) std_hf = 1;
    ESB_CK(launch_normalize(r->prep_img, out, npx, mean_hf, std_hf, st), "esb_prepare_projection");
  } else {
    ESB_CK(cudaMemcpyAsync(out, r->prep_img, npx * sizeof(float), cudaMemcpyDeviceToDevice, st),
           "esb_prepare_projection");
  }
  if (mean_out) *mean_out = meanValue;
  if (std_out) *std_out = stdValue;
  if (bad_out) *bad_out = bad;
  return ok();
}

int esb_rec_cc_displacement(esb_reconstructor* r, const float* residual, const float* model, int max_shift,
                            int multi_peak, float* shift_xy, float* cc_value, float* cc_map, float* cc_map_multi) {
  if (!r || !residual || !model || !shift_xy)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_cc_displacement: NULL argument");
  const int W = r->cfg.proj_x, H = r->cfg.proj_y, N = r->N;
  if (max_shift < 1 || 2 * max_shift > N)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_cc_displacement: max_shift must be in [1, N/2] for the N x N square");
  if (N > 65535) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_rec_cc_displacement: square larger than 65535");
  const long nsq = (long)N * N, nspec = (long)(N / 2 + 1) * N;
  cudaStream_t st = r->stream;
  if (!r->cc_sq) ESB_CK(cudaMalloc(&r->cc_sq, 2 * nsq * sizeof(float)), "esb_rec_cc_displacement");
  if (!r->cc_spec) ESB_CK(cudaMalloc(&r->cc_spec, 2 * nspec * 2 * sizeof(float)), "esb_rec_cc_displacement");
  if (!r->cc_red) ESB_CK(cudaMalloc(&r->cc_red, 4 * sizeof(double) + 2 * sizeof(unsigned long long)),
                         "esb_rec_cc_displacement");
  // the N x N plans: the CTF configuration's, else the preparation's
  cufftHandle r2c = r->r2c, c2r = r->c2r;
  if (!r->plans) {
    if (!r->prep_plans) {
      ESB_FFT(cufftPlan2d(&r->prep_r2c, N, N, CUFFT_R2C), "esb_rec_cc_displacement");
      ESB_FFT(cufftPlan2d(&r->prep_c2r, N, N, CUFFT_C2R), "esb_rec_cc_displacement");
      r->prep_plans = true;
    }
    r2c = r->prep_r2c;
    c2r = r->prep_c2r;
  }
  ESB_FFT(cufftSetStream(r2c, st), "esb_rec_cc_displacement");
  ESB_FFT(cufftSetStream(c2r, st), "esb_rec_cc_displacement");
  float *sqA = r->cc_sq, *sqB = r->cc_sq + nsq;
  float *specA = r->cc_spec, *specB = r->cc_spec + 2 * nspec;
  double* sums = (double*)r->cc_red;  // [sum A, sum of squares A, sum B, sum of squares B]
  unsigned long long* keys = (unsigned long long*)(sums + 4);
  ESB_CK(cudaMemsetAsync(r->cc_red, 0, 4 * sizeof(double) + 2 * sizeof(unsigned long long), st),
         "esb_rec_cc_displacement");
  // Reconstructor.cpp:1769-1815: mirror-padded squares centred on their
  // means, sums of squares, spectra
  ESB_CK(launch_make_square(W, H, W, residual, N, sqA, r->borderX, r->borderY, 0, 0, st), "esb_rec_cc_displacement");
  ESB_CK(launch_cc_center(sqA, nsq, sums, st), "esb_rec_cc_displacement");
  ESB_FFT(cufftExecR2C(r2c, (cufftReal*)sqA, (cufftComplex*)specA), "esb_rec_cc_displacement R2C");
  ESB_CK(launch_make_square(W, H, W, model, N, sqB, r->borderX, r->borderY, 0, 0, st), "esb_rec_cc_displacement");
  ESB_CK(launch_cc_center(sqB, nsq, sums + 2, st), "esb_rec_cc_displacement");
  ESB_FFT(cufftExecR2C(r2c, (cufftReal*)sqB, (cufftComplex*)specB), "esb_rec_cc_displacement R2C");
  // :1817-1866: correlation, normalisation, map, maxShift mask, arg-max
  ESB_CK(launch_cc_conj_mul(specA, specB, nspec, st), "esb_rec_cc_displacement");
  ESB_FFT(cufftExecC2R(c2r, (cufftComplex*)specA, (cufftReal*)sqA), "esb_rec_cc_displacement C2R");
  if (cc_map) ESB_CK(launch_cc_map(sqA, N, max_shift, sums, cc_map, st), "esb_rec_cc_displacement");
  ESB_CK(launch_cc_finish(sqA, N, max_shift, sums, keys, st), "esb_rec_cc_displacement");
  // :1886-1932: the peak nearest the origin among those >= 0.9 x maximum
  if (multi_peak) {
    ESB_CK(launch_cc_peaks(sqA, sqB, N, max_shift, keys, keys + 1, st), "esb_rec_cc_displacement");
    if (cc_map_multi) ESB_CK(launch_cc_map(sqB, N, max_shift, nullptr, cc_map_multi, st), "esb_rec_cc_displacement");
  }
  unsigned long long k[2];
  ESB_CK(cudaMemcpyAsync(k, keys, sizeof(k), cudaMemcpyDeviceToHost, st), "esb_rec_cc_displacement");
  ESB_CK(cudaStreamSynchronize(st), "esb_rec_cc_displacement");
  // key -> value and raster index (the order-preserving map of esb_cc.cu)
  auto value = [](unsigned long long key) {
    if (key == 0ull) return std::numeric_limits<float>::quiet_NaN();
    uint32_t u = (uint32_t)(key >> 32);
    u = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    float v;
    std::memcpy(&v, &u, sizeof(v));
    return v;
  };
  const float maxVal = value(k[0]);
  const unsigned long long kk = multi_peak ? k[1] : k[0];
  const long idx = kk ? (long)(0xFFFFFFFFu - (uint32_t)(kk & 0xFFFFFFFFull)) : 0;
  float sx = (float)(idx % N), sy = (float)(idx / N);
  // :1941-1957: signed shifts; no positive correlation: no shift found
  if (sx > (float)(N / 2)) sx -= (float)N;
  if (sy > (float)(N / 2)) sy -= (float)N;
  if (!(maxVal > 0.0f)) sx = sy = -1000.0f;
  shift_xy[0] = sx;
  shift_xy[1] = sy;
  if (cc_value) *cc_value = maxVal;
  return ok();
}

int esb_sart_run(esb_reconstructor* r, const esb_vol_geom* vg, void* vol, int voxel_type, const float* projections,
                 const int* index_list, int proj_count, int iterations, int sirt_count, int* volume_is_empty) {
  if (!r || !vg || !vol || !projections || !index_list || !volume_is_empty || !valid_vt(voxel_type))
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_sart_run: NULL argument");
  if (proj_count <= 0 || iterations < 0 || sirt_count < 1)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_sart_run: invalid counts");
  for (int i = 0; i < proj_count; ++i)
    if (index_list[i] < 0 || index_list[i] >= r->cfg.n_proj)
      return fail(ESB_ERR_INVALID_ARGUMENT, "esb_sart_run: index list entry out of range");
  const int W = r->cfg.proj_x, H = r->cfg.proj_y;
  const size_t img = (size_t)W * H;
  while ((int)r->sirt_d.size() < sirt_count) {
    float* p = nullptr;
    ESB_CK(cudaMalloc(&p, img * sizeof(float)), "esb_sart_run");
    r->sirt_d.push_back(p);
  }
  int rc;
  int iter = 0;
  if (r->graphs && !r->timing && iterations > 0) {
    // One SART iteration is captured as a CUDA graph and replayed, within
    // this call and by later calls with the same inputs (the graph holds
    // their pointers and geometry). A call with other inputs, or one that
    // starts on an empty volume, first runs an iteration eagerly: it sizes
    // every buffer (slab images, FFT plans) and settles volume_is_empty;
    // the next iteration is then captured (recorded, not run).
    auto& k = r->sart_key;
    const bool same = r->sart_exec && !*volume_is_empty && k.vol == vol && k.voxel_type == voxel_type &&
                      k.projections == projections && k.sirt_count == sirt_count &&
                      memcmp(&k.vg, vg, sizeof(esb_vol_geom)) == 0 && (int)k.index_list.size() == proj_count &&
                      std::equal(k.index_list.begin(), k.index_list.end(), index_list);
    if (!same) {
      if ((rc = sart_iteration(r, vg, vol, voxel_type, projections, index_list, proj_count, sirt_count,
                               volume_is_empty)))
        return rc;
      ++iter;
      if (r->sart_exec) {
        ESB_CK(cudaStreamSynchronize(r->stream), "esb_sart_run");
        cudaGraphExecDestroy(r->sart_exec);
        r->sart_exec = nullptr;
      }
      // The capture records on a private stream (the caller's may be the
      // legacy default stream, which cannot be captured); the graph is then
      // launched on the caller's stream.
      if (!r->capture_stream)
        ESB_CK(cudaStreamCreateWithFlags(&r->capture_stream, cudaStreamNonBlocking), "esb_sart_run capture");
      cudaStream_t user = r->stream;
      if ((rc = esb_reconstructor_set_stream(r, r->capture_stream))) return rc;
      cudaError_t e = cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) {
        esb_reconstructor_set_stream(r, user);
        return cuda_fail(e, "esb_sart_run capture");
      }
      const unsigned long long l0 = g_launches.load();
      rc = sart_iteration(r, vg, vol, voxel_type, projections, index_list, proj_count, sirt_count, volume_is_empty);
      const unsigned long long captured = g_launches.load() - l0;
      cudaGraph_t graph = nullptr;
      e = cudaStreamEndCapture(r->stream, &graph);
      const int rs = esb_reconstructor_set_stream(r, user);
      if (!rc) rc = rs;
      if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
      }
      ESB_CK(e, "esb_sart_run capture");
      const cudaError_t ei = cudaGraphInstantiate(&r->sart_exec, graph, 0);
      cudaGraphDestroy(graph);
      ESB_CK(ei, "esb_sart_run instantiate");
      // the captured launches run when the graph does: counted at each replay
      g_launches.fetch_sub(captured);
      r->sart_graph_launches = captured;
      k.vol = vol;
      k.voxel_type = voxel_type;
      k.projections = projections;
      k.vg = *vg;
      k.index_list.assign(index_list, index_list + proj_count);
      k.sirt_count = sirt_count;
    }
    for (; iter < iterations; ++iter) {
      ESB_CK(cudaGraphLaunch(r->sart_exec, r->stream), "esb_sart_run replay");
      count_launches(r->sart_graph_launches);
    }
    return ok();
  }
  for (; iter < iterations; ++iter) {
    if ((rc = sart_iteration(r, vg, vol, voxel_type, projections, index_list, proj_count, sirt_count,
                             volume_is_empty)))
      return rc;
  }
  return ok();
}

int esb_sart_run_zslab(esb_reconstructor* r, const esb_vol_geom* vg, void* vol, int voxel_type,
                       const float* projections, const int* index_list, int proj_count, int iterations, int sirt_count,
                       int* volume_is_empty, esb_allreduce_fn allreduce, void* user) {
  const char* where = "esb_sart_run_zslab";
  if (!r || !vg || !vol || !projections || !index_list || !volume_is_empty || !valid_vt(voxel_type) || !allreduce)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": NULL argument");
  if (proj_count <= 0 || iterations < 0 || sirt_count < 1)
    return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": invalid counts");
  for (int i = 0; i < proj_count; ++i)
    if (index_list[i] < 0 || index_list[i] >= r->cfg.n_proj)
      return fail(ESB_ERR_INVALID_ARGUMENT, std::string(where) + ": index list entry out of range");
  const size_t img = (size_t)r->cfg.proj_x * r->cfg.proj_y;
  while ((int)r->sirt_d.size() < sirt_count) {
    float* p = nullptr;
    ESB_CK(cudaMalloc(&p, img * sizeof(float)), where);
    r->sirt_d.push_back(p);
  }
  int rc;
  const int steps = (proj_count + sirt_count - 1) / sirt_count;
  for (int it = 0; it < iterations; ++it) {
    for (int s = 0; s < steps; ++s) {
      for (int i = 0; i < sirt_count; ++i) {
        if (s * sirt_count + i >= proj_count) continue;
        const int index = index_list[s * sirt_count + i];
        if ((rc = esb_rec_reset_projections(r))) return rc;
        if ((rc = esb_rec_forward_projection(r, vg, vol, voxel_type, index, *volume_is_empty))) return rc;
        // the slab's line integrals and ray lengths, summed over the ranks in
        // one collective on the stream (Reconstructor.cpp:440-463 gathers
        // both on rank 0 and EmSart.cpp:647 broadcasts the residuals; with
        // the sums on every rank each forms the same residual itself)
        if ((rc = allreduce(r->proj_d, 2 * img, (void*)r->stream, user)))
          return fail(ESB_ERR_CUDA, std::string(where) + ": the all-reduce callback returned " + std::to_string(rc));
        if ((rc = esb_rec_compare(r, vg, projections + (size_t)index * img, index))) return rc;
        ESB_CK(cudaMemcpyAsync(r->sirt_d[i], r->proj_d, img * sizeof(float), cudaMemcpyDeviceToDevice, r->stream),
               where);
      }
      const int in_subset = std::min(sirt_count, proj_count - s * sirt_count);
      bool fused = false;
      if ((rc = rec_back_project_subset(r, vg, vol, voxel_type, index_list + s * sirt_count, in_subset,
                                        (float)sirt_count, r->sirt_d.data(), fused)))
        return rc;
      if (fused) *volume_is_empty = 0;
      for (int i = 0; i < sirt_count && !fused; ++i) {
        if (s * sirt_count + i >= proj_count) continue;
        *volume_is_empty = 0;
        const int index = index_list[s * sirt_count + i];
        if ((rc = rec_back_project_image(r, vg, vol, voxel_type, index, (float)sirt_count, r->sirt_d[i]))) return rc;
      }
    }
  }
  return ok();
}

int esb_subvolume_wbp(esb_reconstructor* r, const esb_vol_geom* full_vol, int n_particles, const esb_vol_geom* sub_geoms,
                      const esb_proj_geom* pair_geoms, const unsigned char* active, float* const* boxes,
                      const float* projections, const int* index_list, int proj_count, int batched) {
  if (!r || !full_vol || !sub_geoms || !pair_geoms || !boxes || !projections || !index_list || n_particles < 0 ||
      proj_count < 0)
    return fail(ESB_ERR_INVALID_ARGUMENT, "esb_subvolume_wbp: invalid argument");
  const esb_recon_config& cf = r->cfg;
  const int W = cf.proj_x, H = cf.proj_y, np = cf.n_proj;
  const size_t img = (size_t)W * H;
  int rc;
  for (int ii = 0; ii < proj_count; ++ii)
    if (index_list[ii] < 0 || index_list[ii] >= np)
      return fail(ESB_ERR_INVALID_ARGUMENT, "esb_subvolume_wbp: index out of range");
  if (batched && cf.variant == ESB_VARIANT_FAST && n_particles > 0 && proj_count > 0) {
    std::vector<KConst> consts((size_t)n_particles * proj_count);
    std::vector<unsigned char> act((size_t)n_particles * proj_count);
    host_parallel_for((long)n_particles * proj_count, [&](long i) {
      const int p = (int)(i / proj_count), ii = (int)(i % proj_count);
      const size_t pair = (size_t)p * np + index_list[ii];
      consts[i] = rec_const(r, pair_geoms[pair], sub_geoms[p], 1);
      act[i] = active ? (active[pair] != 0) : 1;
    });
    if (subvol_batchable(n_particles, boxes, consts.data(), proj_count)) {
      ESB_CK(subvol_batch_build(r->batch, n_particles, boxes, consts.data(), act.data(), proj_count, cf.oversampling,
                                r->stream), "esb_subvolume_wbp");
      if (!cf.ctf_mode) {
        // all projections of the list resident (transposed), a chunk of up
        // to 4 GiB of images per persistent launch
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>(proj_count, ((size_t)4 << 30) / (img * 4)));
        if ((rc = rec_slab_capacity(r, chunk))) return rc;
        SlabTable none;
        none.count = 0;
        for (int t0 = 0; t0 < proj_count; t0 += chunk) {
          const int nt = std::min(chunk, proj_count - t0);
          for (int t = 0; t < nt; ++t)
            ESB_CK(launch_transpose(projections + (size_t)index_list[t0 + t] * img, W, H, W, r->slab_imgs + t * img,
                                    r->stream), "esb_subvolume_wbp");
          PhaseScope ps(r, 1);
          ESB_CK(subvol_batch_launch(r->batch, t0, nt, r->slab_imgs, img, none, W, H, cf.oversampling, 0, r->stream),
                 "esb_subvolume_wbp");
        }
        return ok();
      }
      if (r->subvol_patches) {
        // every tilt's slab images filtered and the patches its pairs read
        // gathered (up to 16 GiB), then all tilts in one persistent launch
        std::vector<SlabTable> Ts(proj_count);
        for (int ii = 0; ii < proj_count; ++ii)
          if ((rc = rec_slab_table(r, full_vol, index_list[ii], Ts[ii]))) return rc;
        bool planned = false;
        ESB_CK(subvol_patch_plan(r->batch, Ts.data(), W, H, (size_t)16 << 30, r->stream, planned),
               "esb_subvolume_wbp");
        if (planned) {
          for (int ii = 0; ii < proj_count; ++ii) {
            const int index = index_list[ii];
            SlabTable T;
            if ((rc = rec_subvol_slab_images(r, full_vol, projections + (size_t)index * img, index, T))) return rc;
            PhaseScope ps(r, 3);
            ESB_CK(subvol_patch_gather(r->batch, ii, r->slab_imgs, img, W, H, r->stream), "esb_subvolume_wbp");
          }
          {
            PhaseScope ps(r, 1);
            ESB_CK(subvol_patch_launch(r->batch, W, H, cf.oversampling, 1, r->stream), "esb_subvolume_wbp");
          }
          unsigned long long misses = 0;
          ESB_CK(subvol_patch_misses(r->batch, r->stream, misses), "esb_subvolume_wbp");
          if (misses)
            return fail(ESB_ERR_UNSUPPORTED, "esb_subvolume_wbp: " + std::to_string(misses) +
                                                 " quad samples fell outside the planned CTF patches");
          return ok();
        }
      }
      for (int ii = 0; ii < proj_count; ++ii) {
        const int index = index_list[ii];
        SlabTable T;
        if ((rc = rec_subvol_slab_images(r, full_vol, projections + (size_t)index * img, index, T))) return rc;
        PhaseScope ps(r, 1);
        ESB_CK(subvol_batch_launch(r->batch, ii, 1, r->slab_imgs, img, T, W, H, cf.oversampling, 1, r->stream),
               "esb_subvolume_wbp");
      }
      return ok();
    }
  }
  // EmSartSubVolumes.cpp:626-683 with Reconstructor.cpp:893-914 / 975-1033
  for (int ii = 0; ii < proj_count; ++ii) {
    const int index = index_list[ii];
    if (index < 0 || index >= np) return fail(ESB_ERR_INVALID_ARGUMENT, "esb_subvolume_wbp: index out of range");
    const float* proj = projections + (size_t)index * img;
    if (!cf.ctf_mode && cf.variant == ESB_VARIANT_FAST) {
      if ((rc = rec_slab_capacity(r, 1))) return rc;
      ESB_CK(launch_transpose(proj, W, H, W, r->slab_imgs, r->stream), "esb_subvolume_wbp");
      SlabTable none;
      none.count = 0;
      for (int p = 0; p < n_particles; ++p) {
        if (active && !active[(size_t)p * np + index]) continue;
        KConst c = rec_const(r, pair_geoms[(size_t)p * np + index], sub_geoms[p], 1);
        PhaseScope ps(r, 1);
        ESB_CK(launch_bp_fast_slabs(c, boxes[p], ESB_VOXEL_F32, r->slab_imgs, 0, none, W, H, W, 1.0f, cf.oversampling,
                                    0.0f, 9999999999999.0f, 0, r->stream, 1), "esb_subvolume_wbp");
      }
      continue;
    }
    if (!cf.ctf_mode) {
      for (int p = 0; p < n_particles; ++p) {
        if (active && !active[(size_t)p * np + index]) continue;
        KConst c = rec_const(r, pair_geoms[(size_t)p * np + index], sub_geoms[p], 1);
        PhaseScope ps(r, 1);
        ESB_CK(rec_bp(r, c, boxes[p], ESB_VOXEL_F32, proj, 1.0f, 0.0f, 9999999999999.0f, 0), "esb_subvolume_wbp");
      }
      continue;
    }
    float t_in, t_out;
    esb_defocus_distances(&r->geoms[index], full_vol, W, H, &t_in, &t_out);
    const float step = cf.ctf_slice_thickness_nm / cf.pixel_size_nm;
    if (cf.variant == ESB_VARIANT_FAST) {
      // Wiener-filtered image per slab of the whole tomogram, then one launch
      // per particle that picks each quad's slab image by its depth
      SlabTable T;
      if ((rc = rec_subvol_slab_images(r, full_vol, proj, index, T))) return rc;
      for (int p = 0; p < n_particles; ++p) {
        if (active && !active[(size_t)p * np + index]) continue;
        KConst c = rec_const(r, pair_geoms[(size_t)p * np + index], sub_geoms[p], 1);
        PhaseScope ps(r, 1);
        ESB_CK(launch_bp_fast_slabs(c, boxes[p], ESB_VOXEL_F32, r->slab_imgs, img, T, W, H, W, 1.0f, cf.oversampling,
                                    0.f, 0.f, 1, r->stream, 1), "esb_subvolume_wbp");
      }
      continue;
    }
    for (float ray = t_in; ray < t_out; ray += step) {
      float dmin, dmax;
      esb_defocus_min_max(ray, r->defocus[3 * index], r->defocus[3 * index + 1], r->tilt[index], cf.add_tilt_angle,
                          cf.pixel_size_nm, cf.ctf_slice_thickness_nm, cf.volume_shift[2], cf.ignore_z_shift_for_ctf,
                          cf.switch_ctf_direction, &dmin, &dmax);
      static const int none[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      // makeSquare without crop on the prepared projection (Reconstructor.cpp:995-1004)
      if ((rc = rec_ctf_chain(r, const_cast<float*>(proj), 0, none, index, dmin, dmax, 0, r->dist_d, nullptr, 0, none))) return rc;
      for (int p = 0; p < n_particles; ++p) {
        if (active && !active[(size_t)p * np + index]) continue;
        KConst c = rec_const(r, pair_geoms[(size_t)p * np + index], sub_geoms[p], 1);
        PhaseScope ps(r, 1);
        ESB_CK(rec_bp(r, c, boxes[p], ESB_VOXEL_F32, r->dist_d, 1.0f, ray, ray + step, 1), "esb_subvolume_wbp");
      }
    }
  }
  return ok();
}

}  // extern "C"
