// EmSart's SART reconstruction with libesb in place of the reference's
// Reconstructor: the integration of INTEGRATION.md ("Replace the
// Reconstructor's device work"), compiled and run.
//
// The host side is the reference's own: Configuration::Config reads
// emsart.cfg, MarkerFile the alignment, Projection and Volume derive the
// detector frames and the volume placement (src/EmSART/Projection.cpp,
// Volume.cpp, utils/Config.cpp, src/EmTools/FileIO/MarkerFile.cpp, compiled
// unmodified from the reference tree by oracle/cpp_caller/build.py), and
// Projection::CreateProjectionIndexList gives the projection order, as in
// EmSart.cpp:83-675. The device work is libesb's C ABI (include/esb.h):
// esb_reconstructor_create and esb_sart_run replace the Reconstructor and
// the SART loop of EmSart.cpp:579-675.
//
// TEST INFRASTRUCTURE: tests/test_cpp_caller.py runs it on a small case
// and compares the volume with the CPU oracle's.
//
//   sart_caller CONFIG MARKERS PROJECTIONS.raw W H VOLUME_OUT.raw VARIANT
//
// PROJECTIONS.raw: n x H x W float32 (prepared projections); VOLUME_OUT.raw:
// the reconstructed volume, z x y x x float32 (not negated); VARIANT: 0
// (ESB_VARIANT_FAITHFUL) or 1 (ESB_VARIANT_FAST).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "MarkerFile.h"
#include "Projection.h"
#include "Volume.h"
#include "esb.h"
#include "utils/Config.h"

// Prepared projections held in host memory (the ProjectionSource the
// reference's Projection reads its size and pixel size from).
class HostStack : public ProjectionSource {
 public:
  HostStack(const char* path, int n, int w, int h, float ps) : n_(n), w_(w), h_(h), ps_(ps), data_((size_t)n * w * h) {
    FILE* f = fopen(path, "rb");
    if (!f || fread(data_.data(), sizeof(float), data_.size(), f) != data_.size())
      throw std::runtime_error("cannot read the projections");
    fclose(f);
  }
  DataType_enum GetDataType() { return DT_FLOAT; }
  char* GetProjection(uint i) { return (char*)(data_.data() + (size_t)i * w_ * h_); }
  float GetPixelSize() { return ps_; }
  int GetWidth() { return w_; }
  int GetHeight() { return h_; }
  int GetProjectionCount() { return n_; }
  const float* Data() const { return data_.data(); }

 private:
  int n_, w_, h_;
  float ps_;
  std::vector<float> data_;
};

static void copy3(float* dst, float3 v) {
  dst[0] = v.x;
  dst[1] = v.y;
  dst[2] = v.z;
}

static void check_esb(int rc) {
  if (rc) throw std::runtime_error(esb_last_error());
}

static void check_cuda(cudaError_t e) {
  if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

int main(int argc, char** argv) {
  if (argc < 8) {
    fprintf(stderr, "usage: sart_caller CONFIG MARKERS PROJECTIONS.raw W H VOLUME_OUT.raw VARIANT\n");
    return 2;
  }
  try {
    Configuration::Config& config = Configuration::Config::GetConfig(argv[1], 0, nullptr, 0);
    MarkerFile markers(argv[2], config.ReferenceMarker);
    const int n = markers.GetProjectionCount();
    const int W = atoi(argv[4]), H = atoi(argv[5]);
    HostStack stack(argv[3], n, W, H, 1.0f);
    Projection proj(&stack, &markers);
    Volume<float> vol(config.RecDimensions, 1, -1);
    vol.PositionInSpace(config.VoxelSize, config.VolumeShift);

    // --- begin: libesb in place of the Reconstructor ---
    // Detector frames and volume placement from the reference's Projection
    // and Volume (Kernels.cpp:1056 takes the detector matrix at os = 1).
    std::vector<esb_proj_geom> geoms(n);
    std::vector<float> tilt(n);
    for (int i = 0; i < n; ++i) {
      copy3(geoms[i].detektor, proj.GetPosition(i));
      copy3(geoms[i].u_pitch, proj.GetPixelUPitch(i));
      copy3(geoms[i].v_pitch, proj.GetPixelVPitch(i));
      copy3(geoms[i].proj_norm, proj.GetNormalVector(i));
      proj.GetDetectorMatrix(i, geoms[i].detector_matrix, 1);
      tilt[i] = markers(MFI_TiltAngle, i, 0);
    }
    esb_vol_geom vg;
    copy3(vg.bbox_min, vol.GetSubVolumeBBoxMin(0));
    copy3(vg.bbox_max, vol.GetSubVolumeBBoxMax(0));
    copy3(vg.bbox_rcp, vol.GetSubVolumeBBoxRcp(0));
    copy3(vg.dim, vol.GetSubVolumeDimension(0));
    copy3(vg.voxel_size, vol.GetVoxelSize());
    vg.z_shift = vol.GetSubVolumeZShift(0);
    copy3(vg.full_dim, vol.GetDimension());
    copy3(vg.full_bbox_min, vol.GetVolumeBBoxMin());
    copy3(vg.full_bbox_max, vol.GetVolumeBBoxMax());

    // The reconstruction parameters from the reference's Configuration.
    esb_recon_config cfg = {};
    cfg.proj_x = W;
    cfg.proj_y = H;
    cfg.n_proj = n;
    cfg.lambda = config.Lambda;
    cfg.oversampling = config.OverSampling;
    cfg.ctf_mode = 0;
    cfg.cut_length[0] = config.CutLength.x;
    cfg.cut_length[1] = config.CutLength.y;
    cfg.dim_length[0] = config.DimLength.x;
    cfg.dim_length[1] = config.DimLength.y;
    const float crop[4] = {config.Crop.x, config.Crop.y, config.Crop.z, config.Crop.w};
    const float crop_dim[4] = {config.CropDim.x, config.CropDim.y, config.CropDim.z, config.CropDim.w};
    for (int k = 0; k < 4; ++k) {
      cfg.crop[k] = crop[k];
      cfg.crop_dim[k] = crop_dim[k];
    }
    cfg.projection_scale_factor = config.ProjectionScaleFactor;
    cfg.add_tilt_angle = config.AddTiltAngle;
    cfg.variant = atoi(argv[7]);
    const float identity[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // no magnification anisotropy
    esb_reconstructor* rec = nullptr;
    check_esb(esb_reconstructor_create(&cfg, geoms.data(), tilt.data(), nullptr, identity, identity, &rec));
    cudaStream_t stream;
    check_cuda(cudaStreamCreate(&stream));
    check_esb(esb_reconstructor_set_stream(rec, stream));

    // Device volume and projections (EmSart.cpp keeps a CUDA array and the
    // host projections; libesb takes plain device arrays).
    const size_t nvox = (size_t)vg.dim[0] * vg.dim[1] * vg.dim[2];
    float *vol_d = nullptr, *proj_d = nullptr;
    check_cuda(cudaMalloc(&vol_d, nvox * sizeof(float)));
    check_cuda(cudaMalloc(&proj_d, (size_t)n * W * H * sizeof(float)));
    check_cuda(cudaMemsetAsync(vol_d, 0, nvox * sizeof(float), stream));
    check_cuda(cudaMemcpyAsync(proj_d, stack.Data(), (size_t)n * W * H * sizeof(float), cudaMemcpyHostToDevice,
                               stream));

    // The projection order of EmSart.cpp, from the reference's Projection.
    int count = 0;
    int* order = nullptr;
    proj.CreateProjectionIndexList(PLT_RANDOM_START_ZERO_TILT, &count, &order);
    int volume_is_empty = 1;
    check_esb(esb_sart_run(rec, &vg, vol_d, ESB_VOXEL_F32, proj_d, order, count, config.Iterations,
                           config.SIRTCount, &volume_is_empty));
    std::vector<float> out(nvox);
    check_cuda(cudaMemcpyAsync(out.data(), vol_d, nvox * sizeof(float), cudaMemcpyDeviceToHost, stream));
    check_cuda(cudaStreamSynchronize(stream));
    check_esb(esb_reconstructor_destroy(rec));
    // --- end ---

    FILE* f = fopen(argv[6], "wb");
    if (!f || fwrite(out.data(), sizeof(float), nvox, f) != nvox) throw std::runtime_error("cannot write the volume");
    fclose(f);
    cudaFree(vol_d);
    cudaFree(proj_d);
    cudaStreamDestroy(stream);
    printf("sart_caller: %d projections (%d in the order), %d iterations, %d per subset, volume %g x %g x %g\n", n,
           count, config.Iterations, config.SIRTCount, vg.dim[0], vg.dim[1], vg.dim[2]);
  } catch (std::exception& e) {
    fprintf(stderr, "sart_caller: %s\n", e.what());
    return 1;
  }
  return 0;
}
