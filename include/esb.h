/*
 * esb.h - C ABI of the B200 (sm_100a) EmSART reconstruction hot path.
 *
 * This header is the drop-in boundary. It replaces the reference's kernel
 * wrappers (src/EmSART/Kernels.h:37-245), which launch named kernels from
 * JIT-loaded PTX modules and pass geometry through __constant__ symbols that
 * SetConstantValues writes by name (src/EmSART/Kernels.cpp:949-1131). Here
 * the geometry travels as a plain struct (esb_constants). The volume is a
 * linear device array of voxels in [z][y][x] order, with no CUDA array,
 * texture or surface. Images are pitched device arrays of float.
 *
 * Conventions:
 *  - Every function returns an int status: ESB_OK (0) on success, or one of
 *    the ESB_ERR_* codes below. esb_last_error() then holds a message for the
 *    calling thread. No C++ exception crosses this boundary (the reference
 *    throws CudaException instead, CudaHelpers/CudaException.h:34-36).
 *  - `stream` is a cudaStream_t passed as void*; NULL means the legacy
 *    default stream. Launch functions are asynchronous. The reference's
 *    wrappers synchronise after every launch and return the elapsed time
 *    (Kernels.cpp:65-86).
 *  - Pointers marked "device" must point to device memory of the current
 *    device; pitches are in BYTES.
 */
#ifndef ESB_H
#define ESB_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ESB_OK 0
#define ESB_ERR_INVALID_ARGUMENT 1
#define ESB_ERR_CUDA 2
#define ESB_ERR_CUFFT 3
#define ESB_ERR_UNSUPPORTED 4
#define ESB_ERR_OUT_OF_MEMORY 5

/* Voxel storage of the volume: FP32 (Volume<float>), FP16 (the reference's
 * FP16Volume, Volume<unsigned short> over a HALF array, EmSart.cpp:404-414),
 * or BF16 (added here). The arithmetic is always FP32. */
#define ESB_VOXEL_F32 0
#define ESB_VOXEL_F16 1
#define ESB_VOXEL_BF16 2

/* Everything SetConstantValues writes into the projector/back-projector
 * modules (Kernels.cpp:949-1101; symbol list DeviceVariables.cuh:13-34). */
typedef struct esb_constants {
  float proj_norm[3];        /* c_projNorm   Projection::GetNormalVector  */
  float detektor[3];         /* c_detektor   Projection::GetPosition      */
  float u_pitch[3];          /* c_uPitch     Projection::GetPixelUPitch   */
  float v_pitch[3];          /* c_vPitch     Projection::GetPixelVPitch   */
  float bbox_min[3];         /* c_bBoxMin    Volume::GetSubVolumeBBoxMin  */
  float bbox_max[3];         /* c_bBoxMax    Volume::GetSubVolumeBBoxMax  */
  float bbox_rcp[3];         /* c_volumeBBoxRcp                           */
  float volume_dim[3];       /* c_volumeDim  (sub-volume dimension)       */
  float voxel_size[3];       /* c_voxelSize                               */
  float z_shift;             /* c_zShiftForPartialVolume (0 for FP, Kernels.cpp:987) */
  int volume_dim_x_quarter;  /* c_volumeDim_x_quarter = dim.x / 4         */
  float detector_matrix[16]; /* c_DetectorMatrix (GetDetectorMatrix, os=1) */
  float mag_aniso[9];        /* c_magAniso    3x3 row-major               */
  float mag_aniso_inv[9];    /* c_magAnisoInv 3x3 row-major               */
} esb_constants;

/* Per-projection alignment as read from the marker file (MarkerFile items
 * MFI_TiltAngle, MFI_X_Shift, MFI_Y_Shift, MFI_Magnifiaction,
 * MFI_RotationPsi; MarkerFile.h:34-46) plus the config keys Projection reads
 * (utils/Config.cpp:303-494). */
typedef struct esb_tilt_config {
  float add_tilt_angle;    /* AddTiltAngle    */
  float add_tilt_x_angle;  /* AddTiltXAngle   */
  int use_fix_psi_angle;   /* UseFixPsiAngle  */
  float psi_angle;         /* PsiAngle        */
  float phi_angle;         /* PhiAngle        */
} esb_tilt_config;

/* Detector frame of one projection, as the reference derives it. */
typedef struct esb_proj_geom {
  float detektor[3];
  float u_pitch[3];
  float v_pitch[3];
  float proj_norm[3];
  float detector_matrix[16];
} esb_proj_geom;

/* Placement of a (sub-)volume in space (Volume.cpp:27-306). */
typedef struct esb_vol_geom {
  float bbox_min[3];  /* sub-volume bbox min */
  float bbox_max[3];  /* sub-volume bbox max */
  float bbox_rcp[3];  /* 1 / (sub-volume dim * voxel size) */
  float dim[3];       /* sub-volume dimension */
  float voxel_size[3];
  float z_shift;      /* Volume::GetSubVolumeZShift */
  float full_dim[3];  /* whole-volume dimension */
  float full_bbox_min[3];
  float full_bbox_max[3];
} esb_vol_geom;

const char* esb_last_error(void);
int esb_version(void);
/* Number of kernel launches this library has issued in the process (all
 * threads; cuFFT's own kernels not included). No counterpart in the
 * reference: a diagnostic for launch-count claims. */
unsigned long long esb_kernel_launches(void);

/* Autotuning of launch shapes (no counterpart in the reference). A
 * reconstructor picks, per GPU and problem shape, the block shape of the fast
 * projector and of the single-axis back-projector the first time it launches
 * them outside stream capture (CUDA events; one warm-up and two timed trial
 * launches per candidate; trials never write the caller's volume), and the
 * choice is cached for the process. Results do not depend on the shape.
 * enable: 1 measure (default), 0 use cached or default shapes only, -1 clear
 * the cache (measuring stays as it was), k >= 2 make every tuned kernel take
 * its candidate k - 2 (the last one where it has fewer; for tests: results
 * must not change); 0 or 1 end that. */
int esb_autotune(int enable);
/* The cached choices as text, one line per problem shape, into buf
 * (NUL-terminated, truncated to len; buf may be NULL with len 0); *needed
 * (may be NULL) = the bytes the whole text takes, NUL included. */
int esb_autotune_report(char* buf, size_t len, size_t* needed);

/* ---------------------------------------------------------------- geometry
 * Host functions; no device work. */

/* Projection::GetPosition / GetPixelUPitch / GetPixelVPitch /
 * GetNormalVector / GetDetectorMatrix(os=1) (Projection.cpp:80-404) for every
 * projection. extra_shift (2 floats per projection, may be NULL) is
 * Projection::SetExtraShift (Projection.cpp:1102-1108). */
int esb_projection_geometry(int n_proj, int width, int height, const float* tilt_deg, const float* x_shift,
                            const float* y_shift, const float* magnification, const float* psi_deg,
                            const float* extra_shift, const esb_tilt_config* cfg, esb_proj_geom* out);

/* Volume(dim, subvol_count, subvol) + PositionInSpace(voxelSize, volumeShift,
 * shiftXY=0) (Volume.cpp:82-114, 270-287), for sub-volume `subvol`. */
int esb_volume_geometry(const int dim[3], int subvol_count, int subvol, const float voxel_size[3],
                        const float volume_shift[3], esb_vol_geom* out);

/* Volume::PositionInSpace for a particle box (Volume.cpp:289-306): a
 * size^3 box of voxel size vs_sub centred on motive-list position pos
 * (1-based) plus shift, inside the full volume `vol`. */
int esb_subvolume_geometry(int size, float vs_sub, const esb_vol_geom* vol, const float pos[3],
                           const float shift[3], esb_vol_geom* out);

/* Reconstructor::GetMagAnistropyMatrix (Reconstructor.cpp:386-426). */
int esb_mag_aniso_matrix(float amount, float angle_deg, float dim_x, float dim_y, float out[9]);

/* RotKernel::computeRotMat (Kernels.cpp:1227-1327): rotation matrix of the
 * motive list's Euler angles phi, psi, theta (degrees, ZXZ), row-major;
 * multiples of 30 and 45 degrees take exact cosines and sines. */
int esb_rotation_matrix(float phi, float psi, float theta, float out[9]);

/* SetConstantValues (Kernels.cpp:949-1101): assembles the kernel constants
 * of projection `p` and sub-volume `v`. for_bp selects the BP variant, which
 * sets c_zShiftForPartialVolume to the sub-volume's z shift; the FP variant
 * sets 0. */
int esb_set_constant_values(const esb_proj_geom* p, const esb_vol_geom* v, const float mag_aniso[9],
                            const float mag_aniso_inv[9], int for_bp, esb_constants* out);

/* Projection::ComputeHitPoints (Projection.cpp:850-1049): the volume's
 * shadow corners pA..pD on the detector as 8 ints (x,y pairs). */
int esb_compute_hit_points(const esb_proj_geom* p, const esb_vol_geom* v, int out[8]);

/* Reconstructor::GetDefocusDistances (Reconstructor.cpp:53-173). */
int esb_defocus_distances(const esb_proj_geom* p, const esb_vol_geom* v, int width, int height, float* t_in,
                          float* t_out);

/* Reconstructor::GetDefocusMinMax (Reconstructor.cpp:178-201). */
int esb_defocus_min_max(float ray, float defocus_min_nm, float defocus_max_nm, float tilt_deg, float add_tilt_deg,
                        float pixel_size_nm, float slice_thickness_nm, float volume_shift_z, int ignore_z_shift,
                        int switch_direction, float* out_min, float* out_max);

/* Projection::CreateProjectionIndexList (Projection.cpp:561-640). type:
 * 0 PLT_NORMAL, 1 PLT_RANDOM, 2 PLT_RANDOM_START_ZERO_TILT. `good` marks the
 * projections MarkerFile::CheckIfProjIndexIsGood accepts (NULL = all). Uses
 * the C library's srand(0)/rand() as the reference does. Returns the count
 * in *count; out holds n_proj ints. */
int esb_projection_index_list(int type, int n_proj, const float* tilt_deg, const int* good, int* out, int* count);

/* ------------------------------------------------------------ kernels
 * One entry point per reference kernel wrapper. Device pointers. */

/* FPKernel::operator() (Kernels.cpp:46-88) -> kernel `march`
 * (ForwardProjectionRayMarcher_TL.cu:58-160). proj += line integral,
 * dist = mean sub-ray chord, for pixels in [roi_x0,roi_x1) x [roi_y0,roi_y1). */
int esb_fp(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj, float* dist,
           size_t pitch, int roi_x0, int roi_y0, int roi_x1, int roi_y1, void* stream);

/* SlicerKernel::operator() (Kernels.cpp:103-150) -> kernel `slicer`
 * (ForwardProjectionSlicer.cu:57-220): proj += integral over t in [tmin,tmax]. */
int esb_fp_slicer(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj,
                  size_t pitch, float tmin, float tmax, int roi_x0, int roi_y0, int roi_x1, int roi_y1, void* stream);

/* VolTravLengthKernel::operator() (Kernels.cpp:160-205) -> kernel
 * `volTraversalLength` (ForwardProjectionSlicer.cu:224-288): dist += chord. */
int esb_vol_traversal_length(const esb_constants* c, int proj_x, int proj_y, float* dist, size_t pitch, int roi_x0,
                             int roi_y0, int roi_x1, int roi_y1, void* stream);

/* CompKernel::operator() (Kernels.cpp:218-260) -> kernel `compare`
 * (Compare.cu:50-130). virt <- tapered residual per unit length. */
int esb_compare(int proj_x, int proj_y, size_t pitch, const float* real, float* virt, const float* dist,
                float real_length, const float crop[4], const float crop_dim[4], float proj_val_scale, void* stream);

/* CropBorderKernel::operator() (Kernels.cpp:276-318) -> kernel `cropBorder`
 * (Compare.cu:171-277). p = pA..pD as (x,y) ints. */
int esb_crop_border(int proj_x, int proj_y, size_t pitch, float* img, const float cut_length[2],
                    const float dim_length[2], const int p[8], void* stream);

/* BPKernel::operator() (Kernels.cpp:327-379) -> kernels `backProjection` /
 * `backProjectionFP16` (BackProjectionSquareOS.cu:263-1291). vol +=
 * lambda * sum(img*chord)/sum(chord) per voxel. Only 4-voxel quads whose
 * first corner's depth lies in [dist_min, dist_max) are updated.
 * linear_filter selects the bilinear sampling of CTF mode
 * (Reconstructor.cpp:318-327). */
int esb_bp(const esb_constants* c, void* vol, int voxel_type, int proj_x, int proj_y, const float* img, size_t pitch,
           float lambda, int oversampling, float dist_min, float dist_max, int linear_filter, void* stream);

/* Reformulated ("fast") variants of the three entry points above, same
 * arguments and results within rel-L2 1e-3 of the reference's arithmetic:
 * esb_fp_fast / esb_fp_slicer_fast sum the trilinear interpolant over each
 * crossed cell in closed form (the reference's sample positions, one cell
 * load per ~5 samples); esb_bp_fast visits only each voxel's own shadow and
 * computes chords in voxel-local coordinates. No counterpart in the
 * reference beyond the kernels they reformulate. */
int esb_fp_fast(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj,
                float* dist, size_t pitch, int roi_x0, int roi_y0, int roi_x1, int roi_y1, void* stream);
int esb_fp_slicer_fast(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y, float* proj,
                       size_t pitch, float tmin, float tmax, int roi_x0, int roi_y0, int roi_x1, int roi_y1,
                       void* stream);
int esb_bp_fast(const esb_constants* c, void* vol, int voxel_type, int proj_x, int proj_y, const float* img,
                size_t pitch, float lambda, int oversampling, float dist_min, float dist_max, int linear_filter,
                void* stream);

/* ------------------------------------------------------- differentiation
 * No counterpart in the reference (its shift search, EmSartRefine.cpp:707-1100,
 * cross-correlates projections instead). The model is esb_fp_fast's
 * projection (march mode, `proj` only) with a detector offset (shift_u,
 * shift_v) in pixels, applied as a rigid in-plane translation of every
 * sample by shift_u * u + shift_v * v (the detector's pixel axes through the
 * magnification anisotropy); each ray keeps the unshifted sample set, so the
 * model is smooth in the offset. With zero offset it equals esb_fp_fast. */

/* grad_vol += A^T img: the exact transpose of that projection (atomic adds,
 * FP32 volume; zero grad_vol first for A^T img alone). */
int esb_fp_adjoint(const esb_constants* c, float* grad_vol, int proj_x, int proj_y, const float* img, size_t pitch,
                   float shift_u, float shift_v, void* stream);

/* One tilt of L = 1/2 sum (A(x, s) - measured)^2, with per-ray
 * recomputation (nothing stored per ray). Adds to out6 (device, 6 doubles):
 * [0] L, [1] dL/dshift_u, [2] dL/dshift_v, and the Gauss-Newton terms
 * [3] sum (dp/dshift_u)^2, [4] sum dp/dshift_u * dp/dshift_v,
 * [5] sum (dp/dshift_v)^2. grad_vol (FP32, may be NULL) += dL/dx.
 * proj_out (may be NULL) = A(x, s). measured may be NULL (taken as 0). For
 * a sub-volume, pass the particle box's constants: the offsets are then
 * per particle and tilt. */
int esb_projection_loss_grad(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y,
                             const float* measured, size_t pitch, float shift_u, float shift_v, float* grad_vol,
                             float* proj_out, double* out6, void* stream);

/* esb_projection_loss_grad over the detector pixels [roi[0], roi[2]) x
 * [roi[1], roi[3]) only (a particle's footprint), with two more sums for a
 * fitted amplitude: out8[6] += sum p^2 and out8[7] += sum p * measured
 * (p = A(x, s)); out8[0..5] as out6. */
int esb_projection_loss_grad_roi(const esb_constants* c, const void* vol, int voxel_type, int proj_x, int proj_y,
                                 const float* measured, size_t pitch, float shift_u, float shift_v, const int roi[4],
                                 float* grad_vol, float* proj_out, double* out8, void* stream);

/* RotKernel::operator() -> `rot3d` (Kernels.cpp:1338-1381,
 * wbpWeighting.cu:389-405): out = in rotated about voxel (size/2, size/2,
 * size/2) (integer division): out(p) = in at c + R^T (p - c), trilinear with
 * clamp addressing, R = rot (esb_rotation_matrix). in, out: size^3 FP32
 * device buffers, [z][y][x], not overlapping. The reference samples through
 * a texture (8-bit filter weights); the weights here are FP32. */
int esb_rotate_volume(const float* in, float* out, int size, const float rot[9], void* stream);

/* CopyToSquareKernel::operator() (Kernels.cpp:808-850) -> `makeSquare`
 * (CopyToSquare.cu:38-92); out is dense maxsize x maxsize. */
int esb_make_square(int proj_x, int proj_y, size_t pitch, const float* in, int maxsize, float* out, int border_x,
                    int border_y, int mirror_y, int fill_zero, void* stream);

/* CTFKernel::operator() (Kernels.cpp:395-436) with the constants of
 * SetConstantValues(CTFKernel...) (Kernels.cpp:1104-1131) -> `ctf`
 * (ctf.cu:82-240), in place on the N/2+1 x N half spectrum. Units as the
 * reference's callers use them: defocus in nm, angle in degrees, pixel size
 * in nm, Cs in mm, voltage in kV. amp_contrast is fixed to 0 by the
 * reference; it is exposed here. */
int esb_ctf(float* spectrum, int n, float defocus_min_nm, float defocus_max_nm, float angle_deg, int apply_for_fp,
            int phase_flip_only, float wiener_noise_level, const float beta_fac[4], float cs_mm, float voltage_kv,
            float amp_contrast, float pixel_size_nm, void* stream);

/* WbpWeightingKernel::operator() (Kernels.cpp:453-490) -> `wbpWeighting`
 * (wbpWeighting.cu:50-144). filter: 0 RAMP, 1 EXACT, 2 CONTRAST2,
 * 3 CONTRAST10, 4 CONTRAST30. */
int esb_wbp_weighting(float* spectrum, int n, float psi_deg, int filter, void* stream);

/* FourFilterKernel (Kernels.cpp:504-540) -> `fourierFilter` (wbpWeighting.cu:148-212). */
int esb_fourier_filter(float* spectrum, int n, float lp, float hp, float lps, float hps, void* stream);

/* DoseWeightingKernel (Kernels.cpp:556-590) -> `doseWeighting` (wbpWeighting.cu:216-240). */
int esb_dose_weighting(float* spectrum, int n, float dose, float pixel_size_a, void* stream);

/* ConvVol3DKernel (Kernels.cpp:1180-1230) -> `convertVolume3DFP16ToFP32`
 * (BackProjectionSquareOS.cu:1326-1355): out = -vol as float. Also accepts
 * FP32 and BF16 storage. */
int esb_convert_volume(const void* vol, int voxel_type, long n_voxels, float* out, int negate, void* stream);

/* Store a float volume into the given voxel type (round to nearest even). */
int esb_store_volume(const float* in, long n_voxels, void* vol, int voxel_type, void* stream);

/* ----------------------------------------------------- reconstructor
 * Reconstructor (Reconstructor.h:181-249) and the EmSART driver loops. The
 * object owns its device buffers (proj_d, dist_d, realproj_d, the padded
 * square image, the half spectrum) and its cuFFT plans, like the
 * reference's Reconstructor (Reconstructor.cpp:203-372). */

typedef struct esb_recon_config {
  int proj_x, proj_y;             /* projection size */
  int n_proj;
  float lambda;                   /* Lambda */
  int oversampling;               /* OverSampling */
  int ctf_mode;                   /* CtfMode */
  float cut_length[2];            /* CutLength */
  float dim_length[2];            /* DimLength */
  float crop[4];                  /* Crop */
  float crop_dim[4];              /* CropDim */
  float projection_scale_factor;  /* ProjectionScaleFactor */
  float pixel_size_nm;            /* projection pixel size in nm */
  float cs_mm, voltage_kv, amp_contrast;  /* Cs, Voltage; ampContrast (0 in the reference) */
  float ctf_slice_thickness_nm;   /* CTFSliceThickness */
  float ctf_beta_fac[4];          /* CTFBetaFac */
  float wiener_noise_level;       /* WienerFilterNoiseLevel */
  int phase_flip_only;            /* PhaseFlipOnly */
  int ignore_z_shift_for_ctf;     /* IgnoreZShiftForCTF */
  int switch_ctf_direction;       /* SwitchCTFDirectionForIMOD */
  float volume_shift[3];          /* VolumeShift */
  float add_tilt_angle;           /* AddTiltAngle */
  int variant;                    /* ESB_VARIANT_FAITHFUL or ESB_VARIANT_FAST kernels */
} esb_recon_config;

#define ESB_VARIANT_FAITHFUL 0
#define ESB_VARIANT_FAST 1

typedef struct esb_reconstructor esb_reconstructor;

/* geoms/tilt_deg: per projection; defocus: per projection (min nm, max nm,
 * astigmatism angle deg) or NULL without CTF; mag_aniso/inv: 3x3 each. */
int esb_reconstructor_create(const esb_recon_config* cfg, const esb_proj_geom* geoms, const float* tilt_deg,
                             const float* defocus, const float mag_aniso[9], const float mag_aniso_inv[9],
                             esb_reconstructor** out);
int esb_reconstructor_destroy(esb_reconstructor* rec);
int esb_reconstructor_set_stream(esb_reconstructor* rec, void* stream);
/* Device pointers to the reconstructor's W x H float images (pitch W*4). */
int esb_reconstructor_buffers(esb_reconstructor* rec, float** proj_d, float** dist_d, float** real_d);

/* Per-phase device timing of the reconstructor's launches (CUDA events on
 * its stream); the reference times every wrapper launch synchronously and
 * returns ms (Kernels.cpp:65-86). Phases: 0 forward projection kernels,
 * 1 back-projection kernel, 2 CTF chain (pad, FFTs, filter, crop),
 * 3 compare and buffer resets. esb_reconstructor_timing synchronises the
 * stream, returns the summed ms and launch counts since the previous call,
 * and restarts the accumulation. */
int esb_reconstructor_enable_timing(esb_reconstructor* rec, int enable);
int esb_reconstructor_timing(esb_reconstructor* rec, double out_ms[4], int counts[4]);

/* CUDA graphs for esb_sart_run (no counterpart in the reference, which
 * launches and synchronises every kernel from the host). When enabled and
 * timing is off, a call with iterations > 1 runs the first iteration
 * eagerly (sizing every buffer), captures the second on the stream and
 * replays that graph for the remaining ones. The volume, projections, index
 * list and subset size must stay those of the call (they are baked into the
 * graph). */
int esb_reconstructor_enable_graphs(esb_reconstructor* rec, int enable);

/* Back-projects each ordered subset of esb_sart_run / esb_sart_run_zslab in
 * one pass over the volume: every voxel is read once per subset, the
 * SIRTCount updates are added to it in the subset's order, and it is stored
 * once. FP32 volumes come out bit for bit as with one pass per projection
 * (EmSart.cpp:649-673); FP16 / BF16 volumes are rounded once per subset
 * instead of once per projection. enable: 1 on, 0 off, -1 (the default) on
 * for FP16 / BF16 volumes only (for FP32 the one-pass launch is no faster:
 * the back-projection is bound by instruction issue, not by volume traffic).
 * Applies to the FAST variant on single-axis geometry without magnification
 * anisotropy, power-of-two oversampling and at most 64 CTF slabs per
 * projection; other subsets are back-projected one projection at a time. */
int esb_reconstructor_fuse_subsets(esb_reconstructor* rec, int enable);

/* esb_subvolume_wbp with CTF, batched: on, after each tilt's CTF chain the
 * parts of its slab images that each particle's box reads are gathered into
 * one patch buffer (up to 16 GiB), and one persistent launch adds every tilt
 * to every box, each box read and written once. Off (the default): one
 * launch per tilt over all boxes, which is as fast (the back-projection is
 * bound by instruction issue, not by box traffic). Both give the same boxes
 * bit for bit. */
int esb_reconstructor_subvolume_patches(esb_reconstructor* rec, int enable);

/* ResetProjectionsDevice (Reconstructor.cpp:1678-1682). */
int esb_rec_reset_projections(esb_reconstructor* rec);
/* ForwardProjection (Reconstructor.cpp:1411-1421), CTF or not. */
int esb_rec_forward_projection(esb_reconstructor* rec, const esb_vol_geom* vg, const void* vol, int voxel_type,
                               int index, int volume_is_empty);
/* ForwardProjectionROI (Reconstructor.cpp:1519-1529 -> ForwardProjectionNoCTFROI
 * :649-712, ForwardProjectionCTFROI :716-859): ForwardProjection for the rays
 * of the detector region [roi[0], roi[2]) x [roi[1], roi[3]) only (the
 * reference's roiMin / roiMax, clipped to the detector), added to the
 * projection buffer; with CTF each slab image is still filtered over the
 * whole detector. EmSartRefine projects the particles' models and the
 * reconstruction without them this way. */
int esb_rec_forward_projection_roi(esb_reconstructor* rec, const esb_vol_geom* vg, const void* vol, int voxel_type,
                                   int index, int volume_is_empty, const int roi[4]);
/* Compare (Reconstructor.cpp:1386-1405). real: device image W x H. */
int esb_rec_compare(esb_reconstructor* rec, const esb_vol_geom* vg, const float* real, int index);
/* BackProjection (Reconstructor.cpp:871-887 / 920-969) of proj_d. */
int esb_rec_back_projection(esb_reconstructor* rec, const esb_vol_geom* vg, void* vol, int voxel_type, int index,
                            float sirt_count);

/* Reconstructor::PrepareProjection (Reconstructor.cpp:1158-1383): the raw
 * projection `in` (device, W x H, input_type) becomes the normalised float
 * image `out` (device, W x H) that the reconstruction reads:
 *   convert to float; pad to the N x N square (mirror padding, flipped in y
 *   for DM4 stacks); mean of the square; bad pixels (> bad_pixel_value *
 *   mean) set to the mean; WBP: normalise the raw window (mean / std /
 *   none, std divided by cos(tilt) with down_weight_tilts) and pad again;
 *   unless skip_filter (or WBP): R2C, band-pass (lp, hp, lps, hps), dose
 *   weighting, WBP weighting (psi, wbp_filter), C2R, / N^2; SART: normalise
 *   the filtered window (mean / std over the whole image, or the centre half
 *   for ESB_PNM_NONE, which keeps the mean and divides by 1):
 *   out = (x - mean) / (-std).
 * mean, std (host, may be NULL) receive the statistics the reference
 * returns, bad_pixels (host, may be NULL) the count. Synchronises the
 * reconstructor's stream (the statistics are read back, as the reference
 * does). Statistics are FP64 sums; the reference's NPP reductions are not
 * pinned. */
#define ESB_PIX_F32 0
#define ESB_PIX_S16 1
#define ESB_PIX_U16 2
#define ESB_PIX_S32 3
#define ESB_PIX_U32 4
#define ESB_PNM_MEAN 0
#define ESB_PNM_STANDARD_DEV 1
#define ESB_PNM_NONE 2
typedef struct {
  int input_type;          /* ESB_PIX_* (ProjectionSource data type) */
  int wbp;                 /* WBP_NoSART */
  int normalization;       /* ProjectionNormalization: ESB_PNM_* */
  int correct_bad_pixels;  /* CorrectBadPixels */
  float bad_pixel_value;   /* BadPixelValue */
  int mirror_y;            /* FileReadMode == FRM_DM4 */
  int skip_filter;         /* SkipFilter */
  float lp, hp, lps, hps;  /* fourFilterLP, fourFilterHP, fourFilterLPS, fourFilterHPS */
  int dose_weighting;      /* DoseWeighting */
  float accumulated_dose;  /* AccumulatedDose[index] */
  float pixel_size_nm;     /* Projection::GetPixelSize() */
  int down_weight_tilts;   /* DownWeightTiltsForWBP */
  float tilt_deg;          /* marker tilt angle of the projection */
  float psi_deg;           /* marker psi of the projection */
  int wbp_filter;          /* WBPFilter: FM_RAMP 0 .. FM_CONTRAST30 4 */
} esb_prepare_config;
int esb_prepare_projection(esb_reconstructor* rec, const esb_prepare_config* pc, const void* in, float* out,
                           float* mean, float* std_dev, int* bad_pixels);

/* Reconstructor::GetDisplacement (Reconstructor.cpp:1746-1960), EmSartRefine's
 * shift measurement: residual (the compare image of the reconstruction
 * without the particles) and model (the particles' projection), device,
 * W x H dense, are mirror-padded to the N x N square, centred on their
 * means and cross-correlated (conjMul, wbpWeighting.cu:244-262); the
 * correlation is divided by N^2 sqrt(SumA SumB), values farther than
 * max_shift from the origin are zeroed (maxShift, :266-293) and the
 * arg-max gives the integer shift (x, y), folded to (-N/2, N/2]. With
 * multi_peak the local maxima of at least 0.9 x the maximum (findPeak,
 * :331-386) are weighted by 1 / (distance + 1e-4) (maxShiftWeighted,
 * :296-327) and that map's arg-max gives the shift. A maximum <= 0 gives
 * (-1000, -1000), as in the reference, and so does a correlation that is
 * NaN everywhere. Ties go to the first pixel in raster order.
 * shift_xy (host, 2 floats); cc_value (host, may be NULL): the maximum of
 * the normalised correlation; cc_map, cc_map_multi (device, may be NULL):
 * the (4 max_shift)^2 fft-shifted centre of the correlation and of the
 * multi-peak map (the reference's ccMap and ccMapMulti). 1 <= max_shift
 * <= N/2. Synchronises the reconstructor's stream. */
int esb_rec_cc_displacement(esb_reconstructor* rec, const float* residual, const float* model, int max_shift,
                            int multi_peak, float* shift_xy, float* cc_value, float* cc_map, float* cc_map_multi);

/* The SART driver loop of EmSart.cpp:579-675 for one GPU: iterations x
 * ordered subsets of sirt_count projections x {FP, compare} then {BP}.
 * projections: device, n_proj images of W x H (already prepared);
 * index_list: the projection order (esb_projection_index_list);
 * *volume_is_empty: in/out flag of EmSart.cpp:425,653. */
int esb_sart_run(esb_reconstructor* rec, const esb_vol_geom* vg, void* vol, int voxel_type, const float* projections,
                 const int* index_list, int proj_count, int iterations, int sirt_count, int* volume_is_empty);

/* The sub-volume reconstruction of EmSartSubVolumes.cpp:611-705 with
 * Reconstructor::BackProjection(vol, subVolumes, ...)
 * (Reconstructor.cpp:893-1033): weighted back-projection (lambda = 1) of
 * n_particles boxes from the prepared (WBP-weighted) projections.
 *   full_vol   - placement of the whole tomogram (CTF slabs are cut on it)
 *   sub_geoms  - per particle placement (esb_subvolume_geometry); boxes may
 *                differ in size
 *   pair_geoms - [n_particles][n_proj] detector frames including the
 *                particle's per-tilt extra shift (esb_projection_geometry
 *                with extra_shift; Projection::SetExtraShift)
 *   active     - [n_particles][n_proj] 0/1, or NULL for all: the reference
 *                skips a tilt whose |shift| >= MaxShift - 0.5
 *                (EmSartSubVolumes.cpp:651-662)
 *   boxes      - per particle device pointer to a FP32 box, accumulated into
 *   projections- device, n_proj prepared images of W x H
 * batched = 0: one launch per particle per tilt (the reference's scheme);
 * batched = 1: one launch per tilt covering every particle. */
int esb_subvolume_wbp(esb_reconstructor* rec, const esb_vol_geom* full_vol, int n_particles,
                      const esb_vol_geom* sub_geoms, const esb_proj_geom* pair_geoms, const unsigned char* active,
                      float* const* boxes, const float* projections, const int* index_list, int proj_count,
                      int batched);

/* The collective of a z-slab SART: sums `count` floats at device address
 * `buf` over the ranks, in place, ordered on `stream` (for example
 * ncclAllReduce(buf, buf, count, ncclFloat, ncclSum, comm, stream), or a
 * host-side reduction that synchronises the stream first); returns 0 on
 * success. */
typedef int (*esb_allreduce_fn)(float* buf, size_t count, void* stream, void* user);

/* EmSart.cpp:579-675 over one z-slab of the volume per rank, the reference's
 * MPI decomposition (Volume(dim, count, part), Volume.cpp:82-114; vg from
 * esb_volume_geometry(dim, ranks, rank, ...), vol the slab's voxels). For
 * every projection the slab's forward projection and ray lengths (one
 * contiguous buffer of 2 x W x H floats: projection, then ray lengths) are
 * summed over the ranks with ONE call of `allreduce`, enqueued on the
 * reconstructor's stream between the forward projection and the compare
 * with no host synchronisation; every rank then forms the same residual
 * and back-projects it into its slab. (The reference gathers both images on
 * rank 0, Reconstructor.cpp:440-463, and broadcasts the residuals,
 * EmSart.cpp:647.) With CTF each rank filters its own slab images before the
 * sum, which equals filtering the sum. Every rank calls it with the same
 * arguments, so the collectives match in order. */
int esb_sart_run_zslab(esb_reconstructor* rec, const esb_vol_geom* vg, void* vol, int voxel_type,
                       const float* projections, const int* index_list, int proj_count, int iterations, int sirt_count,
                       int* volume_is_empty, esb_allreduce_fn allreduce, void* user);

/* ------------------------------------------------ no-allocation variant
 * No counterpart in the reference. One SART update of `vol` from one
 * projection without CTF: the sequence esb_rec_reset_projections,
 * esb_rec_forward_projection, esb_rec_compare and esb_rec_back_projection
 * perform on a reconstructor. This entry point allocates no device memory,
 * for callers that cannot call cudaMalloc: applications whose device memory
 * is owned and budgeted by their own allocator, processes that must not
 * allocate after start-up, and loops that must not pay cudaMalloc's implicit
 * device synchronisation.
 *  - Its two scratch images (forward projection and ray lengths) live in a
 *    fixed array inside the library of 2 x ESB_NOALLOC_MAX_PIXELS floats
 *    (32 MiB). The array stays resident on every GPU that loads it, until the
 *    process exits. Projections larger than ESB_NOALLOC_MAX_PIXELS pixels are
 *    rejected with ESB_ERR_INVALID_ARGUMENT.
 *  - The first call on a device looks up the array's device address (set-up,
 *    once per device and context; looked up again after a device reset
 *    replaced the context). Make that first call before any stream capture.
 *  - cfg->variant selects the kernels as on a reconstructor: FAITHFUL runs
 *    the reference's arithmetic, FAST the closed-form projector and the
 *    per-voxel-shadow back-projector (at the default launch shape: the
 *    reconstructor's launch-shape trials need scratch buffers; the shape
 *    does not change the result).
 *  - Every call shares the one array, and the array keeps the previous call's
 *    images; each call clears them first. Calls that overlap on the GPU (on
 *    different streams, or on different host threads, to the same device)
 *    race on the array and must be serialised by the caller.
 *  - cfg->ctf_mode must be 0 (the CTF chain needs FFT plans, which allocate).
 *  - real: device W x H image (pitch W*4). pg/vg/mag_aniso: as for
 *    esb_set_constant_values. */
#define ESB_NOALLOC_MAX_PIXELS (2048 * 2048)
int esb_sart_projection_update_noalloc(const esb_recon_config* cfg, const esb_proj_geom* pg, const esb_vol_geom* vg,
                                       const float mag_aniso[9], const float mag_aniso_inv[9], void* vol,
                                       int voxel_type, const float* real, float sirt_count, int volume_is_empty,
                                       void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ESB_H */
