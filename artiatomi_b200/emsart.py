"""Python host layer over libesb: the EmSART reconstruction calls.

Mirrors the reference's host interface for the hot path:

* geometry: ``Projection`` (src/EmSART/Projection.h:50-87) and ``Volume``
  (src/EmSART/Volume.h:30-79). Both are computed in C++ by libesb.
* kernel wrappers: FPKernel, SlicerKernel, VolTravLengthKernel, CompKernel,
  CropBorderKernel, BPKernel, CTFKernel, CopyToSquareKernel,
  WbpWeightingKernel, FourFilterKernel, DoseWeightingKernel
  (src/EmSART/Kernels.h:37-245).
* ``Reconstructor`` (src/EmSART/Reconstructor.h:181-249), the SART driver
  loop of EmSart.cpp:579-675, and the sub-volume back-projection of
  EmSartSubVolumes.cpp:611-705.

Device buffers are torch CUDA tensors, used only as memory. Every
computation runs in libesb's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import check, fptr, lib

VOXEL_F32, VOXEL_F16, VOXEL_BF16 = L.VOXEL_F32, L.VOXEL_F16, L.VOXEL_BF16
VARIANT_FAITHFUL, VARIANT_FAST = L.VARIANT_FAITHFUL, L.VARIANT_FAST
PLT_NORMAL, PLT_RANDOM, PLT_RANDOM_START_ZERO_TILT = 0, 1, 2
FM_RAMP, FM_EXACT, FM_CONTRAST2, FM_CONTRAST10, FM_CONTRAST30 = range(5)

_TORCH_DTYPES = None


def _voxel_type_of(t) -> int:
    import torch

    return {torch.float32: VOXEL_F32, torch.float16: VOXEL_F16, torch.bfloat16: VOXEL_BF16}[t.dtype]


def _stream(stream) -> Optional[int]:
    if stream is None:
        import torch

        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def _f32(a, n=None) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    if n is not None and a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


# --------------------------------------------------------------------------- geometry
@dataclass
class Markers:
    """Per-projection alignment items of the marker file (MarkerFile.h:34-46)."""

    tilt_angle: np.ndarray
    x_shift: Optional[np.ndarray] = None
    y_shift: Optional[np.ndarray] = None
    magnification: Optional[np.ndarray] = None
    rotation_psi: Optional[np.ndarray] = None

    @property
    def count(self) -> int:
        return int(np.asarray(self.tilt_angle).size)


@dataclass
class TiltConfig:
    add_tilt_angle: float = 0.0
    add_tilt_x_angle: float = 0.0
    use_fix_psi_angle: bool = False
    psi_angle: float = 0.0
    phi_angle: float = 0.0

    def c(self) -> L.TiltConfig:
        return L.TiltConfig(self.add_tilt_angle, self.add_tilt_x_angle, int(self.use_fix_psi_angle),
                            self.psi_angle, self.phi_angle)


def projection_geometry(markers: Markers, width: int, height: int, cfg: TiltConfig = TiltConfig(),
                        extra_shift=None):
    """Detector frames of all projections: a ctypes array of ProjGeom."""
    n = markers.count
    out = (L.ProjGeom * n)()
    arrs = [_f32(markers.tilt_angle, n)]
    for a in (markers.x_shift, markers.y_shift, markers.magnification, markers.rotation_psi):
        arrs.append(None if a is None else _f32(a, n))
    es = None if extra_shift is None else _f32(extra_shift, 2 * n)
    check(lib.esb_projection_geometry(n, width, height, *[fptr(a) for a in arrs], fptr(es), C.byref(cfg.c()),
                                      C.cast(out, C.c_void_p)))
    return out


def volume_geometry(dims: Sequence[int], voxel_size=(1.0, 1.0, 1.0), volume_shift=(0.0, 0.0, 0.0),
                    subvol_count: int = 1, subvol: int = 0) -> L.VolGeom:
    """Volume(dims, count, part) + PositionInSpace (Volume.cpp:82-114, 270-287)."""
    d = np.asarray(dims, dtype=np.int32)
    vs = _f32(voxel_size if np.size(voxel_size) == 3 else [voxel_size] * 3, 3)
    sh = _f32(volume_shift, 3)
    g = L.VolGeom()
    check(lib.esb_volume_geometry(fptr(d), subvol_count, subvol, fptr(vs), fptr(sh), C.byref(g)))
    return g


def subvolume_geometry(size: int, voxel_size_sub: float, vol: L.VolGeom, pos, shift=(0, 0, 0)) -> L.VolGeom:
    g = L.VolGeom()
    check(lib.esb_subvolume_geometry(size, voxel_size_sub, C.byref(vol), fptr(_f32(pos, 3)), fptr(_f32(shift, 3)),
                                     C.byref(g)))
    return g


def mag_aniso_matrix(amount: float, angle_deg: float, dim_x: float, dim_y: float) -> np.ndarray:
    out = np.zeros(9, np.float32)
    check(lib.esb_mag_aniso_matrix(amount, angle_deg, dim_x, dim_y, fptr(out)))
    return out


def autotune(enable: int = 1) -> None:
    """Launch-shape autotuning of the reconstructor's fast kernels: 1 measure
    (default), 0 cached or default shapes only, -1 clear the cache, k >= 2
    every tuned kernel takes its candidate k - 2 (for tests)."""
    check(lib.esb_autotune(int(enable)))


def autotune_report() -> str:
    """The cached launch-shape choices, one line per problem shape."""
    need = C.c_size_t(0)
    check(lib.esb_autotune_report(None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(lib.esb_autotune_report(buf, need.value, None))
    return buf.value.decode()


def rotation_matrix(phi: float, psi: float, theta: float) -> np.ndarray:
    """RotKernel::computeRotMat: 3 x 3 rotation of the motive list's Euler
    angles (degrees, ZXZ)."""
    out = np.zeros(9, np.float32)
    check(lib.esb_rotation_matrix(float(phi), float(psi), float(theta), fptr(out)))
    return out.reshape(3, 3)


def rotate_volume(vol, out, rot, stream=None) -> None:
    """`rot3d`: out = vol (size^3 FP32, device) rotated about voxel size // 2
    by rot (rotation_matrix), trilinear with clamp addressing."""
    size = int(vol.shape[0])
    if tuple(vol.shape) != (size, size, size) or tuple(out.shape) != (size, size, size):
        raise ValueError("rotate_volume: cubic volumes of equal size expected")
    r = np.ascontiguousarray(np.asarray(rot, np.float32).reshape(9))
    check(lib.esb_rotate_volume(fptr(vol), fptr(out), size, fptr(r), _stream(stream)))


IDENTITY3 = np.eye(3, dtype=np.float32).ravel()


def set_constant_values(pg: L.ProjGeom, vg: L.VolGeom, mag=None, mag_inv=None, for_bp: bool = False) -> L.Constants:
    c = L.Constants()
    m = _f32(IDENTITY3 if mag is None else mag, 9)
    mi = _f32(IDENTITY3 if mag_inv is None else mag_inv, 9)
    check(lib.esb_set_constant_values(C.byref(pg), C.byref(vg), fptr(m), fptr(mi), int(for_bp), C.byref(c)))
    return c


def compute_hit_points(pg: L.ProjGeom, vg: L.VolGeom) -> np.ndarray:
    out = np.zeros(8, np.int32)
    check(lib.esb_compute_hit_points(C.byref(pg), C.byref(vg), fptr(out)))
    return out


def defocus_distances(pg: L.ProjGeom, vg: L.VolGeom, width: int, height: int):
    a, b = C.c_float(), C.c_float()
    check(lib.esb_defocus_distances(C.byref(pg), C.byref(vg), width, height, C.byref(a), C.byref(b)))
    return a.value, b.value


def projection_index_list(kind: int, tilt_deg, good=None) -> np.ndarray:
    t = _f32(tilt_deg)
    n = t.size
    g = None if good is None else np.ascontiguousarray(np.asarray(good, np.int32))
    out = np.zeros(n, np.int32)
    cnt = C.c_int()
    check(lib.esb_projection_index_list(kind, n, fptr(t), fptr(g), fptr(out), C.byref(cnt)))
    return out[: cnt.value].copy()


# --------------------------------------------------------------------------- kernels
def _img_args(img):
    h, w = img.shape[-2:]
    return w, h, img.stride(-2) * 4


def forward_project(c: L.Constants, vol, proj, dist, roi=None, stream=None, fast: bool = False) -> None:
    """FPKernel: proj += line integrals, dist = mean chord (Kernels.cpp:46-88).
    fast selects the closed-form cell-sum projector."""
    w, h, pitch = _img_args(proj)
    x0, y0, x1, y1 = roi if roi is not None else (0, 0, w, h)
    check((lib.esb_fp_fast if fast else lib.esb_fp)(C.byref(c), fptr(vol), _voxel_type_of(vol), w, h, fptr(proj), fptr(dist), pitch, x0, y0, x1, y1,
                     _stream(stream)))


def forward_project_slab(c: L.Constants, vol, proj, tmin: float, tmax: float, roi=None, stream=None,
                         fast: bool = False) -> None:
    w, h, pitch = _img_args(proj)
    x0, y0, x1, y1 = roi if roi is not None else (0, 0, w, h)
    check((lib.esb_fp_slicer_fast if fast else lib.esb_fp_slicer)(C.byref(c), fptr(vol), _voxel_type_of(vol), w, h, fptr(proj), pitch, tmin, tmax, x0, y0,
                            x1, y1, _stream(stream)))


def traversal_length(c: L.Constants, dist, roi=None, stream=None) -> None:
    w, h, pitch = _img_args(dist)
    x0, y0, x1, y1 = roi if roi is not None else (0, 0, w, h)
    check(lib.esb_vol_traversal_length(C.byref(c), w, h, fptr(dist), pitch, x0, y0, x1, y1, _stream(stream)))


def compare(real, virt, dist, real_length: float, crop=(0, 0, 0, 0), crop_dim=(0, 0, 0, 0), scale: float = 1.0,
            stream=None) -> None:
    w, h, pitch = _img_args(virt)
    check(lib.esb_compare(w, h, pitch, fptr(real), fptr(virt), fptr(dist), real_length, fptr(_f32(crop, 4)),
                          fptr(_f32(crop_dim, 4)), scale, _stream(stream)))


def crop_border(img, cut_length, dim_length, points, stream=None) -> None:
    w, h, pitch = _img_args(img)
    p = np.ascontiguousarray(np.asarray(points, np.int32).ravel())
    check(lib.esb_crop_border(w, h, pitch, fptr(img), fptr(_f32(cut_length, 2)), fptr(_f32(dim_length, 2)), fptr(p),
                              _stream(stream)))


def back_project(c: L.Constants, vol, img, lam: float, oversampling: int = 1, dist_min: float = 0.0,
                 dist_max: float = 9999999999999.0, linear: bool = False, stream=None, fast: bool = False) -> None:
    """BPKernel: vol += lam * sum(img*chord)/sum(chord) (Kernels.cpp:327-379).
    fast selects the per-voxel-shadow back-projector."""
    w, h, pitch = _img_args(img)
    check((lib.esb_bp_fast if fast else lib.esb_bp)(C.byref(c), fptr(vol), _voxel_type_of(vol), w, h, fptr(img), pitch, lam, oversampling, dist_min,
                     dist_max, int(linear), _stream(stream)))


def fp_adjoint(c: L.Constants, grad, img, shift=(0.0, 0.0), stream=None) -> None:
    """grad += A^T img, the transpose of forward_project(..., fast=True)'s
    projection with detector offset `shift` (pixels). grad: FP32 volume."""
    w, h, pitch = _img_args(img)
    check(lib.esb_fp_adjoint(C.byref(c), fptr(grad), w, h, fptr(img), pitch, float(shift[0]), float(shift[1]),
                             _stream(stream)))


def projection_loss_grad_roi(c: L.Constants, vol, measured, out, roi, shift=(0.0, 0.0), grad=None, proj_out=None,
                             stream=None) -> None:
    """projection_loss_grad over the detector pixels roi = (x0, y0, x1, y1)
    (end exclusive) only; `out` holds 8 float64: the 6 sums of
    projection_loss_grad, then sum p^2 and sum p * measured."""
    w, h, pitch = _img_args(measured)
    box = np.ascontiguousarray(np.asarray(roi, np.int32).reshape(4))
    check(lib.esb_projection_loss_grad_roi(C.byref(c), fptr(vol), _voxel_type_of(vol), w, h, fptr(measured), pitch,
                                           float(shift[0]), float(shift[1]), fptr(box), fptr(grad),
                                           fptr(proj_out), fptr(out), _stream(stream)))


def projection_loss_grad(c: L.Constants, vol, measured, out, shift=(0.0, 0.0), grad=None, proj_out=None,
                         width: int | None = None, height: int | None = None, stream=None) -> None:
    """One tilt of L = 1/2 ||A(x, shift) - measured||^2. Adds to `out` (6
    float64 on the device): L, dL/dshift_u, dL/dshift_v and the Gauss-Newton
    terms sum (dp/du)^2, sum dp/du dp/dv, sum (dp/dv)^2; grad (FP32 volume,
    optional) += dL/dx; proj_out (optional) = A(x, shift). measured may be
    None (taken as 0), then width/height give the image size."""
    ref = measured if measured is not None else proj_out
    if ref is not None:
        w, h, pitch = _img_args(ref)
    else:
        w, h, pitch = int(width), int(height), int(width) * 4
    check(lib.esb_projection_loss_grad(C.byref(c), fptr(vol), _voxel_type_of(vol), w, h, fptr(measured), pitch,
                                       float(shift[0]), float(shift[1]), fptr(grad), fptr(proj_out), fptr(out),
                                       _stream(stream)))


def make_square(img, maxsize: int, out, border_x: int, border_y: int, mirror_y=False, fill_zero=True, stream=None):
    w, h, pitch = _img_args(img)
    check(lib.esb_make_square(w, h, pitch, fptr(img), maxsize, fptr(out), border_x, border_y, int(mirror_y),
                              int(fill_zero), _stream(stream)))


def ctf(spectrum, n: int, defocus_min_nm: float, defocus_max_nm: float, angle_deg: float, apply_for_fp: bool,
        phase_flip_only: bool = False, wiener: float = 0.1, beta_fac=(200, 0, 0.008, 0), cs_mm: float = 2.7,
        voltage_kv: float = 300.0, amp_contrast: float = 0.0, pixel_size_nm: float = 0.27, stream=None) -> None:
    check(lib.esb_ctf(fptr(spectrum), n, defocus_min_nm, defocus_max_nm, angle_deg, int(apply_for_fp),
                      int(phase_flip_only), wiener, fptr(_f32(beta_fac, 4)), cs_mm, voltage_kv, amp_contrast,
                      pixel_size_nm, _stream(stream)))


def wbp_weighting(spectrum, n: int, psi_deg: float, method: int = FM_RAMP, stream=None) -> None:
    check(lib.esb_wbp_weighting(fptr(spectrum), n, psi_deg, method, _stream(stream)))


def fourier_filter(spectrum, n: int, lp: float, hp: float, lps: float, hps: float, stream=None) -> None:
    check(lib.esb_fourier_filter(fptr(spectrum), n, lp, hp, lps, hps, _stream(stream)))


def dose_weighting(spectrum, n: int, dose: float, pixel_size_a: float, stream=None) -> None:
    check(lib.esb_dose_weighting(fptr(spectrum), n, dose, pixel_size_a, _stream(stream)))


def convert_volume(vol, out, negate: bool = False, stream=None) -> None:
    check(lib.esb_convert_volume(fptr(vol), _voxel_type_of(vol), vol.numel(), fptr(out), int(negate), _stream(stream)))


def store_volume(src, vol, stream=None) -> None:
    check(lib.esb_store_volume(fptr(src), src.numel(), fptr(vol), _voxel_type_of(vol), _stream(stream)))


def sart_projection_update_noalloc(cfg: "ReconConfig", pg, vg, vol, real, sirt_count: float = 1.0,
                                   volume_is_empty: bool = False, mag=None, mag_inv=None, stream=None) -> None:
    """One SART update of `vol` from projection geometry `pg` and measured
    image `real` (no CTF), allocating no device memory.

    For callers that cannot call cudaMalloc (device memory owned and budgeted
    by their own allocator, no allocation after start-up, no implicit device
    synchronisation in the loop). The two scratch images live in a fixed
    32 MiB array inside the library (projections up to 2048 x 2048 pixels),
    shared by all calls: overlapping calls on the GPU race, and the first call
    on a device, which looks up the array's address, should come before any
    stream capture. Same result as Reconstructor.reset_projections /
    forward_projection / compare / back_projection with the kernels that
    cfg.variant names (FAITHFUL or FAST).
    """
    m = _f32(IDENTITY3 if mag is None else mag, 9)
    mi = _f32(IDENTITY3 if mag_inv is None else mag_inv, 9)
    check(lib.esb_sart_projection_update_noalloc(C.byref(cfg.c()), C.byref(pg), C.byref(vg), fptr(m), fptr(mi),
                                                 fptr(vol), _voxel_type_of(vol), fptr(real), sirt_count,
                                                 int(volume_is_empty), _stream(stream)))


class _CudaArray:
    def __init__(self, address: int, shape, typestr: str = "<f4"):
        self.__cuda_array_interface__ = {"data": (int(address), False), "shape": tuple(shape), "typestr": typestr,
                                         "version": 2}


def device_view(address: int, shape, typestr: str = "<f4"):
    """Zero-copy torch view of a device buffer owned by libesb."""
    import torch

    return torch.as_tensor(_CudaArray(address, shape, typestr), device="cuda")


def kernel_launches() -> int:
    """Kernel launches issued by the library so far in this process."""
    return int(lib.esb_kernel_launches())


# --------------------------------------------------------------------------- reconstructor
@dataclass
class ReconConfig:
    """The emsart.cfg keys the hot path reads (utils/Config.cpp:303-494)."""

    proj_x: int
    proj_y: int
    n_proj: int
    lambda_: float = 1.0
    oversampling: int = 1
    ctf_mode: bool = False
    cut_length: tuple = (0.0, 0.0)
    dim_length: tuple = (1.0, 1.0)
    crop: tuple = (0.0, 0.0, 0.0, 0.0)
    crop_dim: tuple = (1.0, 1.0, 1.0, 1.0)
    projection_scale_factor: float = 1.0
    pixel_size_nm: float = 1.0
    cs_mm: float = 2.7
    voltage_kv: float = 300.0
    amp_contrast: float = 0.0
    ctf_slice_thickness_nm: float = 50.0
    ctf_beta_fac: tuple = (200.0, 0.0, 0.008, 0.0)
    wiener_noise_level: float = 0.1
    phase_flip_only: bool = False
    ignore_z_shift_for_ctf: bool = False
    switch_ctf_direction: bool = False
    volume_shift: tuple = (0.0, 0.0, 0.0)
    add_tilt_angle: float = 0.0
    variant: int = L.VARIANT_FAITHFUL

    def c(self) -> L.ReconConfig:
        r = L.ReconConfig()
        r.proj_x, r.proj_y, r.n_proj = self.proj_x, self.proj_y, self.n_proj
        r.lambda_, r.oversampling, r.ctf_mode = self.lambda_, self.oversampling, int(self.ctf_mode)
        r.cut_length[:] = list(self.cut_length)
        r.dim_length[:] = list(self.dim_length)
        r.crop[:] = list(self.crop)
        r.crop_dim[:] = list(self.crop_dim)
        r.projection_scale_factor = self.projection_scale_factor
        r.pixel_size_nm, r.cs_mm, r.voltage_kv = self.pixel_size_nm, self.cs_mm, self.voltage_kv
        r.amp_contrast, r.ctf_slice_thickness_nm = self.amp_contrast, self.ctf_slice_thickness_nm
        r.ctf_beta_fac[:] = list(self.ctf_beta_fac)
        r.wiener_noise_level, r.phase_flip_only = self.wiener_noise_level, int(self.phase_flip_only)
        r.ignore_z_shift_for_ctf = int(self.ignore_z_shift_for_ctf)
        r.switch_ctf_direction = int(self.switch_ctf_direction)
        r.volume_shift[:] = list(self.volume_shift)
        r.add_tilt_angle = self.add_tilt_angle
        r.variant = self.variant
        return r


class Reconstructor:
    """Owner of the projection buffers, FFT plans and geometry of one GPU
    (Reconstructor.cpp:203-372)."""

    def __init__(self, cfg: ReconConfig, geoms, tilt_deg, defocus=None, mag=None, mag_inv=None, stream=None):
        self.cfg = cfg
        self._geoms = geoms
        self._tilt = _f32(tilt_deg, cfg.n_proj)
        self._defocus = None if defocus is None else _f32(defocus, 3 * cfg.n_proj)
        self._mag = _f32(IDENTITY3 if mag is None else mag, 9)
        self._mag_inv = _f32(IDENTITY3 if mag_inv is None else mag_inv, 9)
        h = C.c_void_p()
        check(lib.esb_reconstructor_create(C.byref(cfg.c()), C.cast(geoms, C.c_void_p), fptr(self._tilt),
                                           fptr(self._defocus), fptr(self._mag), fptr(self._mag_inv), C.byref(h)))
        self._h = h
        check(lib.esb_reconstructor_set_stream(self._h, _stream(stream)))

    def close(self):
        if getattr(self, "_h", None):
            lib.esb_reconstructor_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def buffers(self):
        """(proj_d, dist_d, real_d) device addresses."""
        a, b, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib.esb_reconstructor_buffers(self._h, C.byref(a), C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def views(self):
        """(proj_d, dist_d, real_d) as zero-copy torch views (H x W float32)."""
        return tuple(device_view(p, (self.cfg.proj_y, self.cfg.proj_x)) for p in self.buffers())

    def reset_projections(self):
        check(lib.esb_rec_reset_projections(self._h))

    def enable_timing(self, on: bool = True):
        check(lib.esb_reconstructor_enable_timing(self._h, int(on)))

    def enable_graphs(self, on: bool = True):
        """Replay SART iterations 3.. of a sart() call from a CUDA graph
        captured on iteration 2."""
        check(lib.esb_reconstructor_enable_graphs(self._h, int(on)))

    def fuse_subsets(self, on=True):
        """Back-project each ordered subset of sart() in one volume pass:
        True, False, or None for the default (FP16 / BF16 volumes only).
        FP32 volumes come out bit for bit as with one pass per projection."""
        check(lib.esb_reconstructor_fuse_subsets(self._h, -1 if on is None else int(bool(on))))

    def subvolume_patches(self, on: bool = True):
        """subvolume_wbp with CTF: all tilts in one launch from gathered
        slab-image patches, else (the default) one launch per tilt; the
        same boxes bit for bit."""
        check(lib.esb_reconstructor_subvolume_patches(self._h, int(on)))

    def timing(self):
        """{phase: (ms, launches)} since the previous call; phases fp, bp, ctf, compare."""
        ms = np.zeros(4, np.float64)
        cnt = np.zeros(4, np.int32)
        check(lib.esb_reconstructor_timing(self._h, fptr(ms), fptr(cnt)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(("fp", "bp", "ctf", "compare"))}

    def prepare_projection(self, raw, out, **pc):
        """PrepareProjection (Reconstructor.cpp:1158-1383): raw projection
        (device tensor: float32, int16, uint16, int32 or uint32) -> normalised
        float image `out`. Keyword arguments are the fields of
        esb_prepare_config (input_type is taken from raw's dtype). Returns
        (mean, std, bad_pixels)."""
        import torch

        kinds = {torch.float32: 0, torch.int16: 1, torch.int32: 3}
        try:
            kinds[torch.uint16] = 2
            kinds[torch.uint32] = 4
        except AttributeError:
            pass
        c = L.PrepareConfig()
        c.input_type = kinds[raw.dtype]
        c.normalization = 1
        c.correct_bad_pixels = 1
        c.bad_pixel_value = 10.0
        for k, v in pc.items():
            setattr(c, k, v)
        m, s, b = C.c_float(), C.c_float(), C.c_int()
        check(lib.esb_prepare_projection(self._h, C.byref(c), fptr(raw), fptr(out), C.byref(m), C.byref(s),
                                         C.byref(b)))
        return m.value, s.value, b.value

    def cc_displacement(self, residual, model, max_shift: int, multi_peak: bool = False, cc_map=None,
                        cc_map_multi=None):
        """GetDisplacement (Reconstructor.cpp:1746-1960): the integer shift
        (x, y) at the maximum of the normalised cross-correlation of two
        H x W device images, and that maximum. cc_map / cc_map_multi:
        optional (4 max_shift)^2 device tensors for the correlation's centre
        and the multi-peak map."""
        sh = np.zeros(2, np.float32)
        v = C.c_float()
        check(lib.esb_rec_cc_displacement(self._h, fptr(residual), fptr(model), int(max_shift), int(multi_peak),
                                          fptr(sh), C.byref(v), fptr(cc_map), fptr(cc_map_multi)))
        return (float(sh[0]), float(sh[1])), v.value

    def forward_projection(self, vg, vol, index: int, volume_is_empty: bool = False):
        check(lib.esb_rec_forward_projection(self._h, C.byref(vg), fptr(vol), _voxel_type_of(vol), index,
                                             int(volume_is_empty)))

    def forward_projection_roi(self, vg, vol, index: int, roi, volume_is_empty: bool = False):
        """ForwardProjectionROI: the rays of detector region roi = (x0, y0,
        x1, y1) (x1, y1 exclusive), added to the projection buffer."""
        r = np.ascontiguousarray(np.asarray(roi, np.int32))
        check(lib.esb_rec_forward_projection_roi(self._h, C.byref(vg), fptr(vol), _voxel_type_of(vol), index,
                                                 int(volume_is_empty), fptr(r)))

    def compare(self, vg, real, index: int):
        check(lib.esb_rec_compare(self._h, C.byref(vg), fptr(real), index))

    def back_projection(self, vg, vol, index: int, sirt_count: float = 1.0):
        check(lib.esb_rec_back_projection(self._h, C.byref(vg), fptr(vol), _voxel_type_of(vol), index, sirt_count))

    def sart(self, vg, vol, projections, index_list, iterations: int, sirt_count: int, volume_is_empty: bool = True):
        """EmSart.cpp:579-675. Returns the updated volume_is_empty flag."""
        il = np.ascontiguousarray(np.asarray(index_list, np.int32))
        empty = C.c_int(int(volume_is_empty))
        check(lib.esb_sart_run(self._h, C.byref(vg), fptr(vol), _voxel_type_of(vol), fptr(projections), fptr(il),
                               il.size, iterations, sirt_count, C.byref(empty)))
        return bool(empty.value)

    def sart_zslab(self, vg, vol, projections, index_list, iterations: int, sirt_count: int, allreduce,
                   volume_is_empty: bool = True):
        """esb_sart_run_zslab: SART over this rank's z-slab (vg from
        volume_geometry(dims, subvol_count=ranks, subvol=rank)). `allreduce`
        is called once per projection as allreduce(buffer, stream): buffer a
        torch view of the slab's projection and ray lengths (2 x H x W,
        contiguous) to be summed over the ranks in place, stream the
        reconstructor's (a torch.cuda.ExternalStream) on which the sum must be
        ordered. Returns the updated volume_is_empty flag."""
        il = np.ascontiguousarray(np.asarray(index_list, np.int32))
        empty = C.c_int(int(volume_is_empty))
        H, W = self.cfg.proj_y, self.cfg.proj_x
        errors = []

        def cb(buf, count, stream, user):
            import torch

            try:
                assert count == 2 * H * W
                # stream NULL: the reconstructor runs on the default stream
                st = torch.cuda.ExternalStream(stream) if stream else torch.cuda.default_stream()
                allreduce(device_view(buf, (2, H, W)), st)
                return 0
            except Exception as e:  # reported after the call returns
                errors.append(e)
                return 1

        fn = L.ALLREDUCE_FN(cb)
        rc = lib.esb_sart_run_zslab(self._h, C.byref(vg), fptr(vol), _voxel_type_of(vol), fptr(projections),
                                    fptr(il), il.size, iterations, sirt_count, C.byref(empty), C.cast(fn, C.c_void_p),
                                    None)
        if errors:
            raise errors[0]
        check(rc)
        return bool(empty.value)

    def subvolume_wbp(self, full_vg, sub_geoms, pair_geoms, boxes, projections, index_list, active=None,
                      batched: bool = True):
        n = len(boxes)
        sg = (L.VolGeom * n)(*sub_geoms)
        ptrs = (C.c_void_p * n)(*[b.data_ptr() for b in boxes])
        act = None if active is None else np.ascontiguousarray(np.asarray(active, np.uint8))
        il = np.ascontiguousarray(np.asarray(index_list, np.int32))
        check(lib.esb_subvolume_wbp(self._h, C.byref(full_vg), n, C.cast(sg, C.c_void_p),
                                    C.cast(pair_geoms, C.c_void_p), fptr(act), C.cast(ptrs, C.c_void_p),
                                    fptr(projections), fptr(il), il.size, int(batched)))
