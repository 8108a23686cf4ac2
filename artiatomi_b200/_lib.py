"""ctypes binding of libesb.so (include/esb.h).

The shared library is built in-tree by ``python -m artiatomi_b200.build``.
Loading fails with an ImportError if it is missing: this package has no CPU
fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "libesb.so"

ESB_OK = 0
VOXEL_F32, VOXEL_F16, VOXEL_BF16 = 0, 1, 2

f3 = C.c_float * 3
f4 = C.c_float * 4
f9 = C.c_float * 9
f16 = C.c_float * 16


class Constants(C.Structure):
    _fields_ = [("proj_norm", f3), ("detektor", f3), ("u_pitch", f3), ("v_pitch", f3), ("bbox_min", f3),
                ("bbox_max", f3), ("bbox_rcp", f3), ("volume_dim", f3), ("voxel_size", f3), ("z_shift", C.c_float),
                ("volume_dim_x_quarter", C.c_int), ("detector_matrix", f16), ("mag_aniso", f9),
                ("mag_aniso_inv", f9)]


class TiltConfig(C.Structure):
    _fields_ = [("add_tilt_angle", C.c_float), ("add_tilt_x_angle", C.c_float), ("use_fix_psi_angle", C.c_int),
                ("psi_angle", C.c_float), ("phi_angle", C.c_float)]


class ProjGeom(C.Structure):
    _fields_ = [("detektor", f3), ("u_pitch", f3), ("v_pitch", f3), ("proj_norm", f3), ("detector_matrix", f16)]


class VolGeom(C.Structure):
    _fields_ = [("bbox_min", f3), ("bbox_max", f3), ("bbox_rcp", f3), ("dim", f3), ("voxel_size", f3),
                ("z_shift", C.c_float), ("full_dim", f3), ("full_bbox_min", f3), ("full_bbox_max", f3)]


class PrepareConfig(C.Structure):
    _fields_ = [("input_type", C.c_int), ("wbp", C.c_int), ("normalization", C.c_int),
                ("correct_bad_pixels", C.c_int), ("bad_pixel_value", C.c_float), ("mirror_y", C.c_int),
                ("skip_filter", C.c_int), ("lp", C.c_float), ("hp", C.c_float), ("lps", C.c_float),
                ("hps", C.c_float), ("dose_weighting", C.c_int), ("accumulated_dose", C.c_float),
                ("pixel_size_nm", C.c_float), ("down_weight_tilts", C.c_int), ("tilt_deg", C.c_float),
                ("psi_deg", C.c_float), ("wbp_filter", C.c_int)]


class ReconConfig(C.Structure):
    _fields_ = [("proj_x", C.c_int), ("proj_y", C.c_int), ("n_proj", C.c_int), ("lambda_", C.c_float),
                ("oversampling", C.c_int), ("ctf_mode", C.c_int), ("cut_length", C.c_float * 2),
                ("dim_length", C.c_float * 2), ("crop", f4), ("crop_dim", f4),
                ("projection_scale_factor", C.c_float), ("pixel_size_nm", C.c_float), ("cs_mm", C.c_float),
                ("voltage_kv", C.c_float), ("amp_contrast", C.c_float), ("ctf_slice_thickness_nm", C.c_float),
                ("ctf_beta_fac", f4), ("wiener_noise_level", C.c_float), ("phase_flip_only", C.c_int),
                ("ignore_z_shift_for_ctf", C.c_int), ("switch_ctf_direction", C.c_int), ("volume_shift", f3),
                ("add_tilt_angle", C.c_float), ("variant", C.c_int)]

VARIANT_FAITHFUL, VARIANT_FAST = 0, 1


P = C.c_void_p
I = C.c_int
F = C.c_float
SZ = C.c_size_t

_SIGS = {
    "esb_last_error": ([], C.c_char_p),
    "esb_version": ([], I),
    "esb_kernel_launches": ([], C.c_ulonglong),
    "esb_projection_geometry": ([I, I, I, P, P, P, P, P, P, C.POINTER(TiltConfig), P], I),
    "esb_volume_geometry": ([P, I, I, P, P, C.POINTER(VolGeom)], I),
    "esb_subvolume_geometry": ([I, F, C.POINTER(VolGeom), P, P, C.POINTER(VolGeom)], I),
    "esb_mag_aniso_matrix": ([F, F, F, F, P], I),
    "esb_set_constant_values": ([C.POINTER(ProjGeom), C.POINTER(VolGeom), P, P, I, C.POINTER(Constants)], I),
    "esb_compute_hit_points": ([C.POINTER(ProjGeom), C.POINTER(VolGeom), P], I),
    "esb_defocus_distances": ([C.POINTER(ProjGeom), C.POINTER(VolGeom), I, I, C.POINTER(F), C.POINTER(F)], I),
    "esb_defocus_min_max": ([F, F, F, F, F, F, F, F, I, I, C.POINTER(F), C.POINTER(F)], I),
    "esb_projection_index_list": ([I, I, P, P, P, C.POINTER(I)], I),
    "esb_fp": ([C.POINTER(Constants), P, I, I, I, P, P, SZ, I, I, I, I, P], I),
    "esb_fp_slicer": ([C.POINTER(Constants), P, I, I, I, P, SZ, F, F, I, I, I, I, P], I),
    "esb_vol_traversal_length": ([C.POINTER(Constants), I, I, P, SZ, I, I, I, I, P], I),
    "esb_compare": ([I, I, SZ, P, P, P, F, P, P, F, P], I),
    "esb_crop_border": ([I, I, SZ, P, P, P, P, P], I),
    "esb_bp": ([C.POINTER(Constants), P, I, I, I, P, SZ, F, I, F, F, I, P], I),
    "esb_fp_fast": ([C.POINTER(Constants), P, I, I, I, P, P, SZ, I, I, I, I, P], I),
    "esb_fp_slicer_fast": ([C.POINTER(Constants), P, I, I, I, P, SZ, F, F, I, I, I, I, P], I),
    "esb_bp_fast": ([C.POINTER(Constants), P, I, I, I, P, SZ, F, I, F, F, I, P], I),
    "esb_fp_adjoint": ([C.POINTER(Constants), P, I, I, P, SZ, F, F, P], I),
    "esb_projection_loss_grad": ([C.POINTER(Constants), P, I, I, I, P, SZ, F, F, P, P, P, P], I),
    "esb_projection_loss_grad_roi": ([C.POINTER(Constants), P, I, I, I, P, SZ, F, F, P, P, P, P, P], I),
    "esb_rotation_matrix": ([F, F, F, P], I),
    "esb_autotune": ([I], I),
    "esb_autotune_report": ([C.c_char_p, SZ, C.POINTER(SZ)], I),
    "esb_rotate_volume": ([P, P, I, P, P], I),
    "esb_make_square": ([I, I, SZ, P, I, P, I, I, I, I, P], I),
    "esb_ctf": ([P, I, F, F, F, I, I, F, P, F, F, F, F, P], I),
    "esb_wbp_weighting": ([P, I, F, I, P], I),
    "esb_fourier_filter": ([P, I, F, F, F, F, P], I),
    "esb_dose_weighting": ([P, I, F, F, P], I),
    "esb_convert_volume": ([P, I, C.c_long, P, I, P], I),
    "esb_store_volume": ([P, C.c_long, P, I, P], I),
    "esb_reconstructor_create": ([C.POINTER(ReconConfig), P, P, P, P, P, C.POINTER(P)], I),
    "esb_reconstructor_destroy": ([P], I),
    "esb_reconstructor_set_stream": ([P, P], I),
    "esb_reconstructor_buffers": ([P, C.POINTER(P), C.POINTER(P), C.POINTER(P)], I),
    "esb_rec_reset_projections": ([P], I),
    "esb_reconstructor_enable_timing": ([P, I], I),
    "esb_reconstructor_timing": ([P, P, P], I),
    "esb_reconstructor_enable_graphs": ([P, I], I),
    "esb_reconstructor_fuse_subsets": ([P, I], I),
    "esb_reconstructor_subvolume_patches": ([P, I], I),
    "esb_prepare_projection": ([P, C.POINTER(PrepareConfig), P, P, C.POINTER(F), C.POINTER(F), C.POINTER(I)], I),
    "esb_rec_cc_displacement": ([P, P, P, I, I, P, C.POINTER(F), P, P], I),
    "esb_rec_forward_projection": ([P, C.POINTER(VolGeom), P, I, I, I], I),
    "esb_rec_forward_projection_roi": ([P, C.POINTER(VolGeom), P, I, I, I, P], I),
    "esb_rec_compare": ([P, C.POINTER(VolGeom), P, I], I),
    "esb_rec_back_projection": ([P, C.POINTER(VolGeom), P, I, I, F], I),
    "esb_sart_run": ([P, C.POINTER(VolGeom), P, I, P, P, I, I, I, C.POINTER(I)], I),
    "esb_sart_run_zslab": ([P, C.POINTER(VolGeom), P, I, P, P, I, I, I, C.POINTER(I), P, P], I),
    "esb_subvolume_wbp": ([P, C.POINTER(VolGeom), I, P, P, P, P, P, P, I, I], I),
    "esb_sart_projection_update_noalloc": ([C.POINTER(ReconConfig), C.POINTER(ProjGeom), C.POINTER(VolGeom), P, P, P,
                                            I, P, F, I, P], I),
}
NOALLOC_MAX_PIXELS = 2048 * 2048

# esb_allreduce_fn: int (*)(float* buf, size_t count, void* stream, void* user)
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p)


def header_symbols() -> list[str]:
    """Names of every function declared in include/esb.h."""
    import re

    text = (_HERE.parent / "include" / "esb.h").read_text()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(esb_\w+)\s*\(", text, flags=re.M)))


class EsbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"esb error {code}: {msg}")
        self.code = code


def _load():
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m artiatomi_b200.build` "
                          "(the CUDA path has no fallback)")
    lib = C.CDLL(str(LIB_PATH), mode=C.RTLD_GLOBAL)
    for name, (args, res) in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


def check(rc: int) -> None:
    if rc != ESB_OK:
        raise EsbError(rc, lib.esb_last_error().decode())


def ptr(a) -> int | None:
    """Raw address of a numpy array or torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()


def fptr(a):
    """Pointer argument for a numpy array or torch tensor. For numpy arrays the
    returned ctypes object holds a reference to the array, so a temporary
    array stays alive until the foreign call returns."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(C.c_void_p)
    return C.c_void_p(a.data_ptr())
