"""ctypes binding of oracle/_ref/libref_kernels.so: the reference's own kernel
sources compiled for the host (TEST INFRASTRUCTURE; see ref_build.py).

`lib()` returns None when the library is not built (the reference tree is
not present on every machine).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from .lib import NTHREADS, OrcGeom, addr, f32

HERE = Path(__file__).resolve().parent
PATH = HERE / "_ref" / "libref_kernels.so"
P, I, F = C.c_void_p, C.c_int, C.c_float

_SIGS = {
    "ref_march": [C.POINTER(OrcGeom), P, I, I, P, P, I, I],
    "ref_slicer": [C.POINTER(OrcGeom), P, I, I, P, F, F, I, I],
    "ref_vol_traversal_length": [C.POINTER(OrcGeom), I, I, P, I],
    "ref_compare": [I, I, P, P, P, F, P, P, F],
    "ref_crop_border": [I, I, P, P, P, P],
    "ref_bp": [C.POINTER(OrcGeom), P, I, P, I, I, F, I, F, F, I, I, I],
    "ref_make_square": [I, I, I, P, P, I, I, I, I],
    "ref_ctf": [P, I, F, F, F, I, I, F, P, F, F, F, F],
    "ref_wbp_weighting": [P, I, F, I],
    "ref_fourier_filter": [P, I, F, F, F, F],
    "ref_dose_weighting": [P, I, F, F],
    "ref_rot3d": [P, P, I, P, I, I],
    "ref_conj_mul": [P, P, I],
    "ref_max_shift": [P, I, I, I],
    "ref_find_peak": [P, P, I, F],
}

_lib = None


def lib():
    global _lib
    if _lib is None and PATH.exists():
        L = C.CDLL(str(PATH))
        for name, args in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = I
        _lib = L
    return _lib


def march(g, vol, W, H, proj, dist, weight8=0):
    lib().ref_march(C.byref(g), addr(vol), W, H, addr(proj), addr(dist), weight8, NTHREADS)


def slicer(g, vol, W, H, proj, tmin, tmax, weight8=0):
    lib().ref_slicer(C.byref(g), addr(vol), W, H, addr(proj), tmin, tmax, weight8, NTHREADS)


def traversal_length(g, W, H, dist):
    lib().ref_vol_traversal_length(C.byref(g), W, H, addr(dist), NTHREADS)


def compare(real, virt, dist, real_length, crop, crop_dim, scale):
    H, W = virt.shape
    lib().ref_compare(W, H, addr(real), addr(virt), addr(dist), real_length, addr(f32(crop)), addr(f32(crop_dim)),
                      scale)


def crop_border(img, cut, dim, p):
    H, W = img.shape
    lib().ref_crop_border(W, H, addr(img), addr(f32(cut)), addr(f32(dim)), addr(np.asarray(p, np.int32)))


def bp(g, vol, fp16, img, lam, os_, dmin=0.0, dmax=9999999999999.0, linear=0, weight8=0):
    H, W = img.shape
    lib().ref_bp(C.byref(g), addr(vol), int(fp16), addr(img), W, H, lam, os_, dmin, dmax, int(linear), weight8,
                 NTHREADS)


def make_square(img, N, bx, by, mirror=0, fill_zero=1):
    H, W = img.shape
    out = np.zeros((N, N), np.float32)
    lib().ref_make_square(W, H, N, addr(img), addr(out), bx, by, mirror, fill_zero)
    return out


def ctf(spec, dmin, dmax, angle, for_fp, phase_flip, wiener, beta, cs, kv, amp, ps):
    lib().ref_ctf(addr(spec), spec.shape[0], dmin, dmax, angle, int(for_fp), int(phase_flip), wiener, addr(f32(beta)),
                  cs, kv, amp, ps)


def wbp_weighting(spec, psi, fm):
    lib().ref_wbp_weighting(addr(spec), spec.shape[0], psi, fm)


def fourier_filter(spec, lp, hp, lps, hps):
    lib().ref_fourier_filter(addr(spec), spec.shape[0], lp, hp, lps, hps)


def dose_weighting(spec, dose, ps):
    lib().ref_dose_weighting(addr(spec), spec.shape[0], dose, ps)


def conj_mul(a, b):
    """conjMul on complex64 half spectra (N x N/2+1): returns conj(a) * b."""
    out = np.ascontiguousarray(a, np.complex64).copy()
    bb = np.ascontiguousarray(b, np.complex64)
    lib().ref_conj_mul(addr(out), addr(bb), out.shape[0])
    return out


def max_shift(img, s, weighted=False):
    """maxShift / maxShiftWeighted on an N x N float32 image (a copy)."""
    out = f32(img).copy()
    lib().ref_max_shift(addr(out), out.shape[0], int(s), int(weighted))
    return out


def find_peak(img, threshold):
    """findPeak: uint8 mask, 0 at the local maxima >= threshold, 1 elsewhere."""
    im = f32(img)
    mask = np.full(im.shape, 7, np.uint8)
    lib().ref_find_peak(addr(im), addr(mask), im.shape[0], float(threshold))
    return mask
