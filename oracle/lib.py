"""ctypes binding of the oracle's C++ kernels (oracle/esb_oracle.cpp)."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import OUT, build as build_oracle

P, I, F, L = C.c_void_p, C.c_int, C.c_float, C.c_long


class OrcGeom(C.Structure):
    _fields_ = [("det", C.c_float * 3), ("u", C.c_float * 3), ("v", C.c_float * 3), ("n", C.c_float * 3),
                ("detMat", C.c_float * 16), ("bbMin", C.c_float * 3), ("bbMax", C.c_float * 3),
                ("bbRcp", C.c_float * 3), ("dim", C.c_float * 3), ("vs", C.c_float * 3), ("zShift", C.c_float),
                ("dimXQuarter", C.c_int), ("aniso", C.c_float * 9), ("anisoInv", C.c_float * 9)]


_SIGS = {
    "orc_fp_march": [C.POINTER(OrcGeom), P, I, I, I, P, P, I, I, I, I, I, I, I, I],
    "orc_rotate_volume": [P, P, I, P, I, I],
    "orc_fp_slicer": [C.POINTER(OrcGeom), P, I, I, I, P, F, F, I, I, I, I],
    "orc_vol_traversal_length": [C.POINTER(OrcGeom), I, I, P, I, I],
    "orc_compare": [I, I, P, P, P, F, P, P, F],
    "orc_crop_border": [I, I, P, P, P, P],
    "orc_bp": [C.POINTER(OrcGeom), P, I, P, I, I, F, I, F, F, I, I, I, I],
    "orc_make_square": [I, I, I, I, P, P, I, I, I, I],
    "orc_ctf": [P, I, F, F, F, I, I, F, P, F, F, F, F, I],
    "orc_wbp_weighting": [P, I, F, I],
    "orc_fourier_filter": [P, I, F, F, F, F],
    "orc_dose_weighting": [P, I, F, F],
    "orc_r2c": [P, P, I, I],
    "orc_c2r": [P, P, I, I],
    "orc_float_to_half": [P, P, L],
    "orc_half_to_float": [P, P, L],
    "orc_float_to_bf16": [P, P, L],
    "orc_model_loss_grad": [C.POINTER(OrcGeom), P, I, I, P, F, F, P, P, P, I],
}


def _load():
    path = build_oracle()
    lib = C.CDLL(str(path))
    for name, args in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = I
    return lib


olib = _load()
NTHREADS = int(os.environ.get("ORACLE_THREADS", os.cpu_count() or 1))


def addr(a: np.ndarray):
    """Pointer that keeps the (possibly temporary) array alive for the call."""
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("oracle arrays must be C-contiguous")
    return a.ctypes.data_as(C.c_void_p)


def f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))
