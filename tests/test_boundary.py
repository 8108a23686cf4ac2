"""The C ABI library loads, exports every declared entry point and rejects
invalid arguments on the host (no device work)."""
import ctypes as C

import numpy as np
import pytest

import artiatomi_b200 as E
from artiatomi_b200 import _lib as L


def test_library_exports_every_header_symbol():
    names = L.header_symbols()
    assert len(names) >= 30
    cdll = C.CDLL(str(L.LIB_PATH))
    missing = [n for n in names if not hasattr(cdll, n)]
    assert not missing, missing


def test_ctypes_signatures_cover_header():
    assert set(L.header_symbols()) <= set(L._SIGS), set(L.header_symbols()) - set(L._SIGS)


def test_struct_layouts():
    # esb_constants: 9 float3 + z_shift + int + 16 + 9 + 9 floats
    assert C.sizeof(L.Constants) == (27 + 1 + 1 + 16 + 18) * 4
    assert C.sizeof(L.ProjGeom) == (12 + 16) * 4
    assert C.sizeof(L.VolGeom) == (15 + 1 + 9) * 4


def test_invalid_arguments_are_reported():
    rc = L.lib.esb_fp(None, None, 0, 16, 16, None, None, 64, 0, 0, 16, 16, None)
    assert rc == 1
    assert b"constants" in L.lib.esb_last_error()
    c = L.Constants()
    c.volume_dim[:] = [8, 8, 8]
    rc = L.lib.esb_fp(C.byref(c), C.c_void_p(1), 0, 16, 16, C.c_void_p(1), C.c_void_p(1), 8, 0, 0, 16, 16, None)
    assert rc == 1 and b"pitch" in L.lib.esb_last_error()
    rc = L.lib.esb_bp(C.byref(c), C.c_void_p(1), 7, 16, 16, C.c_void_p(1), 64, 1.0, 1, 0.0, 1.0, 0, None)
    assert rc == 1
    rc = L.lib.esb_bp(C.byref(c), C.c_void_p(1), 0, 16, 16, C.c_void_p(1), 64, 1.0, 0, 0.0, 1.0, 0, None)
    assert rc == 1 and b"oversampling" in L.lib.esb_last_error()
    with pytest.raises(L.EsbError):
        E.volume_geometry((0, 4, 4))


def test_reconstructor_rejects_bad_config():
    cfg = E.ReconConfig(proj_x=0, proj_y=8, n_proj=1)
    geoms = E.projection_geometry(E.Markers(np.zeros(1, np.float32)), 8, 8)
    with pytest.raises(L.EsbError):
        E.Reconstructor(cfg, geoms, [0.0], stream=0)
    cfg = E.ReconConfig(proj_x=8, proj_y=8, n_proj=1, ctf_mode=True)
    with pytest.raises(L.EsbError):
        E.Reconstructor(cfg, geoms, [0.0], stream=0)


def test_kernel_launch_counter_starts_without_gpu_work():
    assert E.kernel_launches() >= 0


@pytest.mark.gpu
def test_kernel_launch_counter_counts_launches():
    from tests.helpers import cuda, small_case

    case = small_case()
    W, H = case["W"], case["H"]
    c = E.set_constant_values(case["pg"][0], case["vg"])
    vol = cuda(case["vol"])
    proj = cuda(np.zeros((H, W), np.float32))
    dist = cuda(np.zeros((H, W), np.float32))
    n0 = E.kernel_launches()
    E.forward_project(c, vol, proj, dist)
    E.forward_project(c, vol, proj, dist, fast=True)
    assert E.kernel_launches() - n0 == 2


def test_autotune_switch_and_report():
    """The launch-shape autotuner's C ABI without a GPU: the switch values,
    the refusal of others, and the report of an empty cache."""
    import ctypes as C

    import artiatomi_b200 as E
    from artiatomi_b200 import _lib as L

    try:
        for v in (0, 1, -1, 2, 5, 1):
            E.autotune(v)
        with pytest.raises(L.EsbError):
            E.autotune(-2)
        E.autotune(-1)
        assert E.autotune_report() == ""
        need = C.c_size_t(0)
        assert L.lib.esb_autotune_report(None, 0, C.byref(need)) == 0 and need.value == 1
    finally:
        E.autotune(1)
