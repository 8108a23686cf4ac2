"""Per-kernel parity: each CUDA kernel (through the C ABI) against the CPU
oracle's restatement of the reference kernel on the same seeded inputs.

Tolerances. The faithful projector/back-projector evaluate the reference's
float expressions in the same order as the FP32 oracle, so they agree to the
last bits apart from summation order: rel-L2 <= 1e-5. Against the FP64 oracle
the bar is the parity bar of 1e-3. The Fourier-space and image kernels use
CUDA's libm (expf, sinf, atan2f) against glibc/double: rel-L2 <= 1e-5.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case

pytestmark = pytest.mark.gpu

FAITHFUL_TOL = 1e-5
ORACLE64_TOL = 1e-3


@pytest.fixture(scope="module")
def case():
    return small_case(shift=1.5, psi=0.3)


def _consts(E, case, i, for_bp=False, aniso=None):
    m, mi = (None, None) if aniso is None else aniso
    return E.set_constant_values(case["pg"][i], case["vg"], m, mi, for_bp=for_bp)


def _orc(case, i, for_bp=False, aniso=None):
    from oracle import geometry as G

    m, mi = (None, None) if aniso is None else aniso
    return G.orc_geom(case["og"][i], case["vo"], m, mi, for_bp=for_bp)


@pytest.mark.parametrize("voxel", ["f32", "f16", "bf16"])
def test_forward_projection(case, voxel):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D, lib as OL

    W, H = case["W"], case["H"]
    vol32 = case["vol"]
    dt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[voxel]
    vol_d = cuda(vol32).to(dt)
    if voxel == "f32":
        vol_o, code = vol32, 0
    elif voxel == "f16":
        vol_o, code = np.zeros(vol32.shape, np.uint16), 1
        OL.olib.orc_float_to_half(OL.addr(vol32), OL.addr(vol_o), vol32.size)
    else:
        vol_o, code = np.zeros(vol32.shape, np.uint16), 2
        OL.olib.orc_float_to_bf16(OL.addr(vol32), OL.addr(vol_o), vol32.size)
    for i in range(len(case["tilt"])):
        proj = torch.full((H, W), 0.5, device="cuda")
        dist = torch.zeros((H, W), device="cuda")
        E.forward_project(_consts(E, case, i), vol_d, proj, dist)
        po = np.full((H, W), 0.5, np.float32)
        do = np.zeros((H, W), np.float32)
        D.fp_march(_orc(case, i), vol_o, code, W, H, po, do)
        assert rel_l2(host(proj), po) <= FAITHFUL_TOL
        assert rel_l2(host(dist), do) <= FAITHFUL_TOL
        p64 = np.full((H, W), 0.5, np.float32)
        d64 = np.zeros((H, W), np.float32)
        D.fp_march(_orc(case, i), vol_o, code, W, H, p64, d64, precision=1)
        assert rel_l2(host(proj), p64) <= ORACLE64_TOL


def test_forward_projection_roi_and_aniso(case):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D
    from oracle import geometry as G

    W, H = case["W"], case["H"]
    m = E.mag_aniso_matrix(1.03, 25.0, W, H)
    mi = E.mag_aniso_matrix(1.0 / 1.03, 25.0, W, H)
    vol_d = cuda(case["vol"])
    roi = (5, 9, 50, 41)
    for i in (0, 3):
        proj = torch.zeros((H, W), device="cuda")
        dist = torch.full((H, W), -1.0, device="cuda")
        E.forward_project(_consts(E, case, i, aniso=(m, mi)), vol_d, proj, dist, roi=roi)
        po = np.zeros((H, W), np.float32)
        do = np.full((H, W), -1.0, np.float32)
        D.fp_march(_orc(case, i, aniso=(m, mi)), case["vol"], 0, W, H, po, do, roi=roi)
        p, d = host(proj), host(dist)
        assert rel_l2(p, po) <= FAITHFUL_TOL and rel_l2(d, do) <= FAITHFUL_TOL
        assert np.all(d[:roi[1]] == -1.0) and np.all(p[:, roi[2]:] == 0.0)


def test_slicer_and_traversal_length(case):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D
    from oracle import geometry as G

    W, H = case["W"], case["H"]
    vol_d = cuda(case["vol"])
    for i in range(len(case["tilt"])):
        t0, t1 = G.defocus_distances(case["og"][i], case["vo"])
        mid = 0.5 * (t0 + t1)
        proj = torch.zeros((H, W), device="cuda")
        E.forward_project_slab(_consts(E, case, i), vol_d, proj, mid - 10.0, mid + 5.0)
        po = np.zeros((H, W), np.float32)
        D.fp_slicer(_orc(case, i), case["vol"], 0, W, H, po, mid - 10.0, mid + 5.0)
        assert rel_l2(host(proj), po) <= FAITHFUL_TOL
        dist = torch.full((H, W), 2.0, device="cuda")
        E.traversal_length(_consts(E, case, i), dist)
        do = np.full((H, W), 2.0, np.float32)
        D.travlen(_orc(case, i), W, H, do)
        assert rel_l2(host(dist), do) <= 1e-7


@pytest.mark.parametrize("os_,linear,slab", [(1, False, False), (2, False, False), (2, True, False), (3, True, True)])
def test_back_projection(case, os_, linear, slab):
    import artiatomi_b200 as E
    from oracle import driver as D
    from oracle import geometry as G

    W, H = case["W"], case["H"]
    rng = np.random.default_rng(11)
    vol0 = rng.normal(size=case["vol"].shape).astype(np.float32)
    vol_d = cuda(vol0)
    vol_o = vol0.copy()
    for i in range(len(case["tilt"])):
        img = rng.normal(size=(H, W)).astype(np.float32)
        dmin, dmax = 0.0, 9999999999999.0
        if slab:
            t0, t1 = G.defocus_distances(case["og"][i], case["vo"])
            dmin, dmax = 0.5 * (t0 + t1) - 8.0, 0.5 * (t0 + t1) + 8.0
        E.back_project(_consts(E, case, i, for_bp=True), vol_d, cuda(img), 0.37, os_, dmin, dmax, linear)
        D.bp(_orc(case, i, for_bp=True), vol_o, 0, img, 0.37, os_, dmin, dmax, int(linear))
    assert rel_l2(host(vol_d) - vol0, vol_o - vol0) <= FAITHFUL_TOL


@pytest.mark.parametrize("voxel", ["f16", "bf16"])
def test_back_projection_reduced_storage(case, voxel):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D, lib as OL

    W, H = case["W"], case["H"]
    rng = np.random.default_rng(12)
    vol0 = rng.normal(size=case["vol"].shape).astype(np.float32)
    dt, code = (torch.float16, 1) if voxel == "f16" else (torch.bfloat16, 2)
    vol_d = cuda(vol0).to(dt)
    vol_o = np.zeros(vol0.shape, np.uint16)
    (OL.olib.orc_float_to_half if code == 1 else OL.olib.orc_float_to_bf16)(OL.addr(vol0), OL.addr(vol_o), vol0.size)
    for i in (0, 2, 5):
        img = rng.normal(size=(H, W)).astype(np.float32)
        E.back_project(_consts(E, case, i, for_bp=True), vol_d, cuda(img), 0.5, 2)
        D.bp(_orc(case, i, for_bp=True), vol_o, code, img, 0.5, 2)
    got = host(vol_d.view(torch.int16)).astype(np.int64) if False else None
    g16 = vol_d.view(torch.int16).cpu().numpy().view(np.uint16)
    # identical float math, identical round-to-nearest-even storage
    assert np.mean(g16 != vol_o) < 1e-4


def test_compare_and_crop(case):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D

    W, H = case["W"], case["H"]
    rng = np.random.default_rng(2)
    real = rng.normal(size=(H, W)).astype(np.float32)
    virt = rng.normal(size=(H, W)).astype(np.float32) * 30
    dist = rng.uniform(0, 40, size=(H, W)).astype(np.float32)
    crop, cdim = (2.0, 3.0, 4.0, 1.0), (5.0, 6.0, 7.0, 8.0)
    v_d = cuda(virt)
    E.compare(cuda(real), v_d, cuda(dist), 32.0, crop, cdim, 1.7)
    vo = virt.copy()
    D.compare(real, vo, dist, 32.0, crop, cdim, 1.7)
    assert rel_l2(host(v_d), vo) <= 1e-6
    for p in ([3, 60, 58, 62, 5, 2, 61, 4], [0, H - 1, W - 1, H - 1, 0, 0, W - 1, 0]):
        img = rng.normal(size=(H, W)).astype(np.float32)
        i_d = cuda(img)
        E.crop_border(i_d, (2.0, 3.0), (6.0, 4.0), p)
        D.crop_border(img, (2.0, 3.0), (6.0, 4.0), p)
        assert rel_l2(host(i_d), img) <= 1e-6


@pytest.mark.parametrize("mirror,fill", [(0, 1), (1, 1), (0, 0), (1, 0)])
def test_make_square(mirror, fill):
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D

    img = np.random.default_rng(4).normal(size=(40, 56)).astype(np.float32)
    out = torch.zeros((64, 64), device="cuda")
    E.make_square(cuda(img), 64, out, 4, 12, bool(mirror), bool(fill))
    ref = D.make_square(img, 64, 4, 12, mirror, fill)
    np.testing.assert_array_equal(host(out), ref)


@pytest.mark.parametrize("for_fp,flip", [(True, False), (False, False), (False, True)])
def test_ctf_kernel(for_fp, flip):
    import artiatomi_b200 as E
    from oracle import driver as D

    N = 128
    spec = np.random.default_rng(6).normal(size=(N, N // 2 + 1, 2)).astype(np.float32)
    s_d = cuda(spec)
    cfg = dict(phase_flip_only=flip, wiener_noise_level=0.1, ctf_beta_fac=(20.0, 0.0, 0.008, 0.0), cs_mm=2.7,
               voltage_kv=300.0, amp_contrast=0.07, pixel_size_nm=0.27)
    E.ctf(s_d, N, 3050.0, 3150.0, 33.0, for_fp, flip, 0.1, cfg["ctf_beta_fac"], 2.7, 300.0, 0.07, 0.27)
    D.ctf(spec, 3050.0, 3150.0, 33.0, for_fp, cfg, precision=1)
    assert rel_l2(host(s_d), spec) <= 2e-4


@pytest.mark.parametrize("fm", [0, 1, 2, 3, 4])
def test_wbp_weighting(fm):
    import artiatomi_b200 as E
    from oracle.lib import addr, olib

    N = 96
    spec = np.random.default_rng(7).normal(size=(N, N // 2 + 1, 2)).astype(np.float32)
    s_d = cuda(spec)
    E.wbp_weighting(s_d, N, 1.7, fm)
    olib.orc_wbp_weighting(addr(spec), N, 1.7, fm)
    assert rel_l2(host(s_d), spec) <= 1e-5


def test_fourier_and_dose_filters():
    import artiatomi_b200 as E
    from oracle.lib import addr, olib

    N = 128
    rng = np.random.default_rng(8)
    for args in ((40.0, 5.0, 6.0, 2.0), (0.0, 0.0, 12.0, 0.0), (30.0, 0.0, 0.0, 0.0)):
        spec = rng.normal(size=(N, N // 2 + 1, 2)).astype(np.float32)
        s_d = cuda(spec)
        E.fourier_filter(s_d, N, *args)
        olib.orc_fourier_filter(addr(spec), N, *args)
        assert rel_l2(host(s_d), spec) <= 1e-5
    spec = rng.normal(size=(N, N // 2 + 1, 2)).astype(np.float32)
    s_d = cuda(spec)
    E.dose_weighting(s_d, N, 3.5, 2.7)
    olib.orc_dose_weighting(addr(spec), N, 3.5, 2.7)
    assert rel_l2(host(s_d), spec) <= 1e-5


def test_convert_and_store_volume():
    import torch

    import artiatomi_b200 as E

    x = np.random.default_rng(9).normal(size=(4, 5, 8)).astype(np.float32)
    for dt in (torch.float16, torch.bfloat16, torch.float32):
        v = torch.empty(x.shape, dtype=dt, device="cuda")
        E.store_volume(cuda(x), v)
        np.testing.assert_array_equal(host(v), torch.from_numpy(x).to(dt).float().numpy())
        out = torch.empty(x.shape, device="cuda")
        E.convert_volume(v, out, negate=True)
        np.testing.assert_array_equal(host(out), -torch.from_numpy(x).to(dt).float().numpy())
