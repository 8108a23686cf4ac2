"""Edge cases of the reconstruction path: rectangular detectors with CTF
padding, volume widths that are not a multiple of the 4-voxel quads, empty
work lists, the 256-slab limit and invalid counts."""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2, small_case


@pytest.mark.gpu
def test_fast_sart_ragged_sizes_with_ctf():
    """W != H (the CTF square is padded on one axis only), a volume width of
    50 (the last two voxels of each row lie beyond the last quad and are never
    updated, as in the reference) and an odd depth."""
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = small_case(dims=(50, 44, 17), n_proj=5, W=72, H=56, shift=1.0, psi=0.2)
    W, H, n = case["W"], case["H"], len(case["tilt"])
    rng = np.random.default_rng(3)
    dmid = rng.uniform(2800.0, 3200.0, n)
    defocus = np.stack([dmid - 40.0, dmid + 40.0, rng.uniform(0, 180, n)], 1).astype(np.float32).ravel()
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(max(W, H)), lambda_=0.5, oversampling=2)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    v = cuda(np.zeros(case["vol"].shape, np.float32))
    rec.sart(case["vg"], v, cuda(projs), il, iterations=2, sirt_count=2)
    got = host(v)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=1)
    ref = np.zeros(case["vol"].shape, np.float32)
    orc.sart(case["vo"], ref, 0, projs, il, 2, 2)
    assert np.abs(ref).max() > 0
    assert np.all(got[:, :, 48:] == 0) and np.all(ref[:, :, 48:] == 0)
    assert rel_l2(got, ref) <= 1e-3, rel_l2(got, ref)


@pytest.mark.gpu
def test_empty_work_lists():
    import torch

    import artiatomi_b200 as E
    from artiatomi_b200 import _lib as L

    case = small_case(dims=(32, 32, 16), n_proj=3, W=32, H=32)
    rec = E.Reconstructor(E.ReconConfig(32, 32, 3, variant=E.VARIANT_FAST), case["pg"], case["tilt"])
    projs = torch.zeros((3, 32, 32), device="cuda")
    # no particles, and particles with no projection
    rec.subvolume_wbp(case["vg"], [], (L.ProjGeom * 0)(), [], projs, np.array([0, 1, 2], np.int32))
    box = torch.ones((16, 16, 16), device="cuda")
    sub = [E.subvolume_geometry(16, 1.0, case["vg"], (16, 16, 8))]
    pair = (L.ProjGeom * 3)(*[case["pg"][i] for i in range(3)])
    for batched in (False, True):
        rec.subvolume_wbp(case["vg"], sub, pair, [box], projs, np.zeros(0, np.int32), batched=batched)
        rec.subvolume_wbp(case["vg"], sub, pair, [box], projs, np.array([0, 1, 2], np.int32),
                          active=np.zeros((1, 3), np.uint8), batched=batched)
    assert float(box.min()) == 1.0 and float(box.max()) == 1.0
    # a SART run needs at least one projection
    v = torch.zeros((16, 32, 32), device="cuda")
    with pytest.raises(L.EsbError):
        rec.sart(case["vg"], v, projs, np.zeros(0, np.int32), iterations=1, sirt_count=1)
    with pytest.raises(L.EsbError):
        rec.sart(case["vg"], v, projs, np.array([0, 5], np.int32), iterations=1, sirt_count=1)


@pytest.mark.gpu
def test_more_than_256_ctf_slabs_is_reported():
    import torch

    import artiatomi_b200 as E
    from artiatomi_b200 import _lib as L
    from tests.test_parity_recon import _ctf_cfg

    case = small_case(dims=(64, 64, 64), n_proj=3, W=64, H=64)
    cfgd = dict(_ctf_cfg(64), ctf_slice_thickness_nm=0.05)  # ~0.2 voxel slabs: > 256 per projection
    defocus = np.tile(np.array([3000.0, 3100.0, 10.0], np.float32), 3)
    rec = E.Reconstructor(E.ReconConfig(64, 64, 3, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    rec.reset_projections()
    with pytest.raises(L.EsbError, match="256 CTF slabs"):
        rec.forward_projection(case["vg"], torch.zeros((64, 64, 64), device="cuda"), 1, False)


def _rotated_case(psi_deg, tilt_x):
    """A small case whose tilt axis is rotated in the detector plane by
    psi_deg (plus jitter) and, with tilt_x != 0, tilted out of the volume's
    y axis (AddTiltXAngle: the beam gets a y component)."""
    import artiatomi_b200 as E
    from oracle import geometry as G

    case = small_case(dims=(48, 48, 24), n_proj=7, W=64, H=64, shift=1.0, psi=0.3)
    psi = (case["psi"] + np.float32(psi_deg)).astype(np.float32)
    cfg = dict(add_tilt_x_angle=tilt_x) if tilt_x else {}
    case["pg"] = E.projection_geometry(E.Markers(case["tilt"], case["xs"], case["ys"], None, psi), 64, 64,
                                       E.TiltConfig(**cfg))
    case["og"] = G.projection_geometry(case["tilt"], case["xs"], case["ys"], None, psi, 64, 64, cfg)
    return case


@pytest.mark.gpu
@pytest.mark.parametrize("psi_deg,tilt_x", [(37.0, 0.0), (90.0, 0.0), (-61.0, 0.0), (12.0, 0.8)])
def test_fast_kernels_rotated_and_tilted_axes(psi_deg, tilt_x):
    """The single-axis kernels (layer walk of the projector, trapezoid chords
    of the back-projection on pre-sampled images) at large in-plane rotations,
    and the general 3-D walk / chord kernels under a tilted axis, against the
    oracle: forward projection, one back-projection of the reconstructor, and
    SART with CTF."""
    import torch

    import artiatomi_b200 as E
    from oracle import driver as D
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = _rotated_case(psi_deg, tilt_x)
    W, H, n = case["W"], case["H"], len(case["tilt"])
    vol_d = cuda(case["vol"])
    for i in range(n):
        c = E.set_constant_values(case["pg"][i], case["vg"])
        if tilt_x == 0.0:
            assert abs(c.proj_norm[1]) <= 1e-6
        else:
            assert abs(c.proj_norm[1]) > 1e-3
        proj = torch.zeros((H, W), device="cuda")
        dist = torch.zeros((H, W), device="cuda")
        E.forward_project(c, vol_d, proj, dist, fast=True)
        po = np.zeros((H, W), np.float32)
        do = np.zeros((H, W), np.float32)
        D.fp_march(G.orc_geom(case["og"][i], case["vo"]), case["vol"], 0, W, H, po, do, precision=0)
        assert rel_l2(host(proj), po) <= 1e-4, (i, rel_l2(host(proj), po))
    # one back-projection through the reconstructor (pre-sampled images, OS 2)
    # against the generic per-voxel-shadow kernel on the same cropped image
    # (both take the reference's FP32 macro-cell rectangle) and the FP64
    # oracle. At large rotations the rectangle clips the voxels' shadows and
    # its float rounding decides samples in the clipped band, so the
    # reference's own FP32 result (oracle precision 0) differs from FP64 by
    # up to ~1e-2; that difference bounds the agreement with FP64 there.
    cfgd = dict(lambda_=0.5, oversampling=2, cut_length=(1.0, 1.0), dim_length=(3.0, 3.0))
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"])
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], precision=1)
    rng = np.random.default_rng(8)
    vol0 = rng.normal(size=case["vol"].shape).astype(np.float32)
    proj_v, _, _ = rec.views()
    clipping = abs(psi_deg) % 90.0 > 5.0
    orc32 = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], precision=0)
    for i in (0, n // 2, n - 1):
        img = rng.normal(size=(H, W)).astype(np.float32)
        v = cuda(vol0)
        proj_v.copy_(cuda(img))
        rec.back_projection(case["vg"], v, i, 1.0)
        cropped = img.copy()
        D.crop_border(cropped, cfgd["cut_length"], cfgd["dim_length"], G.compute_hit_points(case["og"][i], case["vo"]))
        vg_ = cuda(vol0)
        E.back_project(E.set_constant_values(case["pg"][i], case["vg"], for_bp=True), vg_, cuda(cropped), 0.5, 2,
                       fast=True)
        e = rel_l2(host(v) - vol0, host(vg_) - vol0)
        assert e <= 1e-5, (i, e)
        vo = vol0.copy()
        orc.back_projection(case["vo"], vo, 0, i, 1.0, img=img.copy())
        e = rel_l2(host(v) - vol0, vo - vol0)
        if clipping:
            v32 = vol0.copy()
            orc32.back_projection(case["vo"], v32, 0, i, 1.0, img=img.copy())
            e_ref = rel_l2(v32 - vol0, vo - vol0)
            assert e <= max(1e-5, 1.5 * e_ref), (i, e, e_ref)
        else:
            assert e <= 1e-5, (i, e)
    # SART with CTF
    rng = np.random.default_rng(3)
    dmid = rng.uniform(2800.0, 3200.0, n)
    defocus = np.stack([dmid - 40.0, dmid + 40.0, rng.uniform(0, 180, n)], 1).astype(np.float32).ravel()
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    cfgd = dict(_ctf_cfg(max(W, H)), lambda_=0.5, oversampling=2)
    rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"], defocus)
    v = cuda(np.zeros(case["vol"].shape, np.float32))
    rec.sart(case["vg"], v, cuda(projs), il, iterations=2, sirt_count=2)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=1)
    ref = np.zeros(case["vol"].shape, np.float32)
    orc.sart(case["vo"], ref, 0, projs, il, 2, 2)
    assert np.abs(ref).max() > 0
    tol = 1e-3
    if clipping:
        ref32 = np.zeros(case["vol"].shape, np.float32)
        OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus, precision=0).sart(case["vo"], ref32, 0,
                                                                                            projs, il, 2, 2)
        tol = max(tol, 1.5 * rel_l2(ref32, ref))
    assert rel_l2(host(v), ref) <= tol, (rel_l2(host(v), ref), tol)


@pytest.mark.gpu
@pytest.mark.parametrize("ctf", [False, True])
def test_subvolume_wbp_rotated_axis(ctf):
    """Sub-volume WBP with the tilt axis rotated 37 degrees in the detector
    plane (single-axis sums, oversampling-2 texel patches, the reference's
    clipping macro-cell rectangle): batched against per-particle launches,
    and both against the FP64 oracle within 1.5x the reference's own FP32
    deviation from it."""
    from tests.test_parity_fast import _subvolume_case, _subvolume_gpu, _subvolume_oracle

    c = _subvolume_case(ctf, [16, 24, 32, 16], n=7, seed=9, psi_deg=37.0)
    il = np.arange(c["n"], dtype=np.int32)
    plain = _subvolume_gpu(c, False, il)
    batch = _subvolume_gpu(c, True, il)
    o64 = _subvolume_oracle(c, il)
    o32 = _subvolume_oracle(c, il, precision=0)
    for a, b, r64, r32 in zip(plain, batch, o64, o32):
        assert np.abs(a).sum() > 0
        assert rel_l2(b, a) <= 1e-5, rel_l2(b, a)
        tol = max(1e-4 if not ctf else 1e-3, 1.5 * rel_l2(r32, r64))
        assert rel_l2(b, r64) <= tol, (rel_l2(b, r64), tol)


@pytest.mark.gpu
def test_fast_projection_of_a_volume_above_2_32_voxels():
    """A 1024 x 4100 x 1024 FP16 volume (4.3e9 voxels, 8.6 GB) with content in
    an 8-plane y band only: single-axis rays stay in one y plane, so the
    projection of the detector columns over the band equals that of the
    band alone (its own 1024 x 8 x 1024 volume at the same place). The walk
    then takes 64-bit element offsets."""
    import ctypes as C

    import torch

    import artiatomi_b200 as E

    X, Y, Z, yb = 1024, 4100, 1024, 4088
    assert X * Y * Z > 2 ** 32
    W, H = 4100, 1600
    tilt = np.array([-50.0, 0.0, 35.0], np.float32)
    pg = E.projection_geometry(E.Markers(tilt), W, H)
    vg = E.volume_geometry((X, Y, Z))
    band = torch.randn((Z, 8, X), device="cuda").half()
    big = torch.zeros((Z, Y, X), dtype=torch.float16, device="cuda")
    big[:, yb:yb + 8, :] = band
    # the band's own volume geometry: vg cut to y planes [yb, yb + 8)
    bg = E.volume_geometry((X, Y, Z))
    vs = float(vg.voxel_size[1])
    bg.bbox_min[1] = vg.bbox_min[1] + yb * vs
    bg.bbox_max[1] = bg.bbox_min[1] + 8 * vs
    bg.dim[1] = 8.0
    bg.bbox_rcp[1] = 1.0 / (8 * vs)
    for i in range(len(tilt)):
        cb = E.set_constant_values(pg[i], vg)
        cs = E.set_constant_values(pg[i], bg)
        # detector columns whose rays cross the band's interior planes
        u = [int(np.floor(np.dot(np.array(cb.detector_matrix[0:3]), [0.0, vg.bbox_min[1] + (yb + k) * vs, 0.0])
                          + cb.detector_matrix[3])) for k in (2, 6)]
        roi = (min(u), 0, max(u), H)
        outs = []
        for vol, c in ((big, cb), (band.contiguous(), cs)):
            proj = torch.zeros((H, W), device="cuda")
            dist = torch.zeros((H, W), device="cuda")
            E.forward_project(c, vol, proj, dist, roi=roi, fast=True)
            outs.append(host(proj)[:, roi[0]:roi[2]])
        assert np.abs(outs[1]).sum() > 0
        assert rel_l2(outs[0], outs[1]) <= 1e-3, (i, rel_l2(outs[0], outs[1]))
    del big
    torch.cuda.empty_cache()


@pytest.mark.gpu
@pytest.mark.parametrize("ctf", [False, True])
def test_autotuned_launch_shapes_do_not_change_results(ctf):
    """The reconstructor's launch-shape autotuner: every candidate shape of
    the fast projector and the single-axis back-projector gives the same
    volume bit for bit, the tuned run as well, and the choices are cached
    per problem shape."""
    import artiatomi_b200 as E
    from tests.test_parity_recon import _ctf_cfg, _projections

    case = small_case(dims=(48, 40, 20), n_proj=5, W=56, H=48, shift=1.0, psi=0.3)
    W, H, n = case["W"], case["H"], len(case["tilt"])
    projs = cuda(_projections(case))
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    defocus = np.tile(np.array([3000.0, 3080.0, 25.0], np.float32), n) if ctf else None
    cfgd = dict(_ctf_cfg(max(W, H)), lambda_=0.5, oversampling=2) if ctf else dict(lambda_=0.5, oversampling=2)

    def run():
        rec = E.Reconstructor(E.ReconConfig(W, H, n, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"],
                              defocus)
        v = cuda(np.zeros(case["vol"].shape, np.float32))
        rec.sart(case["vg"], v, projs, il, iterations=1, sirt_count=2)
        return host(v)

    try:
        vols = []
        for k in range(5):  # candidate k of every tuned kernel
            E.autotune(2 + k)
            vols.append(run())
        E.autotune(-1)
        E.autotune(1)
        vols.append(run())
        report = E.autotune_report()
    finally:
        E.autotune(1)
    assert np.abs(vols[0]).max() > 0
    for v in vols[1:]:
        np.testing.assert_array_equal(v, vols[0])
    assert "bp_axis" in report and ("fp_slicer_fused" if ctf else "fp_march") in report, report
