"""The drop-in reconstruction call: emsart.cfg + tilt series + marker file in,
volume file out (artiatomi_b200.reconstruct), against the same run on the
oracle (PrepareProjection and the SART / WBP loop restated on the CPU)."""
import numpy as np
import pytest

from tests.helpers import rel_l2

DIMS, W, H, N = (64, 64, 24), 64, 64, 9


def _dataset(tmp_path, wbp=False):
    from artiatomi_b200 import fileio as F
    from artiatomi_b200 import phantom as PH
    from oracle import driver as D
    from oracle import geometry as G

    tilt = PH.tilt_series(N, -60.0, 60.0)
    xs, ys, psi = PH.alignment(N, seed=4, shift=1.0, psi_jitter=0.3)
    og = G.projection_geometry(tilt, xs, ys, None, psi, W, H)
    vo = G.volume_geometry(DIMS)
    vol = PH.phantom_numpy(DIMS, 20, seed=6)
    stack = np.zeros((N, H, W), np.float32)
    for i in range(N):
        p = np.zeros((H, W), np.float32)
        d = np.zeros((H, W), np.float32)
        D.fp_march(G.orc_geom(og[i], vo), vol, 0, W, H, p, d)
        stack[i] = p
    raw = np.clip(np.round(1000.0 + 40.0 * stack), 0, 32000).astype(np.int16)  # detector counts
    F.write_mrc(str(tmp_path / "ts.mrc"), raw, 0.5)
    items = np.zeros((1, N, 10), np.float32)
    items[0, :, 0], items[0, :, 1:3] = tilt, 10.0
    items[0, :, 4], items[0, :, 5], items[0, :, 8], items[0, :, 9] = xs, ys, 1.0, psi
    F.write_markers(str(tmp_path / "markers.em"), items)
    cfg = f"""ProjectionFile = {tmp_path / 'ts.mrc'}
OutVolumeFile = {tmp_path / 'vol.em'}
MarkerFile = {tmp_path / 'markers.em'}
Lambda = {1.0 if wbp else 0.5}
Iterations = 2
RecDimesions = {DIMS[0]} {DIMS[1]} {DIMS[2]}
UseFixPsiAngle = false
PhiAngle = 0
VolumeShift = 0 0 0
ReferenceMarker = 0
OverSampling = 2
VoxelSize = 1
DimLength = 4 4
CutLength = 2 2
SkipFilter = false
fourFilterLP = 28
fourFilterLPS = 4
fourFilterHP = 0
fourFilterHPS = 0
SIRTCount = 3
CtfMode = false
BadPixelValue = 10
CorrectBadPixels = true
ProjectionNormalization = std
WBP = {'true' if wbp else 'false'}
WBPFilter = Ramp
"""
    (tmp_path / "emsart.cfg").write_text(cfg)
    return raw, tilt, psi, og, vo


def _oracle_run(cfg, raw, tilt, psi, og, vo):
    import artiatomi_b200 as E
    from oracle.driver import OracleReconstructor, prepare_projection

    pc = dict(wbp=int(cfg.WBP), normalization=cfg.ProjectionNormalization, correct_bad_pixels=1,
              bad_pixel_value=cfg.BadPixelValue, skip_filter=int(cfg.SkipFilter), lp=float(cfg.fourFilterLP),
              hp=float(cfg.fourFilterHP), lps=float(cfg.fourFilterLPS), hps=float(cfg.fourFilterHPS),
              wbp_filter=cfg.WBPFilter)
    prepared = np.stack([prepare_projection(raw[i], max(W, H), dict(pc, tilt_deg=float(tilt[i]),
                                                                    psi_deg=float(psi[i])))[0]
                         for i in range(N)])
    cfgd = dict(lambda_=cfg.Lambda, oversampling=cfg.OverSampling, cut_length=cfg.CutLength,
                dim_length=cfg.DimLength)
    orc = OracleReconstructor(cfgd, W, H, og, tilt, precision=1)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, tilt)
    v = np.zeros(DIMS[::-1], np.float32)
    if cfg.WBP:
        for i in il:
            orc.back_projection(vo, v, 0, int(i), 1.0, img=prepared[int(i)].copy())
    else:
        orc.sart(vo, v, 0, prepared, il, cfg.Iterations, cfg.SIRTCount)
    return -v


@pytest.mark.gpu
@pytest.mark.parametrize("wbp", [False, True])
def test_reconstruct_matches_oracle(tmp_path, wbp):
    from artiatomi_b200 import fileio as F
    from artiatomi_b200.config import EmSartConfig
    from artiatomi_b200.reconstruct import reconstruct

    raw, tilt, psi, og, vo = _dataset(tmp_path, wbp)
    cfg = EmSartConfig.from_file(str(tmp_path / "emsart.cfg"))
    out, stats = reconstruct(cfg)
    written, hdr = F.read_em(str(tmp_path / "vol.em"))
    np.testing.assert_array_equal(written, out)
    assert int(hdr["ObjectPixelSize"]) == 500
    ref = _oracle_run(cfg, raw, tilt, psi, og, vo)
    assert np.abs(ref).max() > 0
    assert rel_l2(out, ref) <= 1e-3, rel_l2(out, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("batched", [False, True])
def test_reconstruct_subvolumes_matches_oracle(tmp_path, batched):
    """EmSartSubVolumes' run from config, motive list and shift file against
    the oracle's sub-volume WBP on the oracle-prepared projections."""
    import artiatomi_b200 as E
    from artiatomi_b200 import fileio as F
    from artiatomi_b200.config import EmSartConfig
    from artiatomi_b200.reconstruct import reconstruct_subvolumes
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor, prepare_projection

    raw, tilt, psi, og, vo = _dataset(tmp_path, wbp=True)
    rng = np.random.default_rng(12)
    n_part, S = 5, 16
    motl = np.zeros((n_part, 20), np.float32)
    motl[:, 3] = np.arange(1, n_part + 1)
    motl[:, 7:10] = np.stack([rng.uniform(20, 44, n_part), rng.uniform(20, 44, n_part), rng.uniform(8, 16, n_part)], 1)
    motl[:, 10:13] = rng.uniform(-1, 1, (n_part, 3))
    F.write_motive_list(str(tmp_path / "motl.em"), motl)
    stored = rng.uniform(-1.8, 1.8, (2, N, n_part)).astype(np.float32)
    F.write_shift_file(str(tmp_path / "shifts.em"), stored)
    (tmp_path / "sub").mkdir()
    text = (tmp_path / "emsart.cfg").read_text() + f"""SizeSubVol = {S}
VoxelSizeSubVol = 1
MotiveList = {tmp_path / 'motl.em'}
SubVolPath = {tmp_path / 'sub'}/
ShiftInputFile = {tmp_path / 'shifts.em'}
BatchSize = 3
MaxShift = 2
ScaleMotivelistShift = 1
ScaleMotivelistPosition = 1
"""
    cfg = EmSartConfig.from_text(text, subvolumes=True)
    got = reconstruct_subvolumes(cfg, batched=batched)
    assert sorted(got) == sorted(str(tmp_path / "sub" / f"{i}.em") for i in range(1, n_part + 1))
    # oracle
    pc = dict(wbp=1, normalization=cfg.ProjectionNormalization, correct_bad_pixels=1,
              bad_pixel_value=cfg.BadPixelValue, skip_filter=int(cfg.SkipFilter), lp=float(cfg.fourFilterLP),
              hp=float(cfg.fourFilterHP), lps=float(cfg.fourFilterLPS), hps=float(cfg.fourFilterHPS),
              wbp_filter=cfg.WBPFilter)
    prepared = np.stack([prepare_projection(raw[i], max(W, H), dict(pc, tilt_deg=float(tilt[i]),
                                                                    psi_deg=float(psi[i])))[0]
                         for i in range(N)])
    xs = F.read_markers(cfg.MarkerFile).item("X_Shift")
    ys = F.read_markers(cfg.MarkerFile).item("Y_Shift")
    es = -np.moveaxis(stored, 0, -1)  # [projection][motive][2]
    subo = [G.subvolume_geometry(S, 1.0, vo, motl[p, 7:10], motl[p, 10:13]) for p in range(n_part)]
    pair_o = [G.projection_geometry(tilt, xs, ys, None, psi, W, H, extra_shift=es[:, p, :]) for p in range(n_part)]
    active = (np.sqrt((es ** 2).sum(2)).T < 1.5).astype(np.uint8)
    cfgd = dict(lambda_=cfg.Lambda, oversampling=cfg.OverSampling, cut_length=cfg.CutLength,
                dim_length=cfg.DimLength)
    orc = OracleReconstructor(cfgd, W, H, og, tilt, precision=1)
    bo = [np.zeros((S, S, S), np.float32) for _ in range(n_part)]
    il = E.projection_index_list(E.PLT_NORMAL, tilt)
    orc.subvolume_wbp(vo, subo, pair_o, bo, prepared, il, active=active)
    for p in range(n_part):
        name = str(tmp_path / "sub" / f"{p + 1}.em")
        box = F.read_em(name)[0]
        np.testing.assert_array_equal(box, got[name])
        assert np.abs(bo[p]).max() > 0
        assert rel_l2(box, -bo[p]) <= 1e-3, (p, rel_l2(box, -bo[p]))
