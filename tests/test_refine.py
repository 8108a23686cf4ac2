"""EmSartRefine's pieces: the rotation of the particle reference (RotKernel /
rot3d), the region-restricted projection loss with amplitude moments, the
refine-mode configuration, and the shift refinement end to end
(artiatomi_b200.refine) on a synthetic tilt series with known extra shifts.

The oracle's rotation is pinned to the reference's own rot3d kernel compiled
for the host (oracle/_ref); the CUDA rotation is checked against the oracle.
"""
import numpy as np
import pytest

from tests.helpers import cuda, host, rel_l2

ANGLES = [(0.0, 0.0, 0.0), (30.0, 45.0, 90.0), (10.5, -20.25, 33.3), (330.0, 135.0, 270.0), (17.0, 0.0, 60.0),
          (-75.0, 200.0, 12.5)]


def test_rotation_matrix_matches_oracle():
    import artiatomi_b200 as E
    from oracle import geometry as G

    table = {0, 30, 45, 60, 90, 120, 135, 150, 180, 210, 225, 240, 270, 300, 315, 330}
    for a in ANGLES:
        R = E.rotation_matrix(*a)
        O = G.rotation_matrix(*a)
        if all(float(x) in table for x in a):
            np.testing.assert_array_equal(R, O)
        else:
            np.testing.assert_allclose(R, O, rtol=0, atol=3e-7)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-6)
    # exact table values where the reference uses them
    np.testing.assert_array_equal(E.rotation_matrix(90.0, 0.0, 0.0), [[0, -1, 0], [1, 0, 0], [0, 0, 1]])


def _orc_rotate(vol, R, q9=0):
    from oracle import lib as OL

    out = np.zeros_like(vol)
    OL.olib.orc_rotate_volume(OL.addr(vol), OL.addr(out), vol.shape[0], OL.addr(np.ascontiguousarray(R, np.float32)),
                              q9, OL.NTHREADS)
    return out


def test_oracle_rotation_pinned_to_reference_kernel():
    from oracle import geometry as G
    from oracle import lib as OL
    from oracle import ref as RF

    L = RF.lib()
    if L is None:
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(4)
    vol = rng.normal(size=(24, 24, 24)).astype(np.float32)
    for a in ANGLES:
        R = np.ascontiguousarray(G.rotation_matrix(*a), np.float32)
        for q9 in (0, 1):
            ref = np.zeros_like(vol)
            assert L.ref_rot3d(OL.addr(vol), OL.addr(ref), 24, OL.addr(R), q9, OL.NTHREADS) == 0
            np.testing.assert_array_equal(_orc_rotate(vol, R, q9), ref)


REFINE_KEYS = """SizeSubVol = 16
VoxelSizeSubVol = 1
MotiveList = /data/motl.em
Reference = /data/ref.em
MaxShift = 3
ShiftOutputFile = /data/shifts.em
GroupMode = MaxCount
GroupSize = 5
SpeedUpDistance = 0
ScaleMotivelistShift = 1
ScaleMotivelistPosition = 1
MultiPeakDetection = false
"""


def test_refine_config_keys():
    from artiatomi_b200.config import EmSartConfig
    from tests.test_fileio import CFG

    c = EmSartConfig.from_text(CFG + REFINE_KEYS, refine=True)
    assert c.Reference == "/data/ref.em" and c.ShiftOutputFile == "/data/shifts.em"
    assert c.SizeSubVol == 16 and c.MaxShift == 3 and c.GroupMode == "MaxCount" and c.GroupSize == 5
    assert not c.MultiPeakDetection
    with pytest.raises(KeyError):  # required as in the reference (utils/Config.cpp:408-470)
        EmSartConfig.from_text(CFG + REFINE_KEYS.replace("Reference = /data/ref.em\n", ""), refine=True)
    with pytest.raises(ValueError):
        EmSartConfig.from_text(CFG + REFINE_KEYS.replace("MaxCount", "Nearest"), refine=True)


@pytest.mark.gpu
@pytest.mark.parametrize("size", [20, 32])
def test_rotate_volume_matches_oracle(size):
    import torch

    import artiatomi_b200 as E

    rng = np.random.default_rng(size)
    vol = rng.normal(size=(size, size, size)).astype(np.float32)
    src = cuda(vol)
    out = torch.empty_like(src)
    for a in ANGLES:
        R = E.rotation_matrix(*a)
        E.rotate_volume(src, out, R)
        ref = _orc_rotate(vol, R)
        # the kernel contracts the sample position into FMAs (~1 ulp of a
        # coordinate ~10); on white noise that moves values by ~1e-6
        assert rel_l2(host(out), ref) <= 1e-5, (a, rel_l2(host(out), ref))
    with pytest.raises(Exception):
        E.rotate_volume(src, src, E.rotation_matrix(10.0, 20.0, 30.0))  # in place is refused


@pytest.mark.gpu
def test_projection_loss_grad_roi_matches_full_image():
    """A particle box whose shadow lies inside the region, measured zero
    outside it: the region's 6 sums equal the whole image's, and the two
    moments equal sum p^2 and sum p b of the projection."""
    import torch

    import artiatomi_b200 as E
    from artiatomi_b200 import phantom as PH

    W = H = 96
    tilt = np.array([-35.0, 0.0, 50.0], np.float32)
    pg = E.projection_geometry(E.Markers(tilt, rotation_psi=np.full(3, 12.0, np.float32)), W, H)
    full = E.volume_geometry((96, 96, 32))
    sub = E.subvolume_geometry(16, 1.0, full, (50.0, 44.0, 16.0))
    box = cuda(PH.phantom_numpy((16, 16, 16), 4, seed=3))
    rng = np.random.default_rng(0)
    roi = (20, 16, 80, 76)
    for i in range(3):
        c = E.set_constant_values(pg[i], sub)
        meas = np.zeros((H, W), np.float32)
        meas[roi[1]:roi[3], roi[0]:roi[2]] = rng.normal(size=(roi[3] - roi[1], roi[2] - roi[0]))
        m = cuda(meas)
        o6 = torch.zeros(6, dtype=torch.float64, device="cuda")
        o8 = torch.zeros(8, dtype=torch.float64, device="cuda")
        p_full = torch.zeros((H, W), device="cuda")
        p_roi = torch.full((H, W), 7.0, device="cuda")
        E.projection_loss_grad(c, box, m, o6, shift=(0.3, -0.4), proj_out=p_full)
        E.projection_loss_grad_roi(c, box, m, o8, roi, shift=(0.3, -0.4), proj_out=p_roi)
        pf, pr = host(p_full), host(p_roi)
        assert np.abs(pf).sum() > 0
        outside = np.ones((H, W), bool)
        outside[roi[1]:roi[3], roi[0]:roi[2]] = False
        assert np.all(pf[outside] == 0.0)  # the shadow lies inside the region
        assert np.all(pr[outside] == 7.0)  # pixels outside the region are not written
        np.testing.assert_array_equal(pr[~outside], pf[~outside])
        np.testing.assert_allclose(host(o8)[:6], host(o6), rtol=1e-9, atol=1e-12)
        pd = pf.astype(np.float64)
        np.testing.assert_allclose(host(o8)[6:], [(pd * pd).sum(), (pd * meas).sum()], rtol=1e-6)


def _refine_dataset(tmp_path, bad=None, layout="single"):
    """Background phantom with the particle cubes zeroed, plus three rotated
    references projected with known extra shifts; files as EmSart and
    EmSartRefine read them. layout "single": one group per particle
    (MaxCount 1); "group": particles 0 and 1 form one class (ByGroup) and
    share their extra shifts; "support": as "group", with particle 2 moved
    to a supporting motive list and shifted with the group."""
    import torch

    import artiatomi_b200 as E
    from artiatomi_b200 import fileio as F
    from artiatomi_b200 import phantom as PH

    dims, W, H, n, S = (96, 96, 32), 128, 128, 5, 16
    tilt = np.linspace(-40.0, 40.0, n).astype(np.float32)
    psi = np.full(n, 8.0, np.float32)
    markers = E.Markers(tilt, rotation_psi=psi)
    pg = E.projection_geometry(markers, W, H)
    vg = E.volume_geometry(dims)
    rng = np.random.default_rng(7)
    pos = np.array([[26.0, 28.0, 16.0], [70.0, 66.0, 17.0], [28.0, 70.0, 15.0]], np.float32)
    angles = np.array([[10.0, 35.0, 70.0], [200.0, 15.0, 45.0], [0.0, 90.0, 30.0]], np.float32)
    es = rng.uniform(-1.5, 1.5, size=(n, 3, 2)).astype(np.float32)  # [projection][motive][2]
    if layout != "single":
        es[:, 1] = es[:, 0]
    if layout == "support":
        es[:, 2] = es[:, 0]
    back = PH.phantom_numpy(dims, 12, seed=2)
    r = S // 2
    for p in range(3):  # Volume::RemoveSubVolume's cube of each particle
        lo = [int(pos[p, k]) - 1 - r for k in range(3)]
        back[lo[2]:lo[2] + 2 * r, lo[1]:lo[1] + 2 * r, lo[0]:lo[0] + 2 * r] = 0.0
    # a particle reference inside a spherical mask (zero near the box faces,
    # so rotated and shifted copies read no clamped border voxels)
    zz, yy, xx = np.mgrid[0:S, 0:S, 0:S] - (S // 2)
    ref = (PH.phantom_numpy((S, S, S), 5, seed=11) * 4.0 * (xx ** 2 + yy ** 2 + zz ** 2 <= 36)).astype(np.float32)
    ref_d = cuda(ref)
    rot = torch.empty_like(ref_d)
    back_d = cuda(back)
    D = torch.zeros((n, H, W), device="cuda")
    dist = torch.zeros((H, W), device="cuda")
    for i in range(n):
        E.forward_project(E.set_constant_values(pg[i], vg), back_d, D[i], dist, fast=True)
    for p in range(3):
        E.rotate_volume(ref_d, rot, E.rotation_matrix(*angles[p]))
        sub = E.subvolume_geometry(S, 1.0, vg, pos[p], (0.0, 0.0, 0.0))
        g = E.projection_geometry(markers, W, H, extra_shift=es[:, p, :])
        for i in range(n):
            E.forward_project(E.set_constant_values(g[i], sub), rot, D[i], dist, fast=True)
    raw = (1000.0 - host(D)).astype(np.float32)
    F.write_mrc(str(tmp_path / "ts.mrc"), raw, 0.5)
    items = np.zeros((1, n, 10), np.float32)
    items[0, :, 0], items[0, :, 1:3], items[0, :, 8], items[0, :, 9] = tilt, 10.0, 1.0, psi
    if bad is not None:
        items[0, bad, 1:3] = -1.0  # reference marker not clicked: projection unusable
    F.write_markers(str(tmp_path / "markers.em"), items)
    F.write_em(str(tmp_path / "vol.em"), -back)  # EmSart writes the volume negated
    F.write_em(str(tmp_path / "ref.em"), -ref)  # an average of negated sub-volumes
    motl = np.zeros((3, 20), np.float32)
    motl[:, 3] = np.arange(1, 4)
    motl[:, 7:10] = pos
    motl[:, 16:19] = angles
    motl[:, 19] = (1, 1, 2) if layout != "single" else (1, 2, 3)
    if layout == "support":
        F.write_motive_list(str(tmp_path / "support.em"), motl[2:])
        motl = motl[:2]
    F.write_motive_list(str(tmp_path / "motl.em"), motl)
    cfg = f"""ProjectionFile = {tmp_path / 'ts.mrc'}
OutVolumeFile = {tmp_path / 'vol.em'}
MarkerFile = {tmp_path / 'markers.em'}
Lambda = 1
Iterations = 1
RecDimesions = {dims[0]} {dims[1]} {dims[2]}
UseFixPsiAngle = false
PhiAngle = 0
VolumeShift = 0 0 0
ReferenceMarker = 0
OverSampling = 1
VoxelSize = 1
DimLength = 1 1
CutLength = 1 1
SkipFilter = true
fourFilterLP = 0
fourFilterLPS = 0
fourFilterHP = 0
fourFilterHPS = 0
SIRTCount = 1
CtfMode = false
BadPixelValue = 10
CorrectBadPixels = false
ProjectionNormalization = none
WBP = false
WBPFilter = Ramp
SizeSubVol = {S}
VoxelSizeSubVol = 1
MotiveList = {tmp_path / 'motl.em'}
Reference = {tmp_path / 'ref.em'}
MaxShift = 3
ShiftOutputFile = {tmp_path / 'shifts.em'}
{"GroupMode = MaxCount" + chr(10) + "GroupSize = 1" if layout == "single" else "GroupMode = ByGroup"}
{"" if layout != "support" else "SupportingReferences = " + str(tmp_path / "ref.em") + chr(10)
 + "SupportingMotiveLists = " + str(tmp_path / "support.em") + chr(10) + "MaxDistanceSupport = 1000"}
SpeedUpDistance = 0
ScaleMotivelistShift = 1
ScaleMotivelistPosition = 1
MultiPeakDetection = false
"""
    (tmp_path / "refine.cfg").write_text(cfg)
    return es if layout != "support" else es[:, :2]


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [None, 2])
def test_refine_recovers_extra_shifts(tmp_path, bad):
    """Every particle's per-tilt extra shift comes back within 0.05 px (the
    data's rays start from the shifted detector, the fitted model translates
    the unshifted rays' samples: their sample depths differ by up to a
    step), and the ShiftFile written is the one EmSARTSubVolumes reads
    (read_shift_file)."""
    from artiatomi_b200 import fileio as F
    from artiatomi_b200.config import EmSartConfig
    from artiatomi_b200.refine import refine_shifts

    es = _refine_dataset(tmp_path, bad)
    cfg = EmSartConfig.from_file(str(tmp_path / "refine.cfg"), refine=True)
    got = refine_shifts(cfg, method="lsq")
    assert got.shape == es.shape
    if bad is not None:  # an unusable projection keeps zero shifts
        assert np.all(got[bad] == 0.0)
        es = es.copy()
        es[bad] = 0.0
    err = np.abs(got - es).max()
    assert err <= 5e-2, (err, got, es)
    np.testing.assert_array_equal(F.read_shift_file(cfg.ShiftOutputFile), got)


@pytest.mark.gpu
@pytest.mark.parametrize("multi", [False, True])
def test_refine_cc_recovers_integer_shifts(tmp_path, multi):
    """The reference's measurement (cross-correlation peak): every shift is
    an integer within 0.6 px of the true extra shift (0.5 from rounding),
    the ShiftFile holds what EmSARTSubVolumes reads, and with CCMapFileName
    set one (4 MaxShift)^2 map per particle is written per projection."""
    from artiatomi_b200 import fileio as F
    from artiatomi_b200.config import EmSartConfig
    from artiatomi_b200.refine import refine_shifts

    es = _refine_dataset(tmp_path)
    cfg = EmSartConfig.from_file(str(tmp_path / "refine.cfg"), refine=True)
    cfg.MultiPeakDetection = multi
    cfg.CCMapFileName = str(tmp_path / "ccmap_")
    got = refine_shifts(cfg)
    assert got.shape == es.shape
    np.testing.assert_array_equal(got, np.round(got))
    err = np.abs(got - es)
    assert err.max() <= 0.6 and err.mean() <= 0.35, (err, got, es)
    np.testing.assert_array_equal(F.read_shift_file(cfg.ShiftOutputFile), got)
    # MaxCount leaders keep zeroed relations (only speed-up receivers get them)
    assert (tmp_path / "shifts.em.relations").read_text() == "0; 0; 0; 0; 0\n" * 3
    S = cfg.MaxShift
    for i in range(es.shape[0]):
        maps, _ = F.read_em(str(tmp_path / f"ccmap_{i}.em"))
        assert maps.shape == (3, 4 * S, 4 * S)
        # the centre of each map is the zero shift; the maximum sits at the
        # measured shift (the unmasked map holds no larger value inside MaxShift)
        for p in range(3):
            c = 2 * S
            m = maps[p].copy()
            yy, xx = np.mgrid[0:4 * S, 0:4 * S]
            m[(xx - c) ** 2 + (yy - c) ** 2 > S * S] = -np.inf
            y, x = np.unravel_index(np.argmax(m), m.shape)
            if not multi:
                assert (x - c, y - c) == (-got[i, p, 0], -got[i, p, 1])
        if multi:
            assert F.read_em(str(tmp_path / f"ccmap_Multi_{i}.em"))[0].shape == (3, 4 * S, 4 * S)


@pytest.mark.gpu
@pytest.mark.parametrize("layout", ["group", "support"])
def test_refine_cc_groups(tmp_path, layout):
    """ByGroup: the two particles of a class are measured together and both
    get the group's shift; with a supporting particle (its own motive list
    and reference) its projection joins the model."""
    from artiatomi_b200.config import EmSartConfig
    from artiatomi_b200.refine import refine_shifts

    es = _refine_dataset(tmp_path, layout=layout)
    cfg = EmSartConfig.from_file(str(tmp_path / "refine.cfg"), refine=True)
    assert cfg.GroupMode == "ByGroup"
    assert len(cfg.SupportingReferences) == (layout == "support")
    got = refine_shifts(cfg)
    assert got.shape == es.shape
    np.testing.assert_array_equal(got[:, 0], got[:, 1])
    err = np.abs(got - es)
    assert err.max() <= 0.6 and err.mean() <= 0.35, (err, got, es)
    # the relations file: particle number, group number, correlation maximum
    lines = (tmp_path / "shifts.em.relations").read_text().splitlines()
    assert len(lines) == es.shape[1]
    fields = [ln.split("; ") for ln in lines]
    assert [f[:4] for f in fields] == ([["1", "0", "0", "0"], ["2", "0", "0", "0"], ["3", "0", "0", "1"]]
                                       if layout == "group" else [["1", "0", "0", "0"], ["2", "0", "0", "0"]])
    assert all(0.0 < float(f[4]) <= 1.0 for f in fields)


def _motl(coords, classes):
    m = np.zeros((len(coords), 20), np.float32)
    m[:, 3] = np.arange(1, len(coords) + 1)
    m[:, 7:10] = np.asarray(coords, np.float32)
    m[:, 19] = classes
    return m


def test_group_members_follow_motive_list_rules():
    """MotiveList::GetNeighbours / GetGroupCount: classes in order of first
    appearance; MaxDistance: the particle, then the others within the
    distance in row order; MaxCount: nearest first, ties by row (a particle
    with equal coordinates and a lower row leads its twin's group)."""
    from artiatomi_b200 import refine as RF

    coords = [(0, 0, 0), (10, 0, 0), (0, 3, 4), (0, 0, 5), (10, 0, 0), (30, 0, 0)]
    m = _motl(coords, (5, 2, 5, 7, 2, 5))
    assert RF.group_count(m, "ByGroup") == 3
    assert [RF.group_members(m, g, "ByGroup") for g in range(3)] == [[0, 2, 5], [1, 4], [3]]
    assert RF.group_members(m, 3, "ByGroup") == []
    assert RF.group_count(m, "MaxCount") == RF.group_count(m, "MaxDistance") == 6
    assert RF.group_members(m, 3, "MaxDistance", max_distance=5.0) == [3, 0, 2]
    assert RF.group_members(m, 0, "MaxCount", group_size=3) == [0, 2, 3]  # distances 0, 5, 5
    assert RF.group_members(m, 4, "MaxCount", group_size=2) == [1, 4]  # twin of row 1
    assert RF.group_members(m, 5, "MaxCount", group_size=99) == [5, 1, 4, 0, 2, 3]
    assert RF.global_index(m, 4) == 4  # rows differ in the particle number
    twin = m.copy()
    twin[4] = twin[1]
    assert RF.global_index(twin, 4) == 1


def test_support_members_and_remove_radius():
    from artiatomi_b200 import refine as RF
    from artiatomi_b200.config import EmSartConfig

    lead = _motl([(0, 0, 0)], (1,))[0]
    s0 = _motl([(3, 4, 0), (30, 0, 0)], (1, 1))
    s1 = _motl([(0, 0, 5.5)], (1,))
    assert RF.support_members(lead, [s0, s1], 5.0) == [(0, 0)]
    assert RF.support_members(lead, [s0, s1], 6.0) == [(0, 0), (1, 0)]
    cfg = EmSartConfig()
    cfg.VoxelSize, cfg.VoxelSizeSubVol = (4.0, 4.0, 4.0), 1.0
    assert RF._remove_radius(64, cfg) == 8  # 64 / 4 / 2
    cfg.VoxelSize, cfg.VoxelSizeSubVol = (3.0, 3.0, 3.0), 2.0
    assert RF._remove_radius(33, cfg) == 11  # 33 / 1.5 / 2 = 11.0
    assert RF._remove_radius(35, cfg) == 11  # 11.67 truncated


def test_refine_config_supporting_lists():
    from artiatomi_b200.config import EmSartConfig
    from tests.test_fileio import CFG

    c = EmSartConfig.from_text(CFG + REFINE_KEYS + "SupportingReferences = /d/a.em;/d/b.em;x;\n"
                               "SupportingMotiveLists = /d/ma.em;/d/mb.em\nMaxDistanceSupport = 40\n", refine=True)
    assert c.SupportingReferences == ["/d/a.em", "/d/b.em"]
    assert c.SupportingMotiveLists == ["/d/ma.em", "/d/mb.em"]
    assert c.MaxDistanceSupport == 40.0
    with pytest.raises(KeyError):
        EmSartConfig.from_text(CFG + REFINE_KEYS + "SupportingReferences = /d/a.em\n", refine=True)
    assert EmSartConfig.from_text(CFG + REFINE_KEYS, refine=True).SupportingReferences == []


def _visit(m, mode, speed_up, **kw):
    """Drive refine's group iteration as refine_shifts does when every group
    gets a shift: (group, receivers) in order."""
    from artiatomi_b200 import refine as RF

    processed = np.zeros(m.shape[0], bool)
    seen = []
    for g, members, lead in RF.groups(m, mode, processed, **kw):
        rec = RF.shift_receivers(m, members, mode, speed_up)
        assert rec[-1] == lead or mode == "ByGroup"
        if mode != "ByGroup":
            processed[rec] = True
        seen.append((g, rec))
    return seen


def test_group_iteration_and_speed_up():
    """EmSartRefine.cpp:697-730 and 1024-1086: a MaxCount / MaxDistance group
    hands its shift to the members within SpeedUpDistance of its leader, and
    a particle that received a shift leads no later group; ByGroup hands it
    to every member and skips nothing."""
    m = _motl([(0, 0, 0), (1, 0, 0), (10, 0, 0), (10.5, 0, 0), (30, 0, 0)], (1, 1, 2, 2, 3))
    assert _visit(m, "MaxCount", 2.0, group_size=2) == [(0, [1, 0]), (2, [3, 2]), (4, [4])]
    assert _visit(m, "MaxCount", 0.5, group_size=2) == [(0, [0]), (1, [1]), (2, [3, 2]), (4, [4])]  # 0.5 <= 0.5
    assert _visit(m, "MaxCount", 0.4, group_size=2) == [(g, [g]) for g in range(5)]
    assert _visit(m, "MaxDistance", 1.0, max_distance=1.0) == [(0, [1, 0]), (2, [3, 2]), (4, [4])]
    assert _visit(m, "MaxDistance", 0.0, max_distance=50.0) == [(g, [g]) for g in range(5)]
    assert _visit(m, "ByGroup", 0.0) == [(0, [0, 1]), (1, [2, 3]), (2, [4])]
    assert _visit(m, "MaxCount", 2.0, group_size=2, only=[2, 4]) == [(2, [3, 2]), (4, [4])]


def test_relations_text_format(tmp_path):
    from artiatomi_b200.refine import write_relations

    rel = np.array([[12, 3, 7, 0], [0, 0, 0, 0], [5, 9, 1, 4]])
    write_relations(str(tmp_path / "r"), rel, np.array([0.8125, 0.0, 1.0e-5], np.float32))
    assert (tmp_path / "r").read_text() == "12; 3; 3; 0; 0.8125\n0; 0; 0; 0; 0\n5; 9; 9; 4; 1e-05\n"


def test_particle_region_with_magnification_anisotropy():
    """EmSartRefine.cpp:815-847: the particle centre's hit point truncated to
    whole pixels, through the inverse anisotropy matrix, then floor / ceil
    -+ safeDist (minima clamped at 0). Checked against the same steps done by
    hand in double: the hit point solved on the detector plane from the
    pixel pitches, the 3 x 3 matrix applied to (x, y, 1). Cases whose hand
    values fall within 1e-3 of a whole pixel are skipped (float and double
    may round them apart)."""
    import math

    import artiatomi_b200 as E
    from types import SimpleNamespace

    from artiatomi_b200.refine import particle_roi, safe_dist

    W = H = 512
    n = 7
    rng = np.random.default_rng(3)
    tilt = np.linspace(-54.0, 54.0, n).astype(np.float32)
    m = E.Markers(tilt, rng.uniform(-3, 3, n).astype(np.float32), rng.uniform(-3, 3, n).astype(np.float32),
                  np.ones(n, np.float32), np.full(n, 4.0, np.float32))
    pg = E.projection_geometry(m, W, H, E.TiltConfig(0.0, 0.0, False, 0.0, 0.0))
    vs = (2.0, 2.0, 2.0)
    vg = E.volume_geometry((256, 256, 96), vs, (0.0, 0.0, 0.0))
    safe = safe_dist(SimpleNamespace(SizeSubVol=24, VoxelSizeSubVol=1.5, MaxShift=7))
    assert safe == 100 + 72 + 14
    inv = E.mag_aniso_matrix(float(np.float32(1) / np.float32(1.04)), 35.0, W, H)
    ident = E.mag_aniso_matrix(1.0, 35.0, W, H)
    A = np.asarray(inv, np.float64).reshape(3, 3)
    checked = moved = 0
    for i in range(n):
        g = pg[i]
        det, n_ = np.array(g.detektor, np.float64), np.array(g.proj_norm, np.float64)
        P = np.stack([np.array(g.u_pitch, np.float64), np.array(g.v_pitch, np.float64)], 1)
        for _ in range(6):
            mot = np.zeros(20, np.float32)
            mot[7:10] = rng.uniform([20, 20, 10], [236, 236, 86])
            mot[10:13] = rng.uniform(-2, 2, 3)
            c = np.array(vg.bbox_min, np.float64) + (mot[7:10].astype(np.float64) + mot[10:13] - 1.0) * 2.0 + 1.0
            t = abs(n_ @ (c - det))
            hit = c - t * n_
            uv = np.linalg.lstsq(P, hit - det, rcond=None)[0]
            if np.min(np.abs(uv - np.round(uv))) < 1e-3:
                continue
            hx, hy = int(uv[0]), int(uv[1])
            x, y = A[0, 0] * hx + A[0, 1] * hy + A[0, 2], A[1, 0] * hx + A[1, 1] * hy + A[1, 2]
            if min(abs(x - round(x)), abs(y - round(y))) < 1e-3:
                continue
            want = (max(math.floor(x) - safe, 0), max(math.floor(y) - safe, 0), math.ceil(x) + safe,
                    math.ceil(y) + safe)
            got = particle_roi(g, mot, vg, vs, safe, inv)
            assert got == want, (i, got, want)
            plain = particle_roi(g, mot, vg, vs, safe, ident)
            moved = max(moved, abs(plain[2] - got[2]), abs(plain[3] - got[3]))
            checked += 1
    assert checked >= 30
    assert moved >= 5  # the anisotropy moves the region by whole pixels
