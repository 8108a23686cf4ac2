"""EM / MRC / marker / CTF files and the emsart.cfg parser.

Pinned to the reference's own file classes (src/EmTools/FileIO, compiled
for the host by oracle/ref_fileio/build.py): tests/golden/ref_written.{em,mrc}
were written by the reference's writers and must read back here;
tests/golden/fileio_reference.json holds what the reference's readers report
for the files artiatomi_b200.fileio writes (tests/golden/make_fileio_golden.py),
and where the reference tree is present the same check runs live.
"""
import json
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from artiatomi_b200 import fileio as F
from artiatomi_b200.config import EmSartConfig, parse_config

GOLDEN = Path(__file__).resolve().parent / "golden"
# reference DataType_enum (src/EmTools/Basics/Default.h)
DT = {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.float32): 5, np.dtype(np.int16): 8,
      np.dtype(np.int32): 9}


def _summary(a):
    return a.shape[2], a.shape[1], a.shape[0], DT[a.dtype], float(a.astype(np.float64).sum())


def test_reads_files_the_reference_wrote():
    ramp = (0.5 * np.arange(6 * 5 * 3, dtype=np.float32) - 7.0).reshape(3, 5, 6)
    a, hdr = F.read_em(str(GOLDEN / "ref_written.em"))
    np.testing.assert_array_equal(a, ramp)
    assert int(hdr["ObjectPixelSize"]) == 270
    b, mh = F.read_mrc(str(GOLDEN / "ref_written.mrc"))
    np.testing.assert_array_equal(b, ramp)
    assert abs(F.mrc_pixel_size_nm(mh) - 0.27) < 1e-6


def _check_reports(reports, files):
    from tests.golden.make_fileio_golden import make_files  # noqa: F401

    for name, text in reports.items():
        p = files[name]
        if name == "ours_markers.em":
            md = F.read_markers(str(p), ref_marker=1)
            rows = [list(map(float, ln.split())) for ln in text.strip().splitlines()]
            good = md.good()
            m = md.markers()
            for i, r in enumerate(rows):
                assert r[:5] == pytest.approx([m.tilt_angle[i], m.x_shift[i], m.y_shift[i], m.magnification[i],
                                               m.rotation_psi[i]], abs=1e-6)
                assert bool(r[5]) == bool(good[i])
        elif name == "ours_ctf.em":
            d = F.read_ctf(str(p))
            rows = np.array([list(map(float, ln.split())) for ln in text.strip().splitlines()])
            np.testing.assert_allclose(d, rows, rtol=1e-6, atol=1e-5)
        elif name == "ours_motl.em":
            m = F.read_motive_list(str(p), 2.0, 0.5)
            for i, ln in enumerate(text.strip().splitlines()):
                v = ln.split()
                np.testing.assert_allclose(m[i, 7:13], list(map(float, v[:6])), rtol=1e-7)
                assert F.index_coding(m[i]) == v[6]
                assert F.index_coding(m[i], tomo_particle=True) == v[7]
        elif name == "ours_shifts.em":
            sh = F.read_shift_file(str(p))  # [projection][motive][2]
            rows = np.array([list(map(float, ln.split())) for ln in text.strip().splitlines()])
            np.testing.assert_array_equal(sh.reshape(-1, 2), rows.astype(np.float32))
        else:
            vals = text.split()
            a = F.read_em(str(p))[0] if name.endswith(".em") else F.read_mrc(str(p))[0]
            nx, ny, nz, dt, s = _summary(a)
            assert [int(v) for v in vals[:4]] == [nx, ny, nz, dt], name
            assert float(vals[5]) == pytest.approx(s, rel=1e-12, abs=1e-9), name
            if name.endswith(".em"):
                assert int(vals[4]) == 270
            else:
                assert float(vals[4]) == pytest.approx(0.27, rel=1e-6)


def test_reference_reads_our_files_golden():
    from tests.golden.make_fileio_golden import make_files

    reports = json.loads((GOLDEN / "fileio_reference.json").read_text())
    with tempfile.TemporaryDirectory() as d:
        files = make_files(Path(d))
        _check_reports(reports, files)


def test_reference_reads_our_files_live():
    from oracle.ref_fileio import build as B
    from tests.golden.make_fileio_golden import make_files, reference_report

    if not B.available():
        pytest.skip("reference tree not present (the golden report covers this machine)")
    exe = B.build()
    with tempfile.TemporaryDirectory() as d:
        files = make_files(Path(d))
        _check_reports(reference_report(exe, files), files)
        # and the reference's writers, fresh
        for kind, ext in (("write_em", "em"), ("write_mrc", "mrc")):
            p = Path(d) / f"ref.{ext}"
            subprocess.run([str(exe), kind, str(p), "4", "3", "2", "0.5"], check=True)
            a = F.read_em(str(p))[0] if ext == "em" else F.read_mrc(str(p))[0]
            np.testing.assert_array_equal(a.ravel(), 0.5 * np.arange(24, dtype=np.float32) - 7.0)


@pytest.mark.parametrize("dt", [np.float32, np.int16, np.int32, np.uint8, np.float16, np.float64, np.complex64])
def test_em_roundtrip(dt, tmp_path):
    a = (np.random.default_rng(0).normal(size=(4, 3, 5)) * 20).astype(dt)
    F.write_em(str(tmp_path / "a.em"), a, {"Voltage": 300, "MagAnisotropyFactor": 1.01})
    b, h = F.read_em(str(tmp_path / "a.em"))
    np.testing.assert_array_equal(b, a)
    assert int(h["Voltage"]) == 300 and abs(float(h["MagAnisotropyFactor"]) - 1.01) < 1e-6
    assert (tmp_path / "a.em").stat().st_size == 512 + a.nbytes


def test_em_big_endian(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(1, 3, 4)
    hdr = np.zeros(1, F._em_header_dtype(">"))[0]
    hdr["MachineCoding"], hdr["DataType"], hdr["DimX"], hdr["DimY"], hdr["DimZ"] = 5, 5, 4, 3, 1
    (tmp_path / "b.em").write_bytes(hdr.tobytes() + a.astype(">f4").tobytes())
    np.testing.assert_array_equal(F.read_em(str(tmp_path / "b.em"))[0], a)


@pytest.mark.parametrize("dt", [np.float32, np.int16, np.uint16, np.uint8, np.float16])
def test_mrc_roundtrip(dt, tmp_path):
    a = np.abs(np.random.default_rng(1).normal(size=(3, 4, 6)) * 30).astype(dt)
    F.write_mrc(str(tmp_path / "a.mrc"), a, 0.54)
    b, h = F.read_mrc(str(tmp_path / "a.mrc"))
    np.testing.assert_array_equal(b, a)
    assert abs(F.mrc_pixel_size_nm(h) - 0.54) < 1e-6
    assert bytes(h["CMAP"]) == b"MAP "


def test_mrc_extended_header_and_half_modes(tmp_path):
    a = np.linspace(-1, 1, 24, dtype=np.float16).reshape(2, 3, 4)
    F.write_mrc(str(tmp_path / "h.mrc"), a, 1.0, half_mode=12)
    assert int(F.read_mrc(str(tmp_path / "h.mrc"))[1]["MODE"]) == 12
    np.testing.assert_array_equal(F.read_mrc(str(tmp_path / "h.mrc"))[0], a)
    # an extended header of NEXT bytes sits between the header and the data
    raw = bytearray((tmp_path / "h.mrc").read_bytes())
    hdr = np.frombuffer(bytes(raw[:1024]), F._mrc_header_dtype("<"))[0].copy()
    hdr["NEXT"] = 256
    (tmp_path / "e.mrc").write_bytes(hdr.tobytes() + b"\x07" * 256 + bytes(raw[1024:]))
    np.testing.assert_array_equal(F.read_mrc(str(tmp_path / "e.mrc"))[0], a)


def test_write_volume_by_extension(tmp_path):
    v = np.random.default_rng(2).normal(size=(2, 3, 4)).astype(np.float32)
    F.write_volume(str(tmp_path / "v.em"), v, 0.27, 2.0)
    a, h = F.read_em(str(tmp_path / "v.em"))
    np.testing.assert_array_equal(a, v)
    assert int(h["ObjectPixelSize"]) == int(0.27 * 2.0 * 1000)
    F.write_volume(str(tmp_path / "v.rec"), v, 0.27, 2.0)
    assert abs(F.mrc_pixel_size_nm(F.read_mrc(str(tmp_path / "v.rec"))[1]) - 0.54) < 1e-6
    F.write_volume(str(tmp_path / "v.raw"), v, 0.27)
    raw = (tmp_path / "v.raw").read_bytes()
    assert list(np.frombuffer(raw[:12], "<i4")) == [4, 3, 2]
    assert np.frombuffer(raw[12:16], "<f4")[0] == v.max()
    np.testing.assert_array_equal(np.frombuffer(raw[16:], "<f4").reshape(v.shape), v)


CFG = """# EmSART configuration
CudaDeviceID = 0
ProjectionFile = /data/ts.mrc
OutVolumeFile = /data/vol.em
MarkerFile = /data/markers.em
Lambda = 0.5
Iterations = 3
RecDimesions = 256, 256, 128
UseFixPsiAngle = false
PhiAngle = 0
VolumeShift = [0 0 -10]
ReferenceMarker = 1
OverSampling = 2
VoxelSize = 2
DimLength = 20 20
CutLength = {10; 10}
SkipFilter = true
fourFilterLP = 100
fourFilterLPS = 20
fourFilterHP = 2
fourFilterHPS = 1
SIRTCount = 4
CtfMode = YES
CtfFile = /data/defocus.em
Cs = 2.7
Voltage = 300
BadPixelValue = 8
CorrectBadPixels = true
ProjectionNormalization = std
WBPFilter = Contrast10
MagAnisotropy = 1.02 35
group = (
  Unused = 1
)
"""


def test_config_parser():
    c = EmSartConfig.from_text(CFG)
    assert c.ProjectionFile == "/data/ts.mrc" and c.OutVolumeFile == "/data/vol.em"
    assert c.Lambda == 0.5 and c.Iterations == 3 and c.RecDimensions == (256, 256, 128)
    assert c.VolumeShift == (0.0, 0.0, -10.0) and c.VoxelSize == (2.0, 2.0, 2.0)
    assert c.DimLength == (20.0, 20.0) and c.CutLength == (10.0, 10.0)
    assert c.SkipFilter and c.CtfMode and c.CtfFile == "/data/defocus.em"
    assert c.SIRTCount == 4 and c.OverSampling == 2 and c.ReferenceMarker == 1
    assert c.ProjectionNormalization == 1 and c.WBPFilter == 3 and c.MagAnisotropy == (1.02, 35.0)
    assert c.CTFBetaFac == (200.0, 0.0, 0.008, 0.0) and c.CTFSliceThickness == 50.0  # defaults
    assert parse_config(CFG)["Unused"] == "1"
    # as in the reference's parser, a line holding ')' closes a group and is
    # never read as a value
    assert "RecDimesions" not in parse_config("RecDimesions = (1, 2, 3)\n")
    with pytest.raises(KeyError):
        EmSartConfig.from_text(CFG.replace("Lambda = 0.5\n", ""))
