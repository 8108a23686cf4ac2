"""Generate the file-format fixtures of tests/test_fileio.py from the
reference's own file classes (oracle/ref_fileio, compiled from the
reference tree by oracle/ref_fileio/build.py):

* ref_written.em / ref_written.mrc: float ramp volumes (6 x 5 x 3, pixel size
  0.27 nm) written by EmFile::InitHeader / MRCFile::InitHeaders +
  WriteRawData;
* fileio_reference.json: what the reference's readers report for files that
  artiatomi_b200.fileio writes (EM/MRC of several types, a marker file, a
  CTF file), made by make_files() below.

  python tests/golden/make_fileio_golden.py    (needs the reference tree)
"""
from __future__ import annotations

import json
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
HERE = Path(__file__).resolve().parent


def make_files(d: Path) -> dict:
    """Files written by artiatomi_b200.fileio; name -> path."""
    from artiatomi_b200 import fileio as F

    rng = np.random.default_rng(5)
    out = {}
    for name, dt in (("f32", np.float32), ("i16", np.int16), ("i32", np.int32), ("u8", np.uint8)):
        a = (rng.normal(size=(3, 5, 7)) * 40).astype(dt)
        p = d / f"ours_{name}.em"
        F.write_em(str(p), a, {"ObjectPixelSize": 270})
        out[p.name] = p
    for name, dt in (("f32", np.float32), ("i16", np.int16), ("u16", np.uint16), ("u8", np.uint8)):
        a = np.abs(rng.normal(size=(3, 5, 7)) * 40).astype(dt)
        p = d / f"ours_{name}.mrc"
        F.write_mrc(str(p), a, 0.27)
        out[p.name] = p
    items = np.zeros((2, 4, 10), np.float32)
    items[:, :, 0] = np.array([-30, -10, 10, 30], np.float32)
    items[:, :, 1:3] = 100.0
    items[1, 2, 1:3] = -1.0  # marker 1 not clicked on projection 2
    items[:, :, 4] = np.array([1.5, -0.5, 0.25, 2.0], np.float32)
    items[:, :, 5] = np.array([-1.0, 0.75, 0.0, 0.5], np.float32)
    items[:, :, 8] = 1.0
    items[:, :, 9] = np.array([0.1, -0.2, 0.3, 0.0], np.float32)
    p = d / "ours_markers.em"
    F.write_markers(str(p), items)
    out[p.name] = p
    p = d / "ours_ctf.em"
    F.write_ctf(str(p), [3000.0, 3100.0, 3200.0], [3050.0, 3150.0, 3250.0], [0.1, 1.2, -0.4])
    out[p.name] = p
    motl = np.zeros((3, 20), np.float32)
    motl[:, 3] = [1, 2, 1234567]
    motl[:, 4], motl[:, 5] = [7, 7, 8], [3, 4, 12.5]
    motl[:, 7:10] = [[10.5, 20, 30], [40, 50.25, 60], [70, 80, 90.75]]
    motl[:, 10:13] = [[0.5, -0.25, 1], [0, 0, 0], [-2, 1.5, 0.125]]
    p = d / "ours_motl.em"
    F.write_motive_list(str(p), motl)
    out[p.name] = p
    stored = (np.arange(2 * 4 * 3, dtype=np.float32).reshape(2, 4, 3) - 10.0) * 0.25
    p = d / "ours_shifts.em"
    F.write_shift_file(str(p), stored)
    out[p.name] = p
    return out


def reference_report(exe: Path, files: dict) -> dict:
    rep = {}
    for name, p in files.items():
        if name == "ours_markers.em":
            args = ["markers", str(p), "1"]
        elif name == "ours_ctf.em":
            args = ["ctf", str(p), "3"]
        elif name == "ours_motl.em":
            args = ["motl", str(p), "2", "0.5"]
        elif name == "ours_shifts.em":
            args = ["shifts", str(p)]
        else:
            args = ["read", str(p)]
        rep[name] = subprocess.run([str(exe), *args], check=True, capture_output=True, text=True).stdout
    return rep


def main():
    from oracle.ref_fileio import build as B

    exe = B.build(verbose=True)
    if exe is None:
        raise SystemExit("reference file classes not available")
    subprocess.run([str(exe), "write_em", str(HERE / "ref_written.em"), "6", "5", "3", "0.27"], check=True)
    subprocess.run([str(exe), "write_mrc", str(HERE / "ref_written.mrc"), "6", "5", "3", "0.27"], check=True)
    with tempfile.TemporaryDirectory() as t:
        rep = reference_report(exe, make_files(Path(t)))
    (HERE / "fileio_reference.json").write_text(json.dumps(rep, indent=1, sort_keys=True))
    print("wrote", HERE / "ref_written.em", HERE / "ref_written.mrc", HERE / "fileio_reference.json")


if __name__ == "__main__":
    main()
