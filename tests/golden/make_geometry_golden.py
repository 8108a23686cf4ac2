"""Write tests/golden/geometry_reference.json: the reference's own host
geometry (Projection / Volume / Config / MarkerFile, compiled unmodified from
the reference tree into oracle/_ref/ref_geometry by
oracle/ref_geometry/build.py) on seeded alignment cases.

Each case stores its inputs (marker items, tilt configuration keys, detector
size, pixel size, volume dimensions, voxel size, volume shift, z-slab count)
and the harness's output: per z-slab the bounding box, reciprocal, dimension
and z shift; per projection the detector corner, u / v pitch, normal and
detector matrix; per projection and slab the four hit points. Floats are
kept as hex strings (exact).

    python tests/golden/make_geometry_golden.py
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

OUT = Path(__file__).resolve().parent / "geometry_reference.json"

# (name, projections, W, H, dims, subvols, tilt config, voxel size, volume shift, magnification, shift, psi jitter)
CASES = [
    ("single_axis", 9, 64, 64, (64, 64, 32), 1, {}, 1.0, (0, 0, 0), None, 2.0, 0.0),
    ("shifts_psi_jitter", 13, 96, 80, (96, 80, 40), 2, {}, 1.0, (0, 0, 0), None, 2.0, 0.3),
    ("magnification", 7, 64, 48, (64, 48, 24), 1, {}, 1.0, (0, 0, 0), 1.02, 1.5, 0.2),
    ("add_tilt_and_phi", 7, 64, 64, (64, 64, 32), 3, {"AddTiltAngle": 1.5, "PhiAngle": 0.7}, 1.0, (0, 0, 0), None,
     1.0, 0.1),
    ("tilted_axis", 7, 64, 64, (64, 64, 32), 1, {"AddTiltXAngle": 2.0}, 1.0, (0, 0, 0), None, 1.0, 0.0),
    ("fix_psi_voxel_size_shift", 9, 128, 96, (64, 48, 20), 2, {"UseFixPsiAngle": "true", "PsiAngle": 0.4}, 2.0,
     (3.0, -2.0, 5.0), None, 2.0, 0.0),
]

CFG = """ProjectionFile = {d}/ts.mrc
OutVolumeFile = {d}/vol.em
MarkerFile = {d}/m.em
Lambda = 0.5
Iterations = 1
RecDimesions = {nx} {ny} {nz}
UseFixPsiAngle = {fix}
PsiAngle = {psi}
PhiAngle = {phi}
AddTiltAngle = {addt}
AddTiltXAngle = {addx}
VolumeShift = {vsx} {vsy} {vsz}
ReferenceMarker = 0
OverSampling = 1
VoxelSize = {vs}
DimLength = 4 4
CutLength = 2 2
SkipFilter = false
fourFilterLP = 28
fourFilterLPS = 4
fourFilterHP = 0
fourFilterHPS = 0
SIRTCount = 1
CtfMode = false
BadPixelValue = 10
CorrectBadPixels = true
ProjectionNormalization = std
WBP = false
WBPFilter = Ramp
CudaDeviceID = 0
SizeSubVol = 0
VoxelSizeSubVol = 1
MotiveList = none
ProjectionScaleFactor = 1
CtfFile = none
"""


def case_inputs(name, n, W, H, dims, nsub, tc, vs, vshift, mag, shift, psi, seed):
    rng = np.random.default_rng(seed)
    items = np.zeros((1, n, 10), np.float32)
    items[0, :, 0] = np.linspace(-60.0, 60.0, n).astype(np.float32)
    items[0, :, 1:3] = 10.0  # the reference marker is clicked on every projection
    items[0, :, 4] = rng.uniform(-shift, shift, n)
    items[0, :, 5] = rng.uniform(-shift, shift, n)
    items[0, :, 8] = 1.0 if mag is None else mag
    items[0, :, 9] = rng.uniform(-psi, psi, n) if psi else 0.0
    return dict(name=name, W=W, H=H, dims=list(dims), subvols=nsub, pixel_size_nm=0.5, voxel_size=vs,
                volume_shift=list(vshift), add_tilt_angle=float(tc.get("AddTiltAngle", 0.0)),
                add_tilt_x_angle=float(tc.get("AddTiltXAngle", 0.0)),
                use_fix_psi_angle=tc.get("UseFixPsiAngle", "false") == "true", psi_angle=float(tc.get("PsiAngle", 0.0)),
                phi_angle=float(tc.get("PhiAngle", 0.0)), items=items[0].tolist())


def run_reference(exe: str, case: dict) -> dict:
    """The harness's output for one case (written to a scratch directory)."""
    from artiatomi_b200 import fileio as F

    with tempfile.TemporaryDirectory() as d:
        items = np.asarray(case["items"], np.float32)[None]
        F.write_markers(f"{d}/m.em", items)
        nx, ny, nz = case["dims"]
        vsx, vsy, vsz = case["volume_shift"]
        Path(f"{d}/c.cfg").write_text(CFG.format(d=d, nx=nx, ny=ny, nz=nz, fix="true" if case["use_fix_psi_angle"]
                                                 else "false", psi=case["psi_angle"], phi=case["phi_angle"],
                                                 addt=case["add_tilt_angle"], addx=case["add_tilt_x_angle"],
                                                 vsx=vsx, vsy=vsy, vsz=vsz, vs=case["voxel_size"]))
        r = subprocess.run([exe, f"{d}/c.cfg", f"{d}/m.em", str(case["W"]), str(case["H"]),
                            str(case["pixel_size_nm"]), str(nx), str(ny), str(nz), str(case["subvols"])],
                           capture_output=True, text=True, check=True)
    vols, projs, hits = [], [], []
    for line in r.stdout.split("\n"):
        t = line.split()
        if not t:
            continue
        if "vol" in t:  # (the reference's Config may print before it on the same line)
            t = t[t.index("vol"):]
            vols.append({"min": t[3:6], "max": t[7:10], "rcp": t[11:14], "dim": t[15:18], "zshift": t[19]})
        elif t[0] == "proj":
            projs.append({"det": t[3:6], "u": t[7:10], "v": t[11:14], "n": t[15:18], "mat": t[19:35]})
        elif t[0] == "hit":
            hits.append([int(x) for x in t[1:]])
    return {"vols": vols, "projs": projs, "hits": hits}


def main():
    from oracle.ref_geometry import build as ref_geometry_build

    exe = ref_geometry_build.build(verbose=True)
    if exe is None:
        sys.exit("the reference tree is needed to build oracle/_ref/ref_geometry")
    cases = []
    for k, c in enumerate(CASES):
        inp = case_inputs(*c, seed=100 + k)
        inp["reference"] = run_reference(str(exe), inp)
        cases.append(inp)
    OUT.write_text(json.dumps({"cases": cases}, indent=0))
    print(f"wrote {OUT} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
