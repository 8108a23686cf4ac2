"""Build oracle/_ref/ref_fileio: the reference's own EM / MRC / marker / CTF
file classes (src/EmTools/FileIO, FilterGraph/Matrix, FilterGraph/PointF,
Minimization/levmar: compiled unmodified from the reference tree, not
copied) linked with the harness oracle/ref_fileio/ref_fileio.cpp.

TEST INFRASTRUCTURE: used by tests/test_fileio.py and
tests/golden/make_fileio_golden.py to pin artiatomi_b200.fileio to the
reference's readers and writers. Needs the reference tree (oracle/refroot.py); without it the build is skipped.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref" / "ref_fileio"
if str(HERE.parent.parent) not in sys.path:
    sys.path.insert(0, str(HERE.parent.parent))
from oracle.refroot import REF_ROOT  # noqa: E402
TOOLS = REF_ROOT / "src" / "EmTools"
SOURCES = ["FileIO/EmFile.cpp", "FileIO/MRCFile.cpp", "FileIO/File.cpp", "FileIO/FileReader.cpp",
           "FileIO/FileWriter.cpp", "FileIO/FileIOException.cpp", "FileIO/ImageBase.cpp", "FileIO/MarkerFile.cpp",
           "FileIO/CtfFile.cpp", "FileIO/ImodFiducialFile.cpp", "FileIO/MotiveList.cpp", "FileIO/ShiftFile.cpp", "FilterGraph/Matrix.cpp", "FilterGraph/PointF.cpp",
           "Minimization/levmar.cpp"]


def available() -> bool:
    return (TOOLS / "FileIO" / "EmFile.cpp").is_file()


def build(force: bool = False, verbose: bool = False) -> Path | None:
    if not available():
        if verbose:
            print(f"reference file classes not found under {TOOLS}: skipping oracle/_ref/ref_fileio", flush=True)
        return OUT if OUT.exists() else None
    OUT.parent.mkdir(exist_ok=True)
    harness = HERE / "ref_fileio.cpp"
    if not force and OUT.exists() and OUT.stat().st_mtime >= harness.stat().st_mtime:
        return OUT
    inc = []
    for d in ("FileIO", "Basics", "", "FilterGraph", "Minimization"):
        inc += ["-I", str(TOOLS / d) if d else str(TOOLS)]
    cuda_inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    cmd = ["g++", "-O1", "-std=c++14", "-fpermissive", "-w", *inc, "-I", cuda_inc, str(harness),
           *[str(TOOLS / s) for s in SOURCES], "-o", str(OUT)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
