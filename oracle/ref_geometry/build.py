"""Build oracle/_ref/ref_geometry: the reference's own host geometry
(src/EmSART/Projection.cpp, Volume.cpp, utils/Config.cpp and the file
classes it reads through: src/EmTools/FileIO, FilterGraph/Matrix, PointF,
Minimization/levmar; compiled unmodified from the reference tree, not copied)
linked with the harness oracle/ref_geometry/ref_geometry.cpp.

TEST INFRASTRUCTURE: used by tests/golden/make_geometry_golden.py and
tests/test_geometry_reference.py to pin the library's geometry to the
reference's bit for bit. Needs the reference tree (oracle/refroot.py); without it the build is skipped.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE.parent / "_ref" / "ref_geometry"
if str(HERE.parent.parent) not in sys.path:
    sys.path.insert(0, str(HERE.parent.parent))
from oracle.refroot import REF_ROOT  # noqa: E402
SRC = REF_ROOT / "src"
SOURCES = ["EmSART/Projection.cpp", "EmSART/Volume.cpp", "EmSART/utils/Config.cpp", "EmSART/utils/ConfigExceptions.cpp",
           "EmSART/utils/log.cpp", "EmTools/FileIO/MarkerFile.cpp", "EmTools/FileIO/ImodFiducialFile.cpp",
           "EmTools/FileIO/EmFile.cpp", "EmTools/FileIO/File.cpp", "EmTools/FileIO/FileReader.cpp",
           "EmTools/FileIO/FileWriter.cpp", "EmTools/FileIO/FileIOException.cpp", "EmTools/FileIO/ImageBase.cpp",
           "EmTools/FileIO/MotiveList.cpp", "EmTools/FilterGraph/Matrix.cpp", "EmTools/FilterGraph/PointF.cpp",
           "EmTools/Minimization/levmar.cpp"]
INCLUDES = ["EmSART", "EmSART/io", "EmSART/utils", "EmSART/cuda_kernels", "EmTools/FileIO", "EmTools/Basics", "EmTools",
            "EmTools/FilterGraph", "EmTools/Minimization", "EmTools/CudaHelpers"]


def available() -> bool:
    return (SRC / "EmSART" / "Projection.cpp").is_file()


def build(force: bool = False, verbose: bool = False) -> Path | None:
    if not available():
        if verbose:
            print(f"reference geometry sources not found under {SRC}: skipping oracle/_ref/ref_geometry", flush=True)
        return OUT if OUT.exists() else None
    OUT.parent.mkdir(exist_ok=True)
    harness = HERE / "ref_geometry.cpp"
    if not force and OUT.exists() and OUT.stat().st_mtime >= harness.stat().st_mtime:
        return OUT
    inc = []
    for d in INCLUDES:
        inc += ["-I", str(SRC / d)]
    cuda_inc = os.environ.get("CUDA_HOME", "/usr/local/cuda") + "/include"
    cmd = ["g++", "-O1", "-std=c++14", "-fpermissive", "-w", *inc, "-I", cuda_inc, str(harness),
           *[str(SRC / s) for s in SOURCES], "-o", str(OUT)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
