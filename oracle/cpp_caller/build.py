"""Build oracle/_ref/sart_caller: the C++ program of
oracle/cpp_caller/sart_caller.cpp (EmSart's SART run with the reference's
own Config / MarkerFile / Projection / Volume, compiled unmodified from the
reference tree, and libesb for the device work), linked against
artiatomi_b200/libesb.so and the CUDA runtime.

TEST INFRASTRUCTURE: tests/test_cpp_caller.py runs it. Needs the reference
tree (oracle/refroot.py) and a built libesb.so; without the
reference tree the build is skipped.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
OUT = HERE.parent / "_ref" / "sart_caller"
LIBESB = REPO / "artiatomi_b200" / "libesb.so"

if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))
from oracle.ref_geometry.build import INCLUDES, SOURCES, SRC, available  # noqa: E402  (the reference sources)


def build(force: bool = False, verbose: bool = False) -> Path | None:
    if not available() or not LIBESB.exists():
        if verbose:
            print("reference sources or libesb.so missing: skipping oracle/_ref/sart_caller", flush=True)
        return OUT if OUT.exists() else None
    OUT.parent.mkdir(exist_ok=True)
    src = HERE / "sart_caller.cpp"
    deps = [src, LIBESB, REPO / "include" / "esb.h"]
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    inc = []
    for d in INCLUDES:
        inc += ["-I", str(SRC / d)]
    cmd = ["g++", "-O1", "-std=c++14", "-fpermissive", "-w", *inc, "-I", f"{cuda}/include", "-I", str(REPO / "include"),
           str(src), *[str(SRC / s) for s in SOURCES],
           "-L", str(LIBESB.parent), "-lesb", "-L", f"{cuda}/lib64", "-lcudart",
           "-Wl,-rpath,$ORIGIN/../../artiatomi_b200", f"-Wl,-rpath,{cuda}/lib64", "-o", str(OUT)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
