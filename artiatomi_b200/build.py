"""Build libesb.so (the sm_100a CUDA library behind include/esb.h) in-tree.

Usage: python artiatomi_b200/build.py [--force]

(Run it as a file: importing the package loads libesb.so, which is what this
script builds.)

The library is compiled with nvcc for sm_100a only and linked against cuFFT.
The projector/back-projector translation unit is compiled with --fmad=false
so that its float arithmetic follows the reference's expressions operation
by operation. The other units use the default contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "libesb.so"
BUILD = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3"]

# (source, extra flags)
UNITS = [
    ("esb_projector.cu", ["--fmad=false"]),
    ("esb_projector_fast.cu", []),
    ("esb_backprojector_fast.cu", []),
    ("esb_subvolume.cu", []),
    ("esb_adjoint.cu", []),
    ("esb_refine.cu", []),
    ("esb_cc.cu", ["--fmad=false"]),
    ("esb_image.cu", ["--fmad=false"]),
    ("esb_ctf.cu", []),
    ("esb_api.cu", []),
    ("esb_noalloc.cu", []),
    ("esb_geometry.cpp", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libesb")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    force_link = False
    headers = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [PKG.parent / "include" / "esb.h"]
    objs = []
    for src, extra in UNITS:
        s = CSRC / src
        if not s.exists():
            continue
        o = BUILD / (s.stem + ".o")
        objs.append(o)
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-I", str(PKG.parent / "include"), "-c", str(s), "-o", str(o)]
        if s.suffix == ".cpp":
            cmd = ["g++", "-O3", "-std=c++17", "-fPIC", "-I", str(PKG.parent / "include"), "-c", str(s), "-o", str(o)]
        stamp = o.with_suffix(".cmd")
        flags_changed = not stamp.exists() or stamp.read_text() != " ".join(cmd)
        if force or flags_changed or _stale(o, [s] + headers):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            stamp.write_text(" ".join(cmd))
            force_link = True
    if force or force_link or _stale(OUT, objs):
        # cudart is linked statically (nvcc's default); cuFFT from the toolkit,
        # found through the rpath so that another cuFFT in the process (torch's)
        # is not picked up by accident.
        cuda_lib = str(Path(nvcc()).resolve().parent.parent / "lib64")
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(OUT), *map(str, objs), "-cudart", "static", "-L", cuda_lib,
               "-lcufft", "-Xlinker", f"-rpath={cuda_lib}"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
