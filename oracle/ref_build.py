"""Build oracle/_ref/libref_kernels.so: the reference's kernel sources,
host-compiled; and oracle/_ref/libref_ctf_gpu.so: the reference's `ctf`
kernel (the one kernel of its EmSART path that CUDA 12 still compiles) built
for sm_100a with a launcher (oracle/ref_gpu/ref_ctf_gpu.cu).

Recipe (TEST INFRASTRUCTURE): every wrapper in oracle/ref_shim/ includes one
of the reference's .cu files from its place in the reference tree
(src/EmSART/cuda_kernels/, read-only, not copied). g++ compiles it for the
host against the CUDA-execution shim in oracle/ref_shim/ (esb_ref_shim.h and
the stand-in headers in oracle/ref_shim/include/). The shared library goes to
oracle/_ref/, which git ignores. It is used only to pin the oracle against
the reference's own kernel code. Needs the reference tree (oracle/refroot.py); without it the build is skipped.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SHIM = HERE / "ref_shim"
OUT = HERE / "_ref" / "libref_kernels.so"
OUT_CTF_GPU = HERE / "_ref" / "libref_ctf_gpu.so"
if str(HERE.parent) not in sys.path:
    sys.path.insert(0, str(HERE.parent))
from oracle.refroot import REF_ROOT  # noqa: E402
KERNELS = REF_ROOT / "src" / "EmSART" / "cuda_kernels"
UNITS = ["ref_runtime.cpp", "ref_fp.cpp", "ref_slicer.cpp", "ref_compare.cpp", "ref_bp.cpp", "ref_square.cpp",
         "ref_ctf.cpp", "ref_wbp.cpp"]


def available() -> bool:
    return KERNELS.is_dir()


def build(force: bool = False, verbose: bool = False) -> Path | None:
    if not available():
        if verbose:
            print(f"reference kernels not found at {KERNELS}: skipping oracle/_ref", flush=True)
        return OUT if OUT.exists() else None
    OUT.parent.mkdir(exist_ok=True)
    srcs = [SHIM / u for u in UNITS]
    deps = srcs + list(SHIM.glob("*.h")) + list((SHIM / "include").glob("*.h"))
    if not force and OUT.exists() and all(OUT.stat().st_mtime >= d.stat().st_mtime for d in deps):
        build_ctf_gpu(force, verbose)
        return OUT
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared", "-pthread",
           "-w", "-D__CUDACC__", "-I", str(SHIM / "include"), "-I", str(SHIM), "-I", str(KERNELS),
           *map(str, srcs), "-o", str(OUT)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    build_ctf_gpu(force, verbose)
    return OUT


def build_ctf_gpu(force: bool = False, verbose: bool = False) -> Path | None:
    """The reference's ctf.cu for sm_100a, through oracle/ref_gpu/ref_ctf_gpu.cu."""
    if not available():
        return OUT_CTF_GPU if OUT_CTF_GPU.exists() else None
    src = HERE / "ref_gpu" / "ref_ctf_gpu.cu"
    deps = [src, KERNELS / "ctf.cu"]
    if not force and OUT_CTF_GPU.exists() and all(OUT_CTF_GPU.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return OUT_CTF_GPU
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-w", "-I", str(KERNELS), str(src), "-o", str(OUT_CTF_GPU)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return OUT_CTF_GPU


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
