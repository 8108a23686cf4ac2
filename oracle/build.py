"""Build the CPU oracle (test infrastructure) into oracle/build/liboracle.so.

The oracle is compiled with -ffp-contract=off so that float expressions are
evaluated one IEEE operation at a time, in the reference's order.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "build" / "liboracle.so"
SRC = HERE / "esb_oracle.cpp"


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT.parent.mkdir(exist_ok=True)
    if force or not OUT.exists() or OUT.stat().st_mtime < SRC.stat().st_mtime:
        cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
               "-pthread", str(SRC), "-o", str(OUT)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
