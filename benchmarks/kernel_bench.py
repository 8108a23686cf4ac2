"""Time single kernels of the hot path with CUDA events (for tuning and ncu).

  python -m benchmarks.kernel_bench --kernel fp|slicer|bp|bp_linear
      [--dims X Y Z] [--proj W H] [--tilt DEG] [--os N] [--voxel f32|f16|bf16]
      [--reps R] [--warmup N] [--fast]

Prints one JSON line per kernel: mean ms per launch and algorithmic GB/s
(forward projection: volume read once + projection/ray-length writes;
back-projection: volume read + write + projection read). The volume is
random; the geometry is one tilt of a single-axis series. --fast times the
closed-form projector / per-voxel-shadow back-projector instead of the
faithful kernels.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main(argv=None):
    import torch

    from artiatomi_b200 import emsart as E

    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="fp", choices=["fp", "slicer", "bp", "bp_linear", "travlen"])
    ap.add_argument("--dims", type=int, nargs=3, default=[1024, 1024, 256])
    ap.add_argument("--proj", type=int, nargs=2, default=None)
    ap.add_argument("--tilt", type=float, default=30.0)
    ap.add_argument("--os", type=int, default=2)
    ap.add_argument("--voxel", default="f32", choices=["f32", "f16", "bf16"])
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--slab", type=float, default=111.1, help="slab thickness in voxels (slicer, bp slabs)")
    ap.add_argument("--fast", action="store_true")
    a = ap.parse_args(argv)
    nx, ny, nz = a.dims
    W, H = a.proj if a.proj else (ny, nx)
    dt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[a.voxel]
    s = {"f32": 4, "f16": 2, "bf16": 2}[a.voxel]
    g = torch.Generator(device="cuda").manual_seed(0)
    vol = torch.rand((nz, ny, nx), generator=g, device="cuda").to(dt)
    pg = E.projection_geometry(E.Markers(np.array([a.tilt], np.float32)), W, H)
    vg = E.volume_geometry((nx, ny, nz))
    fc = E.set_constant_values(pg[0], vg)
    bc = E.set_constant_values(pg[0], vg, for_bp=True)
    proj = torch.zeros((H, W), device="cuda")
    dist = torch.zeros((H, W), device="cuda")
    img = torch.rand((H, W), generator=g, device="cuda")
    t0, t1 = E.defocus_distances(pg[0], vg, W, H)
    mid = 0.5 * (t0 + t1)

    def launch():
        if a.kernel == "fp":
            E.forward_project(fc, vol, proj, dist, fast=a.fast)
        elif a.kernel == "slicer":
            E.forward_project_slab(fc, vol, proj, mid - 0.5 * a.slab, mid + 0.5 * a.slab, fast=a.fast)
        elif a.kernel == "travlen":
            E.traversal_length(fc, dist)
        elif a.kernel == "bp":
            E.back_project(bc, vol, img, 1e-3, a.os, fast=a.fast)
        else:
            E.back_project(bc, vol, img, 1e-3, a.os, mid - 0.5 * a.slab, mid + 0.5 * a.slab, True, fast=a.fast)

    for _ in range(a.warmup):
        launch()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.reps)]
    for e0, e1 in ev:
        e0.record()
        launch()
        e1.record()
    torch.cuda.synchronize()
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    V, P = nx * ny * nz, W * H
    if a.kernel in ("fp",):
        nbytes = V * s + 3 * P * 4
    elif a.kernel == "slicer":
        frac = min(1.0, a.slab / max(t1 - t0, 1e-6))
        nbytes = V * s * frac + 2 * P * 4
    elif a.kernel == "travlen":
        nbytes = 2 * P * 4
    elif a.kernel == "bp":
        nbytes = 2 * V * s + P * 4
    else:
        frac = min(1.0, a.slab / max(t1 - t0, 1e-6))
        nbytes = 2 * V * s * frac + P * 4
    mean = float(np.mean(ms))
    print(json.dumps({"kernel": a.kernel, "fast": a.fast, "dims": a.dims, "proj": [W, H], "tilt": a.tilt, "os": a.os,
                      "voxel": a.voxel, "ms_mean": mean, "ms_min": float(np.min(ms)),
                      "algorithmic_GBps": nbytes / (mean * 1e-3) / 1e9}), flush=True)


if __name__ == "__main__":
    main()
