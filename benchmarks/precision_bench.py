"""Volume storage precision: FP32, FP16 and BF16 SART with FP32 arithmetic.

  python -m benchmarks.precision_bench [--workload c5_precision] [--iterations 5]
      [--no-graphs] [--crop-oracle]

Runs the full SART + 3-D CTF reconstruction of the workload (default: the
2048x2048x512 volume, 61 x 2048^2 projections, oversampling 2, 8 projections
per subset, 5 iterations) once per storage type, each with the subset loop
replayed from a captured CUDA graph (iterations 2..5), and prints one JSON
line: time per iteration and voxel-updates/s per storage type, the speed-up
of each over FP32 and the relative L2 difference of each volume from the
FP32 one. --crop-oracle adds the 256x256x64 counterpart (c5_crop) run on the
GPU in all three storage types and by the FP64 CPU oracle, with the relative
L2 error of each against FP64.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import time

import numpy as np

DTYPES = ("f32", "f16", "bf16")


def _run(wl, dtype, iterations, graphs):
    import torch

    from artiatomi_b200 import emsart as E

    td = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[dtype]
    cfg = dataclasses.replace(wl.cfg, variant=E.VARIANT_FAST)
    rec = E.Reconstructor(cfg, wl.pg, wl.tilt, wl.defocus)
    rec.enable_graphs(graphs)
    vol = torch.zeros(wl.params["dims"][::-1], dtype=td, device="cuda")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    rec.sart(wl.vg, vol, wl.projections, wl.index_list, iterations=iterations, sirt_count=wl.params["sirt"],
             volume_is_empty=True)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    rec.close()
    return vol, ms


def _rel(a, b):
    num = float(((a.float() - b.float()).double() ** 2).sum())
    den = float((b.double() ** 2).sum())
    return (num / den) ** 0.5


def main(argv=None):
    import torch

    from artiatomi_b200 import workloads as WL

    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="c5_precision")
    ap.add_argument("--iterations", type=int, default=None)
    ap.add_argument("--no-graphs", action="store_true")
    ap.add_argument("--crop-oracle", action="store_true")
    a = ap.parse_args(argv)
    t0 = time.time()
    wl = WL.build(a.workload)
    setup_s = time.time() - t0
    it = a.iterations or wl.params["iterations"]
    vols, ms = {}, {}
    for dt in DTYPES:
        vols[dt], ms[dt] = _run(wl, dt, it, not a.no_graphs)
    vu = wl.voxels * len(wl.index_list)
    line = {"workload": a.workload, "dims": list(wl.params["dims"]), "projections": wl.params["n_proj"],
            "projection_size": [wl.params["W"], wl.params["H"]], "iterations": it, "sirt_count": wl.params["sirt"],
            "graphs": not a.no_graphs, "setup_s": round(setup_s, 1),
            "ms_per_iteration": {d: ms[d] / it for d in DTYPES},
            "voxel_updates_per_s": {d: vu * it / (ms[d] * 1e-3) for d in DTYPES},
            "speedup_vs_f32": {d: ms["f32"] / ms[d] for d in DTYPES},
            "rel_l2_vs_f32": {d: _rel(vols[d], vols["f32"]) for d in ("f16", "bf16")}}
    del vols
    torch.cuda.empty_cache()
    if a.crop_oracle:
        line["crop"] = crop_vs_oracle(it)
    print(json.dumps(line), flush=True)


def crop_vs_oracle(iterations):
    """c5_crop on the GPU (three storage types) against the FP64 oracle."""
    import torch

    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    from artiatomi_b200 import workloads as WL

    wl = WL.build("c5_crop")
    tilt, xs, ys, psi = wl.markers
    W, H = wl.params["W"], wl.params["H"]
    og = G.projection_geometry(tilt, xs, ys, None, psi, W, H)
    vo = G.volume_geometry(wl.params["dims"])
    projs = wl.projections.cpu().numpy()
    t0 = time.time()
    orc = OracleReconstructor(wl.cfg_kw, W, H, og, tilt, wl.defocus, precision=1)
    ref = np.zeros(wl.params["dims"][::-1], np.float32)
    orc.sart(vo, ref, 0, projs, wl.index_list, iterations, wl.params["sirt"])
    oracle_s = time.time() - t0
    ref_t = torch.from_numpy(ref).cuda()
    out = {"dims": list(wl.params["dims"]), "iterations": iterations, "oracle_s": round(oracle_s, 1)}
    for dt in DTYPES:
        v, _ = _run(wl, dt, iterations, True)
        out[f"rel_l2_{dt}_vs_fp64"] = _rel(v, ref_t)
    return out


if __name__ == "__main__":
    main()
