#!/usr/bin/env python
"""Benchmark of the EmSART SART + 3D-CTF iteration on B200.

One step = one SART iteration of the 1024x1024x256 / 61 x 1024^2 / CTF /
oversampling 2 / 4-projection ordered subsets workload: for every projection
forward projection over the 30 nm defocus slabs (slicer + CTF chain),
compare, and per ordered subset the CTF-slab back-projections. The metric is
voxel-updates per second (one voxel back-projected from one projection,
forward projection and compare of that projection included).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl esb|reference]

Multi-GPU (torchrun): every rank reconstructs its own tomogram (independent
tilt series), so the per-GPU work is fixed and scaling is weak; no collective
runs on the data path. The timing is taken with CUDA events on the
reconstructor's stream between barriers, maximum over ranks.

--impl reference times the CPU oracle (the multithreaded C++ restatement of
the reference's kernels; the reference's own GPU code cannot be compiled with
CUDA 12.9) on a bounded sample of the same workload and prints the same line.
That arm never loads this library: it reads the workload parameters and the
phantom generator by path.

The GPU arm replays the SART subset loop from a captured CUDA graph
(esb_reconstructor_enable_graphs). After the timed steps it reports the
parity of the same kernels at the C2 geometry cropped to 256x256x64 (rel-L2
of the reconstructed volume against the FP32 and FP64 CPU oracles), with the
CPU baseline.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def _load_by_path(name: str, rel: str):
    """A module of the package loaded from its file, without the package's
    __init__ (which loads the CUDA library)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(name, ROOT / rel)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def workload_config(name: str, params: dict, ws: int = 1) -> dict:
    """The `config` object of both arms' JSON lines."""
    vox = params["dims"][0] * params["dims"][1] * params["dims"][2]
    return {"workload": name, "volume": list(params["dims"]), "projections": params["n_proj"],
            "projection_size": [params["W"], params["H"]], "oversampling": params["os"],
            "sirt_count": params["sirt"], "ctf": params["ctf"], "ctf_slab_nm": 30.0 if params["ctf"] else None,
            "voxel_storage": "f32", "l2": f"inputs larger than L2 (volume {vox * 4 / 2**20:.0f} MiB)",
            "parallelism": f"replicas x{ws}"}


METRIC = "SART voxel-updates/s (SART+3D-CTF iteration, 1024x1024x256, 61x1024^2)"
UNIT = "voxel-updates/s"


# DRAM bytes per launch measured by ncu (dram__bytes_read.sum,
# dram__bytes_write.sum) on the 1024x1024x64 volume / 1024^2 detector case,
# per unit of the roofline: forward projection = k_slicer_axis (volume read,
# slab images written) + k_travlen (ray lengths written), back-projection =
# k_bp_axis (volume read and written, pre-sampled slab images read). The
# volume part scales with the voxels, the image part with the pixels.
DRAM_V, DRAM_P = 1024 * 1024 * 64, 1024 * 1024
DRAM_FP_READ, DRAM_FP_IMG = 268.44e6, 8.47e6 + 4.20e6
DRAM_BP_READ, DRAM_BP_WRITE, DRAM_BP_IMG = 268.44e6, 211.57e6, 292.94e6 - 268.44e6


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, name in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def _dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def cpu_sample(workload_params, n_proj_sample: int = 4, y_extent: int = 8):
    """Time the CPU oracle on a bounded sample of the workload.

    The sample keeps the full workload's geometry, tilt angles, CTF slabs and
    1024^2 FFTs but cuts the volume to `y_extent` voxels along the tilt axis
    (y; the detector's u axis), where the rays of a single-axis tilt series
    stay in constant-y planes, so the per-voxel and per-pixel work of the
    projector and back-projector equals the full problem's. The voxel work is
    extrapolated by the volume ratio; the CTF chain (crop, pad, 1024^2 FFT
    pair, filter) is counted at full size. Returns (voxel-updates/s, detail).
    """
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    PH = _load_by_path("esb_phantom", "artiatomi_b200/phantom.py")

    p = workload_params
    nx, ny, nz = p["dims"]
    W, H = p["W"], p["H"]
    n = p["n_proj"]
    tilt = PH.tilt_series(n, -60.0, 60.0)
    xs, ys, psi = PH.alignment(n, seed=0, shift=p.get("shift", 0.0), psi_jitter=0.0)
    sub_dims = (nx, y_extent, nz)
    Ws = y_extent  # detector u follows volume y
    og = G.projection_geometry(tilt, xs, ys, None, psi, Ws, H)
    vo = G.volume_geometry(sub_dims)
    vol = PH.phantom_numpy(sub_dims, max(4, p["n_ell"] * y_extent // ny), seed=1)
    rng = np.random.default_rng(3)
    defocus = None
    cfgd = dict(lambda_=p["lam"], oversampling=p["os"], cut_length=(10.0, 10.0), dim_length=(20.0, 20.0))
    if p["ctf"]:
        dmid = rng.uniform(2500.0, 3500.0, n)
        defocus = np.stack([dmid - 50.0, dmid + 50.0, rng.uniform(0.0, 180.0, n)], 1).astype(np.float32).ravel()
        cfgd.update(ctf_mode=True, pixel_size_nm=0.27, ctf_slice_thickness_nm=30.0)
    orc = OracleReconstructor(cfgd, Ws, H, og, tilt, defocus, precision=0)
    orc.N = max(W, H)  # full-size FFTs as in the full workload
    orc.bx, orc.by = (orc.N - Ws) // 2, (orc.N - H) // 2
    projs = rng.normal(size=(n, H, Ws)).astype(np.float32)
    idx = [int(i) for i in np.linspace(0, n - 1, n_proj_sample).round()]
    t_fp = t_bp = t_ctf = 0.0
    # time the kernels and the CTF chain separately by wrapping the oracle's steps
    orig_chain = orc._ctf_chain
    ctf_time = [0.0]

    def timed_chain(*a, **k):
        t0 = time.perf_counter()
        r = orig_chain(*a, **k)
        ctf_time[0] += time.perf_counter() - t0
        return r

    orc._ctf_chain = timed_chain
    t0 = time.perf_counter()
    for i in idx:
        orc.reset()
        orc.forward_projection(vo, vol, 0, i, False)
        orc.compare(vo, projs[i], i)
    t_fp = time.perf_counter() - t0
    t0 = time.perf_counter()
    for i in idx:
        orc.back_projection(vo, vol, 0, i, float(p["sirt"]), img=projs[i].copy())
    t_bp = time.perf_counter() - t0
    t_ctf = ctf_time[0]
    scale = ny / y_extent
    per_proj = ((t_fp + t_bp - t_ctf) * scale + t_ctf) / len(idx)
    vu = nx * ny * nz / per_proj
    from oracle.lib import NTHREADS

    return vu, dict(per_projection_s=per_proj, sample_s=t_fp + t_bp,
                    sample=f"{len(idx)} projections of the workload on a {nx}x{y_extent}x{nz} tilt-axis slice "
                    f"(volume {nx}x{ny}x{nz}), timed; value extrapolated to the full volume: voxel work x{scale:.0f}, "
                    f"CTF chains ({max(W, H)}^2 FFTs) counted once", cores=NTHREADS)


def run_reference(args):
    ws, rank, _ = _dist_setup()
    if rank != 0:
        return 0
    params = _load_by_path("esb_configs", "artiatomi_b200/configs.py").CONFIGS[args.workload]
    for _ in range(args.warmup):
        cpu_sample(params, n_proj_sample=1)
    vals, secs = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        v, det = cpu_sample(params, n_proj_sample=2)
        secs.append(time.perf_counter() - t0)
        vals.append(v)
    value = float(np.median(vals))
    full_ms = params["dims"][0] * params["dims"][1] * params["dims"][2] * params["n_proj"] / value * 1e3
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(secs)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args.workload, params, ws),
            "extrapolated": True,
            "extrapolation": "a step is the bounded sample below (ms_per_step: its measured time); value is the "
                             "sample's throughput extrapolated to the full workload (full_step_ms_extrapolated)",
            "full_step_ms_extrapolated": full_ms,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": det["cores"], "kind": "port",
                             "sample": det["sample"], "sample_s": float(np.mean(secs))},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _mean_slabs(E, wl, params) -> float:
    """CTF slabs per projection of the workload, averaged over its
    projections: the library's slab recurrence (ray += thickness from the
    volume's entry depth while ray < its exit depth, in float)."""
    step = np.float32(wl.cfg.ctf_slice_thickness_nm) / np.float32(wl.cfg.pixel_size_nm)
    counts = []
    for i in wl.index_list:
        t_in, t_out = E.defocus_distances(wl.pg[int(i)], wl.vg, params["W"], params["H"])
        ray, k = np.float32(t_in), 0
        while ray < np.float32(t_out):
            ray = np.float32(ray + step)
            k += 1
        counts.append(k)
    return float(np.mean(counts))


def config_parity(name: str = "c2_crop") -> dict:
    """The SART volume of workload `name` (this library's FAST kernels, and
    its FAITHFUL ones) against the FP32 and FP64 CPU oracles, on the same
    measured projections."""
    from oracle.parity import rel_l2, run_config

    t0 = time.perf_counter()
    run = run_config(name, variants=("fast", "faithful"), precisions=(0, 1))
    p = run.params
    return {"workload": name, "volume": list(p["dims"]), "projections": p["n_proj"], "iterations": p["iterations"],
            "oversampling": p["os"], "sirt_count": p["sirt"], "ctf": p["ctf"],
            "rel_l2_vs_fp32_oracle": rel_l2(run.volumes["fast"], run.oracle[0]),
            "rel_l2_vs_fp64_oracle": rel_l2(run.volumes["fast"], run.oracle[1]),
            "fp32_oracle_vs_fp64_oracle": rel_l2(run.oracle[0], run.oracle[1]),
            "faithful_rel_l2_vs_fp32_oracle": rel_l2(run.volumes["faithful"], run.oracle[0]),
            "seconds": round(time.perf_counter() - t0, 1)}


def run_esb(args):
    import torch
    import torch.distributed as dist

    ws, rank, local = _dist_setup()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local if ws > 1 else 0)
    torch.cuda.set_device(dev)

    import artiatomi_b200 as E
    from artiatomi_b200 import workloads as WL

    params = dict(WL.CONFIGS[args.workload])
    wl = WL.build(args.workload, params, seed=rank)
    stream = torch.cuda.Stream()
    import dataclasses

    cfg = dataclasses.replace(wl.cfg, variant=E.VARIANT_FAST if args.variant == "fast" else E.VARIANT_FAITHFUL)
    rec = E.Reconstructor(cfg, wl.pg, wl.tilt, wl.defocus, stream=stream)
    graphs = not args.no_graphs
    rec.enable_graphs(graphs)  # the subset loop replays from a captured CUDA graph
    vol = torch.zeros(params["dims"][::-1], dtype=torch.float32, device=dev)
    sirt = params["sirt"]

    def step(projs):
        rec.sart(wl.vg, vol, projs, wl.index_list, iterations=1, sirt_count=sirt, volume_is_empty=False)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(wl.projections)
    torch.cuda.synchronize()

    # ---- device-resident timing
    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    launches0 = E.kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev.index) as clk:
        torch.cuda.nvtx.range_push("esb_timed")
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                step(wl.projections)
            e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms_total = e0.elapsed_time(e1)
    gpu_launches = E.kernel_launches() - launches0
    barrier()

    # ---- per-phase device time and launch-group counts: one more step, run
    # eagerly with an event pair around every launch group (kept out of the
    # timed steps, where the events would add host work per launch)
    rec.enable_timing(True)
    rec.timing()
    with torch.cuda.stream(stream):
        step(wl.projections)
    torch.cuda.synchronize()
    phases = rec.timing()
    rec.enable_timing(False)
    barrier()
    t = torch.tensor([ms_total], device=dev)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_step = float(t.item()) / args.steps
    vu_step = wl.voxel_updates_per_iteration
    value = vu_step * ws / (ms_step * 1e-3)

    # ---- end to end: host projections in, host volume out, every step
    host_in = torch.empty(wl.projections.shape, dtype=torch.float32, pin_memory=True)
    host_in.copy_(wl.projections.cpu())
    host_out = torch.empty(vol.shape, dtype=torch.float32, pin_memory=True)
    dev_in = torch.empty_like(wl.projections)
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e2.record(stream)
        for _ in range(args.steps):
            dev_in.copy_(host_in, non_blocking=True)
            step(dev_in)
            host_out.copy_(vol, non_blocking=True)
        e3.record(stream)
    torch.cuda.synchronize()
    t2 = torch.tensor([e2.elapsed_time(e3)], device=dev)
    if ws > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_ms = float(t2.item()) / args.steps
    e2e_value = vu_step * ws / (e2e_ms * 1e-3)

    # ---- roofline of the dominant kernel (per projection of one step)
    hbm, hbm_kind = _peaks()
    V = wl.voxels
    P = params["W"] * params["H"]
    nproj = len(wl.index_list)
    fp_ms, fp_n = phases["fp"]
    bp_ms, bp_n = phases["bp"]
    if bp_ms >= fp_ms:
        slabs = bp_n / nproj
        bytes_unit = 2 * V * 4 + slabs * P * 4
        traffic = (DRAM_BP_READ + DRAM_BP_WRITE) / DRAM_V * V + DRAM_BP_IMG / DRAM_P * P
        name, t_unit, launches = "back-projection (all slab launches of one projection)", bp_ms / nproj, bp_n
    else:
        slabs = _mean_slabs(E, wl, params) if params["ctf"] else 1.0
        # the volume read once; per CTF slab one image written; the ray
        # lengths written once
        bytes_unit = V * 4 + (slabs + 1) * P * 4
        traffic = DRAM_FP_READ / DRAM_V * V + DRAM_FP_IMG / DRAM_P * P
        name, t_unit, launches = "forward projection (slicer launches + traversal length of one projection)", \
            fp_ms / nproj, fp_n
    achieved = bytes_unit / (t_unit * 1e-3) / 1e9

    cpu = None
    parity = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        v, det = cpu_sample(params, n_proj_sample=1)
        cpu = {"value": v, "unit": UNIT, "cores": det["cores"], "kind": "port", "sample": det["sample"],
               "extrapolated": True}
        if args.workload.startswith("c2_"):
            parity = config_parity("c2_crop")

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded ellipsoid+bead phantom, "
                "projections from this library's projector + noise)",
                "config": workload_config(args.workload, params, ws),
                "kernels": args.variant, "graphs": graphs,
                "launch_shapes": E.autotune_report().strip().splitlines(),
                "e2e": {"value": e2e_value, "unit": UNIT,
                        "h2d_bytes_per_step": int(wl.projections.numel() * 4),
                        "d2h_bytes_per_step": int(vol.numel() * 4)},
                "gpu_launches": int(gpu_launches),
                "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": hbm,
                             "peak_kind": hbm_kind, "unit": "GB/s", "frac": achieved / hbm,
                             "traffic": traffic, "traffic_source": "ncu dram__bytes_read.sum + "
                             "dram__bytes_write.sum per launch on the 1024x1024x64 case, volume part scaled by "
                             "voxels, image part by pixels", "algorithmic_bytes_per_unit": bytes_unit, "ms_per_unit": t_unit,
                             "launches": launches},
                "phases_ms_per_step": {k: v[0] for k, v in phases.items()},
                "clocks": clk.summary(),
                "cpu_baseline": cpu,
                "parity": parity}
        print(json.dumps(line), flush=True)
    rec.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["esb", "reference"], default="esb")
    ap.add_argument("--workload", default="c2_sart_ctf")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline and the oracle parity of the C2 crop")
    ap.add_argument("--no-graphs", action="store_true", help="launch the subset loop eagerly")
    ap.add_argument("--variant", choices=["fast", "faithful"], default="fast",
                    help="fast: closed-form cell-sum projector and per-voxel-shadow back-projector; "
                         "faithful: the reference's per-sample arithmetic")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_esb(args)


if __name__ == "__main__":
    sys.exit(main())
