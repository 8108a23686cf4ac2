"""Parity of a whole benchmark configuration against the CPU oracle (TEST
INFRASTRUCTURE).

Runs one named workload (seeded phantom, geometry and measured projections,
built on the GPU) through the library's SART reconstruction and through the
oracle's restatement of the reference's SART loop (EmSart.cpp:579-675) on the
same measured projections, and returns the relative L2 distance of the
volumes. Used by the config-size parity tests and by the parity field of
bench.py; the product never imports it.
"""
from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import geometry as G
from .driver import OracleReconstructor


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


@dataclasses.dataclass
class ConfigRun:
    name: str
    params: dict
    projections: np.ndarray  # (n, H, W) measured projections, host copy
    index_list: np.ndarray
    volumes: dict            # variant -> reconstructed volume (host)
    oracle: dict             # precision (0 FP32, 1 FP64) -> oracle volume
    oracle_s: dict           # precision -> seconds of oracle work
    workload: object = None


def reconstruct_gpu(wl, variant, voxel_type="f32"):
    """SART of workload `wl` on the GPU with kernels `variant` ("fast" or
    "faithful"); returns the volume on the host as float32."""
    import torch

    import artiatomi_b200 as E

    p = wl.params
    cfg = dataclasses.replace(wl.cfg, variant=E.VARIANT_FAST if variant == "fast" else E.VARIANT_FAITHFUL)
    rec = E.Reconstructor(cfg, wl.pg, wl.tilt, wl.defocus)
    dt = {"f32": torch.float32, "f16": torch.float16, "bf16": torch.bfloat16}[voxel_type]
    vol = torch.zeros(tuple(p["dims"][::-1]), dtype=dt, device="cuda")
    rec.sart(wl.vg, vol, wl.projections, wl.index_list, iterations=p["iterations"], sirt_count=p["sirt"])
    torch.cuda.synchronize()
    out = vol.float().cpu().numpy()
    rec.close()
    return out


def reconstruct_oracle(wl, projections_host, precision):
    """The oracle's SART (precision 0: the reference's FP32 arithmetic, 1:
    FP64) on the same measured projections."""
    p = wl.params
    tilt, xs, ys, psi = wl.markers
    W, H = p["W"], p["H"]
    og = G.projection_geometry(tilt, xs, ys, None, psi, W, H)
    vo = G.volume_geometry(tuple(p["dims"]))
    orc = OracleReconstructor(wl.cfg_kw, W, H, og, tilt, wl.defocus, precision=precision)
    v = np.zeros(tuple(p["dims"][::-1]), np.float32)
    orc.sart(vo, v, 0, projections_host, wl.index_list, p["iterations"], p["sirt"])
    return v


def run_config(name, variants=("fast",), precisions=(0, 1), seed=0, params=None) -> ConfigRun:
    from artiatomi_b200 import workloads as WL

    p = dict(WL.CONFIGS[name]) if params is None else dict(params)
    wl = WL.build(name, p, seed=seed)
    projs = wl.projections.cpu().numpy()
    vols = {v: reconstruct_gpu(wl, v) for v in variants}
    orc, secs = {}, {}
    for prec in precisions:
        t0 = time.perf_counter()
        orc[prec] = reconstruct_oracle(wl, projs, prec)
        secs[prec] = time.perf_counter() - t0
    return ConfigRun(name, p, projs, np.asarray(wl.index_list), vols, orc, secs, wl)
