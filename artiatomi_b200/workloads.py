"""Synthetic workloads of the benchmark configurations, built on the GPU.

Each workload holds the geometry, the prepared projections and the
reconstruction parameters of one configuration. Phantoms are seeded ellipsoid
(+ bead) volumes. The measured projections are forward projections of the
phantom through this library's own projector (CTF slab model included when
the configuration uses CTF) plus Gaussian noise at the stated SNR.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import emsart as E
from . import phantom as PH
from .configs import CONFIGS  # noqa: F401  (the parameters of each workload)


@dataclass
class Workload:
    name: str
    params: dict
    cfg: E.ReconConfig
    pg: object
    tilt: np.ndarray
    defocus: np.ndarray | None
    vg: object
    index_list: np.ndarray
    projections: object  # torch (n, H, W) float32 on the device
    phantom: object      # torch (z, y, x) float32 on the device
    cfg_kw: dict | None = None   # ReconConfig keyword arguments
    markers: tuple | None = None  # (tilt, x shift, y shift, psi) per projection

    @property
    def voxels(self) -> int:
        d = self.params["dims"]
        return d[0] * d[1] * d[2]

    @property
    def voxel_updates_per_iteration(self) -> int:
        return self.voxels * len(self.index_list)


def scaled(name: str, scale_xy: int = 1, scale_z: int = 1, n_proj: int | None = None) -> dict:
    p = dict(CONFIGS[name])
    d = p["dims"]
    p["dims"] = (d[0] // scale_xy, d[1] // scale_xy, d[2] // scale_z)
    p["W"] //= scale_xy
    p["H"] //= scale_xy
    p["n_ell"] = max(1, p["n_ell"] // (scale_xy * scale_xy * scale_z))
    p["n_beads"] = max(0, p["n_beads"] // (scale_xy * scale_xy * scale_z))
    if n_proj:
        p["n_proj"] = n_proj
    return p


def build(name: str, params: dict | None = None, seed: int = 0, device: str = "cuda") -> Workload:
    import torch

    p = dict(CONFIGS[name]) if params is None else params
    nx, ny, nz = p["dims"]
    W, H, n = p["W"], p["H"], p["n_proj"]
    tilt = PH.tilt_series(n, -60.0, 60.0)
    xs, ys, psi = PH.alignment(n, seed=seed, shift=p.get("shift", 0.0), psi_jitter=p.get("psi", 0.0))
    pg = E.projection_geometry(E.Markers(tilt, xs, ys, None, psi), W, H)
    vg = E.volume_geometry((nx, ny, nz))
    rng = np.random.default_rng(seed + 7)
    defocus = None
    cfg_kw = dict(lambda_=p["lam"], oversampling=p["os"], cut_length=(10.0, 10.0), dim_length=(20.0, 20.0))
    if p["ctf"]:
        dmid = rng.uniform(2500.0, 3500.0, n)
        defocus = np.stack([dmid - 50.0, dmid + 50.0, rng.uniform(0.0, 180.0, n)], 1).astype(np.float32).ravel()
        cfg_kw.update(ctf_mode=True, pixel_size_nm=0.27, cs_mm=2.7, voltage_kv=300.0, amp_contrast=0.0,
                      ctf_slice_thickness_nm=30.0, ctf_beta_fac=(200.0, 0.0, 0.008, 0.0), wiener_noise_level=0.1)
    cfg = E.ReconConfig(W, H, n, **cfg_kw)
    phantom = PH.phantom_torch((nx, ny, nz), p["n_ell"], seed=seed, device=device, n_beads=p.get("n_beads", 0))
    # measured projections: this library's projector on the phantom + noise
    rec = E.Reconstructor(cfg, pg, tilt, defocus)
    proj_v, _, _ = rec.views()
    projs = torch.empty((n, H, W), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device).manual_seed(seed + 3)
    for i in range(n):
        rec.reset_projections()
        rec.forward_projection(vg, phantom, i, False)
        img = proj_v.clone()
        if "snr" in p:
            sig = img.std() / float(np.sqrt(p["snr"]))
        else:
            sig = img.std() * p.get("noise_sigma_rel", 0.0)
        img += torch.randn(img.shape, generator=gen, device=device) * sig
        projs[i] = img
    torch.cuda.synchronize()
    rec.close()
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, tilt)
    return Workload(name, p, cfg, pg, tilt, defocus, vg, il, projs, phantom, cfg_kw, (tilt, xs, ys, psi))
