"""Shared helpers of the test suite: seeded small cases and comparisons."""
from __future__ import annotations

import numpy as np


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def small_case(dims=(64, 64, 32), n_proj=7, W=64, H=64, seed=3, n_ell=25, shift=0.0, psi=0.0, mag=None,
               t_min=-60.0, t_max=60.0):
    """Phantom + markers + geometries (oracle and product) of a small case."""
    import artiatomi_b200 as E
    from artiatomi_b200 import phantom as PH
    from oracle import geometry as G

    vol = PH.phantom_numpy(dims, n_ell, seed=seed)
    tilt = PH.tilt_series(n_proj, t_min, t_max)
    xs, ys, ps = PH.alignment(n_proj, seed=seed, shift=shift, psi_jitter=psi)
    m = None if mag is None else np.full(n_proj, mag, np.float32)
    pg = E.projection_geometry(E.Markers(tilt, xs, ys, m, ps), W, H)
    og = G.projection_geometry(tilt, xs, ys, m, ps, W, H)
    return dict(vol=vol, tilt=tilt, xs=xs, ys=ys, psi=ps, mag=m, pg=pg, og=og, dims=dims, W=W, H=H,
                vg=E.volume_geometry(dims), vo=G.volume_geometry(dims))


def cuda(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch

    torch.cuda.synchronize()
    return t.detach().float().cpu().numpy()
