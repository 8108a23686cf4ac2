"""Throughput of EmSartRefine's shift measurement (method "cc").

  python -m benchmarks.refine_bench [--particles 16] [--dims 1024 1024 256]
      [--proj 1024] [--n-proj 61] [--size 64] [--max-shift 10] [--no-ctf]

One measurement is one particle in one projection, as EmSartRefine.cpp:
825-980 makes it for a group of one particle: the rotated reference's
projection over the particle's detector region (ForwardProjectionROI, the
reference's safeDist around the particle's hit point), the projection of the
reconstruction with the particle's cube zeroed over the same region, Compare
against the prepared projection, and GetDisplacement (two 1024^2 R2C, one
C2R, the normalisation, the maxShift mask and the arg-max). With CTF both
projections are CTF-filtered slab by slab over the whole detector, as
ForwardProjectionCTFROI does. The volume, the projections and the
references are random (the work does not depend on the values); the
particle centres are uniform in the volume away from its faces.

Prints one JSON line: measurements per second, ms per measurement (host wall
clock: every measurement ends with the arg-max read back to the host, as in
the reference) and the library's kernel launches per measurement.
"""
from __future__ import annotations

import argparse
import json
import time
import types

import numpy as np


def main(argv=None):
    import torch

    from artiatomi_b200 import emsart as E
    from artiatomi_b200.refine import _cc_shift, _particle_roi, _remove_radius, _remove_subvolume

    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=16)
    ap.add_argument("--dims", type=int, nargs=3, default=[1024, 1024, 256])
    ap.add_argument("--proj", type=int, default=1024)
    ap.add_argument("--n-proj", type=int, default=61)
    ap.add_argument("--size", type=int, default=64)
    ap.add_argument("--max-shift", type=int, default=10)
    ap.add_argument("--no-ctf", action="store_true")
    ap.add_argument("--multi-peak", action="store_true")
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    torch.manual_seed(a.seed)
    rng = np.random.default_rng(a.seed)
    dims, W, n, S = tuple(a.dims), a.proj, a.n_proj, a.size
    tilt = np.linspace(-60.0, 60.0, n).astype(np.float32)
    pg = E.projection_geometry(E.Markers(tilt), W, W)
    vg = E.volume_geometry(dims)
    ctf = not a.no_ctf
    cfgd = dict(ctf_mode=True, pixel_size_nm=0.27, ctf_slice_thickness_nm=30.0,
                ctf_beta_fac=(10.0, 0.0, 0.008, 0.0)) if ctf else {}
    defocus = None
    if ctf:
        dmid = rng.uniform(2500.0, 3500.0, n)
        defocus = np.stack([dmid - 50.0, dmid + 50.0, rng.uniform(0.0, 180.0, n)], 1).astype(np.float32).ravel()
    rec = E.Reconstructor(E.ReconConfig(W, W, n, variant=E.VARIANT_FAST, cut_length=(10.0, 10.0),
                                        dim_length=(20.0, 20.0), **cfgd), pg, tilt, defocus)
    vol = torch.rand(dims[::-1], device="cuda") - 0.5
    prepared = torch.randn((n, W, W), device="cuda")
    ref = torch.rand((S, S, S), device="cuda")
    rot = torch.empty_like(ref)
    R = types.SimpleNamespace(rec=rec, prepared=prepared)
    cfg = types.SimpleNamespace(VoxelSize=(1.0, 1.0, 1.0), VoxelSizeSubVol=1.0)
    safe = int(100 + S * 2 + a.max_shift * 2)
    bufs = (torch.zeros((W, W), device="cuda"), rec.views()[0])
    margin = S // 2 + 2
    pos = np.stack([rng.uniform(margin + 1, d - margin, a.particles) for d in dims], 1).astype(np.float32)
    ang = rng.uniform(0.0, 360.0, (a.particles, 3)).astype(np.float32)
    vs = np.ones(3)

    def particle(p):
        m = np.zeros(20, np.float32)
        m[7:10], m[16:19] = pos[p], ang[p]
        E.rotate_volume(ref, rot, E.rotation_matrix(*ang[p]))
        sub = E.subvolume_geometry(S, 1.0, vg, pos[p], (0.0, 0.0, 0.0))
        saved = []
        _remove_subvolume(vol, m, _remove_radius(S, cfg), saved)
        done = 0
        for i in range(n):
            roi = _particle_roi(E.set_constant_values(pg[i], vg), m, vg, vs, safe, W, W)
            _cc_shift(R, vg, i, vol, [(sub, rot, roi)], roi, bufs, a.max_shift, a.multi_peak, (None, None))
            done += 1
        for region, keep in reversed(saved):
            region.copy_(keep)
        return done

    for p in range(min(a.warmup, a.particles)):  # plans, slab buffers, autotuning
        particle(p)
    torch.cuda.synchronize()
    l0 = E.kernel_launches()
    t0 = time.perf_counter()
    count = sum(particle(p) for p in range(a.particles))
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    launches = E.kernel_launches() - l0
    print(json.dumps({
        "metric": "shift measurements/s (one particle in one projection, EmSartRefine cross-correlation)",
        "value": count / dt, "unit": "measurements/s", "ms_per_measurement": 1e3 * dt / count,
        "measurements": count, "launches_per_measurement": launches / count,
        "config": {"dims": list(dims), "projection": [W, W], "n_proj": n, "box": S, "max_shift": a.max_shift,
                   "ctf": ctf, "ctf_slab_nm": 30.0 if ctf else None, "multi_peak": a.multi_peak,
                   "region": 2 * safe + 1, "particles": a.particles},
    }))
    rec.close()


if __name__ == "__main__":
    main()
