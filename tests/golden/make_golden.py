"""Generate tests/golden/reference_kernels.npz from the reference's own kernels.

Runs the reference's kernel sources (src/EmSART/cuda_kernels/*.cu, compiled
for the host by oracle/ref_build.py) on small seeded inputs and stores
inputs and outputs. tests/test_oracle_pinning.py checks the CPU oracle
against these vectors where the reference tree is absent.

  python tests/golden/make_golden.py    (needs the reference tree; see oracle/ref_build.py)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

OUT = Path(__file__).resolve().parent / "reference_kernels.npz"

# The case: a 32x32x16 phantom, 5 tilts of 32^2 with shifts and psi jitter.
DIMS, W, H, TILTS = (32, 32, 16), 32, 32, (-60.0, -27.0, 0.0, 33.0, 60.0)


def geometry():
    from oracle import geometry as G

    rng = np.random.default_rng(2024)
    n = len(TILTS)
    xs = rng.uniform(-1.5, 1.5, n).astype(np.float32)
    ys = rng.uniform(-1.5, 1.5, n).astype(np.float32)
    psi = rng.uniform(-0.5, 0.5, n).astype(np.float32)
    tilt = np.array(TILTS, np.float32)
    og = G.projection_geometry(tilt, xs, ys, None, psi, W, H)
    return tilt, xs, ys, psi, og, G.volume_geometry(DIMS)


def inputs():
    from artiatomi_b200 import phantom as PH

    rng = np.random.default_rng(7)
    vol = PH.phantom_numpy(DIMS, 12, seed=3)
    imgs = rng.normal(size=(len(TILTS), H, W)).astype(np.float32)
    spec = rng.normal(size=(64, 33, 2)).astype(np.float32)
    return vol, imgs, spec


def main():
    from oracle import geometry as G
    from oracle import ref as R
    from oracle import ref_build

    ref_build.build(verbose=True)
    if R.lib() is None:
        raise SystemExit("reference kernels are not built (reference tree missing)")
    tilt, xs, ys, psi, og, vo = geometry()
    vol, imgs, spec = inputs()
    out = dict(tilt=tilt, xs=xs, ys=ys, psi=psi, vol=vol, imgs=imgs, spec=spec)
    for i in range(len(TILTS)):
        g = G.orc_geom(og[i], vo)
        p = np.zeros((H, W), np.float32)
        d = np.zeros((H, W), np.float32)
        R.march(g, vol, W, H, p, d)
        out[f"march_proj_{i}"], out[f"march_dist_{i}"] = p, d
        t0, t1 = G.defocus_distances(og[i], vo)
        s = np.zeros((H, W), np.float32)
        R.slicer(g, vol, W, H, s, t0 + 2.0, t0 + 9.5)
        out[f"slicer_{i}"] = s
        gb = G.orc_geom(og[i], vo, for_bp=True)
        for os_, lin in ((1, 0), (2, 1), (3, 0)):
            v = np.zeros(vol.shape, np.float32)
            R.bp(gb, v, 0, imgs[i], 0.5, os_, linear=lin)
            out[f"bp_{i}_{os_}_{lin}"] = v
        c = imgs[i].copy()
        R.compare(imgs[(i + 1) % len(TILTS)] * 3, c, np.abs(imgs[(i + 2) % len(TILTS)]) * 20, 16.0,
                  (1.0, 2.0, 1.0, 2.0), (3.0, 4.0, 3.0, 4.0), 1.0)
        out[f"compare_{i}"] = c
        cb = imgs[i].copy()
        R.crop_border(cb, (1.0, 2.0), (4.0, 3.0), G.compute_hit_points(og[i], vo))
        out[f"crop_{i}"] = cb
    for fp in (1, 0):
        sp = spec.copy()
        R.ctf(sp, 3050.0, 3150.0, 33.0, fp, 0, 0.1, (5.0, 0.0, 0.008, 0.0), 2.7, 300.0, 0.0, 0.27)
        out[f"ctf_{fp}"] = sp
    for fm in range(5):
        sp = spec.copy()
        R.wbp_weighting(sp, 1.3, fm)
        out[f"wbp_{fm}"] = sp
    sp = spec.copy()
    R.fourier_filter(sp, 20.0, 3.0, 4.0, 1.0)
    out["fourier"] = sp
    sp = spec.copy()
    R.dose_weighting(sp, 3.5, 2.7)
    out["dose"] = sp
    sq_in = np.ascontiguousarray(imgs[0][:, :24])
    out["square_zero"] = R.make_square(sq_in, 40, 8, 4, 0, 1)
    out["square_mirror"] = R.make_square(sq_in, 40, 8, 4, 1, 0)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
