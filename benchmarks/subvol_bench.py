"""Batched against per-particle sub-volume weighted back-projection.

  python -m benchmarks.subvol_bench [--particles 2000] [--frame 4096 4096 1024]
      [--proj 4096] [--n-proj 61] [--os 2] [--no-ctf] [--warmup 1] [--reps 1]

The sub-volume workload of EmSARTSubVolumes: particle centres uniform in the
tomogram frame, cubic boxes of 48/64/96 voxels in a 50/35/15 split, 61 tilts
(-60..+60 degrees), per-particle per-tilt extra shifts U(+-1.5 px), 3-D CTF
(300 kV, Cs 2.7 mm, pixel 0.27 nm, 30 nm slabs, defocus 3000 +- 500 nm with
100 nm astigmatism) whose slab depth follows each particle's z. The
projections are synthetic: random ellipses with the line-integral profile of
an ellipsoid plus Gaussian noise, made on the GPU.

All paths run through esb_subvolume_wbp: batched = 1 (FAST variant) runs
one persistent launch over all particles and all tilts (with CTF from the
slab-image patches gathered after each tilt's CTF chain); with CTF the
per_tilt arm runs it once per tilt over the whole slab images
(esb_reconstructor_subvolume_patches off); batched = 0 launches the
back-projection once per particle per tilt, with the FAST kernel (all slabs
of a tilt in one launch, --plain fast) or, as the reference does, with the
FAITHFUL kernel once per particle per slab (--plain faithful). Prints one
JSON line with the timings (CUDA events around the whole call, and the
back-projection phase alone), the speed-ups and the relative L2 difference
of the results.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import time

import numpy as np


def synthetic_projections(n, W, H, seed, n_ell=400):
    import torch

    g = torch.Generator(device="cuda").manual_seed(seed)
    rng = np.random.default_rng(seed)
    out = torch.empty((n, H, W), dtype=torch.float32, device="cuda")
    cx, cy = rng.uniform(0, W, n_ell), rng.uniform(0, H, n_ell)
    ax, ay = rng.uniform(4, 40, n_ell), rng.uniform(4, 40, n_ell)
    rho = rng.uniform(0.2, 1.0, n_ell)
    for i in range(n):
        img = torch.zeros((H, W), dtype=torch.float32, device="cuda")
        ang = rng.uniform(0, np.pi, n_ell)
        for e in range(n_ell):
            r = int(max(ax[e], ay[e])) + 1
            x0, x1 = max(int(cx[e]) - r, 0), min(int(cx[e]) + r + 1, W)
            y0, y1 = max(int(cy[e]) - r, 0), min(int(cy[e]) + r + 1, H)
            if x1 <= x0 or y1 <= y0:
                continue
            yy, xx = torch.meshgrid(torch.arange(y0, y1, device="cuda", dtype=torch.float32) + 0.5 - cy[e],
                                    torch.arange(x0, x1, device="cuda", dtype=torch.float32) + 0.5 - cx[e],
                                    indexing="ij")
            c, s = float(np.cos(ang[e])), float(np.sin(ang[e]))
            q = ((c * xx + s * yy) / ax[e]) ** 2 + ((-s * xx + c * yy) / ay[e]) ** 2
            img[y0:y1, x0:x1] += float(2.0 * rho[e] * min(ax[e], ay[e])) * torch.sqrt(torch.clamp(1.0 - q, min=0.0))
        img += torch.randn((H, W), generator=g, device="cuda") * (0.5 * img.std())
        out[i] = img
    return out


def build(particles, frame, W, H, n, os_, ctf, seed=0):
    from artiatomi_b200 import _lib as L
    from artiatomi_b200 import emsart as E

    rng = np.random.default_rng(seed)
    tilt = np.linspace(-60.0, 60.0, n).astype(np.float32)
    full = E.volume_geometry(tuple(frame))
    sizes = rng.choice([48, 64, 96], size=particles, p=[0.5, 0.35, 0.15])
    pos = np.stack([rng.uniform(s / 2, f - s / 2, particles) for s, f in zip((sizes, sizes, sizes), frame)], 1)
    shifts = rng.uniform(-1.5, 1.5, size=(particles, n, 2)).astype(np.float32)
    sub = [E.subvolume_geometry(int(s), 1.0, full, p) for s, p in zip(sizes, pos)]
    pair = (L.ProjGeom * (particles * n))()
    for p in range(particles):
        g = E.projection_geometry(E.Markers(tilt), W, H, extra_shift=shifts[p])
        for i in range(n):
            pair[p * n + i] = g[i]
    dmid = rng.uniform(2500.0, 3500.0, n)
    defocus = np.stack([dmid - 50.0, dmid + 50.0, rng.uniform(0.0, 180.0, n)], 1).astype(np.float32).ravel()
    kw = dict(oversampling=os_, variant=E.VARIANT_FAST)
    if ctf:
        kw.update(ctf_mode=True, pixel_size_nm=0.27, cs_mm=2.7, voltage_kv=300.0, amp_contrast=0.0,
                  ctf_slice_thickness_nm=30.0, ctf_beta_fac=(200.0, 0.0, 0.008, 0.0), wiener_noise_level=0.1)
    cfg = E.ReconConfig(W, H, n, **kw)
    pg = E.projection_geometry(E.Markers(tilt), W, H)
    return dict(tilt=tilt, full=full, sizes=sizes, sub=sub, pair=pair, cfg=cfg, pg=pg,
                defocus=defocus if ctf else None)


def main(argv=None):
    import torch

    from artiatomi_b200 import emsart as E

    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=2000)
    ap.add_argument("--frame", type=int, nargs=3, default=[4096, 4096, 1024])
    ap.add_argument("--proj", type=int, default=4096)
    ap.add_argument("--n-proj", type=int, default=61)
    ap.add_argument("--os", type=int, default=2)
    ap.add_argument("--no-ctf", action="store_true")
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--plain", choices=["fast", "faithful"], default="fast")
    a = ap.parse_args(argv)
    W = H = a.proj
    t_build = time.time()
    w = build(a.particles, a.frame, W, H, a.n_proj, a.os, not a.no_ctf, a.seed)
    projs = synthetic_projections(a.n_proj, W, H, a.seed + 1)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, w["tilt"])
    plain_cfg = dataclasses.replace(w["cfg"], variant=E.VARIANT_FAST if a.plain == "fast" else E.VARIANT_FAITHFUL)
    # arms: plain (one launch per particle per tilt), per_tilt (batched, one
    # launch per tilt over all boxes), batched (with CTF: all tilts in one
    # launch from the gathered slab-image patches)
    arms = ("plain", "per_tilt", "batched") if not a.no_ctf else ("plain", "batched")
    recs = {}
    for arm in arms:
        recs[arm] = E.Reconstructor(plain_cfg if arm == "plain" else w["cfg"], w["pg"], w["tilt"], w["defocus"])
        recs[arm].subvolume_patches(arm == "batched")  # per_tilt: the library's default
    boxes = {arm: [torch.zeros((int(s),) * 3, dtype=torch.float32, device="cuda") for s in w["sizes"]]
             for arm in arms}
    torch.cuda.synchronize()
    t_build = time.time() - t_build

    def run(arm):
        for b in boxes[arm]:
            b.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        recs[arm].subvolume_wbp(w["full"], w["sub"], w["pair"], boxes[arm], projs, il, batched=arm != "plain")
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    res = {}
    for arm in arms:
        for _ in range(a.warmup):
            run(arm)
        ms = [run(arm) for _ in range(a.reps)]
        # phase breakdown from one more run with per-launch events (kept out
        # of the timed runs: they add host work per launch)
        recs[arm].enable_timing(True)
        recs[arm].timing()
        run(arm)
        ph = recs[arm].timing()
        recs[arm].enable_timing(False)
        res[arm] = dict(ms=float(np.median(ms)), bp_ms=ph["bp"][0], bp_launches=ph["bp"][1], ctf_ms=ph["ctf"][0],
                        gather_ms=ph["compare"][0])

    def rel(x_arm, y_arm):
        num = sum(float(((x - y).double() ** 2).sum()) for x, y in zip(boxes[x_arm], boxes[y_arm]))
        den = sum(float((y.double() ** 2).sum()) for y in boxes[y_arm])
        return float(np.sqrt(num / max(den, 1e-300)))

    voxels = int(sum(int(s) ** 3 for s in w["sizes"]))
    updates = voxels * len(il)
    for r in recs.values():
        r.close()
    out = {
        "workload": "subvolume_wbp", "particles": a.particles, "frame": a.frame, "proj": [W, H],
        "n_proj": a.n_proj, "oversampling": a.os, "ctf": not a.no_ctf, "voxels": voxels, "plain": a.plain,
        "plain_ms": res["plain"]["ms"], "batched_ms": res["batched"]["ms"],
        "speedup": res["plain"]["ms"] / res["batched"]["ms"],
        "plain_bp_ms": res["plain"]["bp_ms"], "batched_bp_ms": res["batched"]["bp_ms"],
        "bp_speedup": res["plain"]["bp_ms"] / max(res["batched"]["bp_ms"], 1e-9),
        "plain_bp_launches": res["plain"]["bp_launches"], "batched_bp_launches": res["batched"]["bp_launches"],
        "plain_ctf_ms": res["plain"]["ctf_ms"], "batched_ctf_ms": res["batched"]["ctf_ms"],
        "batched_voxel_updates_per_s": updates / (res["batched"]["ms"] * 1e-3),
        "rel_l2_batched_vs_plain": rel("batched", "plain"),
        "setup_s": round(t_build, 1),
    }
    if "per_tilt" in res:
        out.update({"per_tilt_ms": res["per_tilt"]["ms"], "per_tilt_bp_ms": res["per_tilt"]["bp_ms"],
                    "per_tilt_bp_launches": res["per_tilt"]["bp_launches"],
                    "batched_gather_ms": res["batched"]["gather_ms"],
                    "speedup_vs_per_tilt": res["per_tilt"]["ms"] / res["batched"]["ms"],
                    "batched_equals_per_tilt": rel("batched", "per_tilt") == 0.0})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
