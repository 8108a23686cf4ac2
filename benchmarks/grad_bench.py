"""Differentiation workload: gradients of the projection loss and shift refinement.

  python -m benchmarks.grad_bench [--dims 512 512 128] [--proj 512] [--n-proj 41]
      [--max-shift 3] [--steps 20]

Volume: a seeded ellipsoid phantom of the given size; 41 tilts (-60..+60
degrees) of W x W pixels, per-tilt detector offsets U(+-max_shift px)
injected into the measured projections b = A(x, s_true). Times one pass of
esb_projection_loss_grad over all tilts (loss, dL/dx for the whole volume,
dL/ds and Gauss-Newton terms per tilt), then runs `steps` Gauss-Newton steps
on the per-tilt offsets from s = 0 with the volume known, and prints one JSON
line: per-pass time, volume gradient throughput, the largest remaining
offset error in pixels after the last step and the loss history.
"""
from __future__ import annotations

import argparse
import json

import numpy as np


def main(argv=None):
    import torch

    from artiatomi_b200 import emsart as E
    from artiatomi_b200 import phantom as PH

    ap = argparse.ArgumentParser()
    ap.add_argument("--dims", type=int, nargs=3, default=[512, 512, 128])
    ap.add_argument("--proj", type=int, default=512)
    ap.add_argument("--n-proj", type=int, default=41)
    ap.add_argument("--max-shift", type=float, default=3.0)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--n-ell", type=int, default=400)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    nx, ny, nz = a.dims
    W = H = a.proj
    n = a.n_proj
    tilt = PH.tilt_series(n, -60.0, 60.0)
    pg = E.projection_geometry(E.Markers(tilt), W, H)
    vg = E.volume_geometry((nx, ny, nz))
    consts = [E.set_constant_values(pg[i], vg) for i in range(n)]
    vol = PH.phantom_torch((nx, ny, nz), a.n_ell, seed=a.seed)
    rng = np.random.default_rng(a.seed + 1)
    true = rng.uniform(-a.max_shift, a.max_shift, size=(n, 2))
    outs = torch.zeros((n, 6), dtype=torch.float64, device="cuda")
    meas = torch.zeros((n, H, W), device="cuda")
    for i in range(n):
        E.projection_loss_grad(consts[i], vol, None, outs[i], shift=tuple(true[i]), proj_out=meas[i])
    grad = torch.zeros_like(vol)

    def full_pass(s):
        outs.zero_()
        grad.zero_()
        for i in range(n):
            E.projection_loss_grad(consts[i], vol, meas[i], outs[i], shift=tuple(s[i]), grad=grad)

    s0 = np.zeros((n, 2))
    full_pass(s0)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    full_pass(s0)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    s = s0.copy()
    losses = []
    for _ in range(a.steps):
        outs.zero_()
        for i in range(n):
            E.projection_loss_grad(consts[i], vol, meas[i], outs[i], shift=tuple(s[i]))
        o = outs.cpu().numpy()
        losses.append(float(o[:, 0].sum()))
        for i in range(n):
            Hm = np.array([[o[i, 3], o[i, 4]], [o[i, 4], o[i, 5]]]) + np.eye(2) * 1e-6 * (o[i, 3] + o[i, 5])
            step = np.linalg.solve(Hm, o[i, 1:3])
            nrm = np.linalg.norm(step)
            if nrm > 1.0:
                step /= nrm
            s[i] -= step
    err = float(np.abs(s - true).max())
    print(json.dumps({"workload": "projection_loss_grad", "dims": a.dims, "proj": [W, H], "n_proj": n,
                      "max_shift_px": a.max_shift, "ms_per_pass": ms,
                      "voxel_tilt_pairs_per_s": nx * ny * nz * n / (ms * 1e-3),
                      "gauss_newton_steps": a.steps, "max_shift_error_px": err,
                      "loss_first": losses[0] if losses else None, "loss_last": losses[-1] if losses else None}))


if __name__ == "__main__":
    main()
