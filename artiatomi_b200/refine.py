"""EmSartRefine's per-particle shift measurement on libesb.

`refine_shifts(cfg)` reads what EmSartRefine reads (emsart.cfg in refine
mode: the reconstruction OutVolumeFile, the tilt series, marker file, motive
list and the particle Reference) and measures, for every particle and every
usable projection, the particle's extra detector shift. The shifts go to
ShiftOutputFile in the ShiftFile layout that EmSARTSubVolumes reads as its
ShiftInputFile (`reconstruct_subvolumes`).

For each particle (EmSartRefine.cpp:700-1100, one particle per group) and
projection:
- the reconstruction with the particle's cube zeroed (Volume::RemoveSubVolume,
  Volume.cpp:565-645) is forward projected over the particle's detector
  region (ForwardProjectionROI);
- the Reference, rotated to the particle's Euler angles (esb_rotate_volume,
  the reference's rot3d) and placed at the particle (esb_subvolume_geometry),
  is the model.
Both volumes are read negated, as Volume::LoadFromFile (Volume.cpp:498-550)
reads every volume (EmSart and EmSARTSubVolumes write theirs negated).

method "cc" (the reference's): the compare image of the reconstruction's
projection (Reconstructor::Compare) and the model's projection go through
Reconstructor::GetDisplacement (esb_rec_cc_displacement): the integer
arg-max of their normalised cross-correlation within MaxShift, optionally
with MultiPeakDetection; the correlation maps are written to
CCMapFileName<index>.em when that name is set. method "lsq": the model is
fitted to the residual (prepared projection minus the reconstruction's
projection) with a detector offset s, min over (alpha, s) of
1/2 ||alpha A(ref, s) - r||^2, Gauss-Newton on s
(esb_projection_loss_grad_roi) with the amplitude alpha in closed form: a
sub-pixel estimate. Both use the projector without the CTF of CtfMode.

Every computation runs in the library's CUDA kernels; this module moves
files and buffers and solves the 2 x 2 Gauss-Newton systems.
"""
from __future__ import annotations

import math

import numpy as np

from . import emsart as E
from . import fileio as F
from .config import EmSartConfig
from .reconstruct import _setup


def _particle_roi(c, m, vg, vs, safe, W, H):
    """Detector region around the particle centre (Projection::ComputeHitPoint
    of the voxel centre, widened by the reference's safeDist)."""
    bmin = np.array(vg.bbox_min[:], np.float64)
    p = bmin + (m[7:10].astype(np.float64) + m[10:13] - 1.0) * vs + 0.5 * vs
    M = np.array(c.detector_matrix[:], np.float64).reshape(4, 4)
    u = M[0, :3] @ p + M[0, 3]
    v = M[1, :3] @ p + M[1, 3]
    return (max(int(math.floor(u)) - safe, 0), max(int(math.floor(v)) - safe, 0),
            min(int(math.ceil(u)) + safe, W), min(int(math.ceil(v)) + safe, H))


def _fit_shift(c_sub, ref, target, roi, iterations, max_shift, out):
    """Gauss-Newton on the detector offset s of alpha A(ref, s) ~ target.
    Returns s (pixels, u and v) or None when the model does not reach the
    region or the fitted amplitude is not positive."""
    import torch

    x0, y0, x1, y1 = roi
    s = np.zeros(2)
    out.zero_()
    E.projection_loss_grad_roi(c_sub, ref, target, out, roi, shift=s)
    o = out.cpu().numpy()
    if not (o[6] > 0.0):
        return None
    alpha = o[7] / o[6]
    if not (alpha > 0.0):
        return None
    scaled = torch.zeros_like(target)
    for _ in range(iterations):
        # residual against target / alpha: the gradient and Gauss-Newton
        # terms of 1/2 ||A(ref, s) - target / alpha||^2
        scaled[y0:y1, x0:x1] = target[y0:y1, x0:x1] / alpha
        out.zero_()
        E.projection_loss_grad_roi(c_sub, ref, scaled, out, roi, shift=s)
        o = out.cpu().numpy()
        g = o[1:3]
        Hm = np.array([[o[3], o[4]], [o[4], o[5]]])
        if not (np.linalg.det(Hm) > 0.0):
            break
        step = -np.linalg.solve(Hm, g)
        s = np.clip(s + step, -max_shift, max_shift)
        if o[6] > 0.0 and o[7] > 0.0:
            alpha *= o[7] / o[6]
        if np.hypot(*step) < 1e-4:
            break
    return s


def _cc_shift(R, vg, i, c_full, vol, c_sub, rot, roi, bufs, max_shift, multi, maps):
    """GetDisplacement of projection i (EmSartRefine.cpp:825-980): the
    compare image of the holey reconstruction's projection against the
    model's projection. Returns the shift (x, y) as the ShiftFile stores it."""
    residual, model, mdist = bufs
    rec = R.rec
    pv, dv, _ = rec.views()
    rec.reset_projections()
    E.forward_project(c_full, vol, pv, dv, roi=roi, fast=True)
    rec.compare(vg, R.prepared[i], i)
    residual.copy_(pv)
    model.zero_()
    mdist.zero_()
    E.forward_project(c_sub, rot, model, mdist, roi=roi, fast=True)
    cmap, cmulti = maps
    (sx, sy), _ = rec.cc_displacement(residual, model, max_shift, multi, cmap, cmulti)
    return sx, sy


def refine_shifts(cfg: EmSartConfig, write: bool = True, iterations: int = 10, particles=None, method: str = "cc"):
    """Extra shifts [projection][motive][2] of every particle (the layout
    `fileio.read_shift_file` returns); written to cfg.ShiftOutputFile when
    `write`. particles: motive list rows to refine (default all); the other
    rows keep zero shifts. Projections marked unusable in the marker file and
    particles whose region misses a projection keep zero shifts there.
    method: "cc" (the reference's cross-correlation peak, integer shifts;
    (-1000, -1000) stored where no positive correlation is found, which
    EmSARTSubVolumes then leaves out) or "lsq" (sub-pixel least squares;
    iterations bounds its Gauss-Newton steps)."""
    import torch

    if method not in ("cc", "lsq"):
        raise ValueError(f"method must be 'cc' or 'lsq', not {method!r}")
    R = _setup(cfg, E.VARIANT_FAST)
    vg, dev, W, H = R.vg, R.dev, R.W, R.H
    dims = tuple(int(d) for d in cfg.RecDimensions)
    volf, _ = F.read_em(cfg.OutVolumeFile)
    if volf.shape != dims[::-1]:
        raise ValueError(f"{cfg.OutVolumeFile}: volume {volf.shape[::-1]} does not match RecDimensions {dims}")
    # Volume::LoadFromFile negates what it reads (EmSart wrote the volume
    # negated, Volume::Invert); so does it for the Reference
    vol = torch.from_numpy(np.ascontiguousarray(-volf.astype(np.float32))).to(dev)
    S = cfg.SizeSubVol
    reff, _ = F.read_em(cfg.Reference)
    if reff.shape != (S, S, S):
        raise ValueError(f"{cfg.Reference}: reference {reff.shape} is not SizeSubVol^3 = {S}^3")
    ref = torch.from_numpy(np.ascontiguousarray(-reff.astype(np.float32))).to(dev)
    rot = torch.empty_like(ref)
    motl = F.read_motive_list(cfg.MotiveList, cfg.ScaleMotivelistPosition, cfg.ScaleMotivelistShift)
    n_part, n_proj = motl.shape[0], len(R.tilt)
    index_list = E.projection_index_list(E.PLT_NORMAL, R.tilt, R.good.astype(np.int32))
    vs = np.array(cfg.VoxelSize, np.float64)
    radius = int(S / (cfg.VoxelSize[0] / cfg.VoxelSizeSubVol) / 2)  # RemoveSubVolume's half width
    safe = int(100 + cfg.VoxelSizeSubVol * S * 2 + cfg.MaxShift * 2)  # EmSartRefine's safeDist
    proj = torch.zeros((H, W), device=dev)
    dist = torch.zeros((H, W), device=dev)
    target = torch.zeros((H, W), device=dev)
    out = torch.zeros(8, dtype=torch.float64, device=dev)
    extra = np.zeros((n_proj, n_part, 2), np.float32)
    max_shift = int(cfg.MaxShift)
    multi = bool(cfg.MultiPeakDetection)
    dump = method == "cc" and len(cfg.CCMapFileName) > 3
    cc_maps, cc_multi = {}, {}
    if method == "cc":
        bufs = (torch.zeros((H, W), device=dev), torch.zeros((H, W), device=dev), torch.zeros((H, W), device=dev))
        cmap = torch.zeros((4 * max_shift, 4 * max_shift), device=dev) if dump else None
        cmulti = torch.zeros((4 * max_shift, 4 * max_shift), device=dev) if dump and multi else None
    for p in (range(n_part) if particles is None else particles):
        m = motl[p]
        E.rotate_volume(ref, rot, E.rotation_matrix(m[16], m[17], m[18]))
        sub = E.subvolume_geometry(S, cfg.VoxelSizeSubVol, vg, m[7:10], m[10:13])
        # Volume::RemoveSubVolume at the particle's position + shift (as int)
        lo = [int(m[7 + k] + m[10 + k]) - 1 - radius for k in range(3)]
        box = [(max(lo[k], 0), min(lo[k] + 2 * radius, dims[k])) for k in range(3)]
        region = vol[box[2][0]:box[2][1], box[1][0]:box[1][1], box[0][0]:box[0][1]]
        saved = region.clone()
        region.zero_()
        for i in index_list:
            i = int(i)
            c_full = E.set_constant_values(R.pg[i], vg)
            roi = _particle_roi(c_full, m, vg, vs, safe, W, H)
            x0, y0, x1, y1 = roi
            if x1 <= x0 or y1 <= y0:
                continue
            c_sub = E.set_constant_values(R.pg[i], sub)
            if method == "cc":
                sx, sy = _cc_shift(R, vg, i, c_full, vol, c_sub, rot, roi, bufs, max_shift, multi, (cmap, cmulti))
                extra[i, p] = (-sx, -sy)  # the file holds the shift; the extra shift is its negation
                if dump:
                    cc_maps.setdefault(i, []).append(cmap.cpu().numpy().copy())
                    if multi:
                        cc_multi.setdefault(i, []).append(cmulti.cpu().numpy().copy())
                continue
            proj.zero_()
            E.forward_project(c_full, vol, proj, dist, roi=roi, fast=True)
            target.zero_()
            target[y0:y1, x0:x1] = R.prepared[i][y0:y1, x0:x1] - proj[y0:y1, x0:x1]
            s = _fit_shift(c_sub, rot, target, roi, iterations, float(cfg.MaxShift), out)
            if s is not None:
                # the fitted model moves the particle's image by -s; the
                # extra shift that moves it back is -s
                extra[i, p] = -s
        region.copy_(saved)
    if write:
        # the file holds the measured displacement (ShiftFile::SetValue);
        # EmSARTSubVolumes reads it negated as the extra shift
        F.write_shift_file(cfg.ShiftOutputFile, np.moveaxis(-extra, -1, 0))
        # one slice per refined particle (EmSartRefine.cpp:986-1010)
        for i, maps in cc_maps.items():
            F.write_em(f"{cfg.CCMapFileName}{i}.em", np.stack(maps))
        for i, maps in cc_multi.items():
            F.write_em(f"{cfg.CCMapFileName}Multi_{i}.em", np.stack(maps))
    return extra
