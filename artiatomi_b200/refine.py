"""EmSartRefine's per-particle shift measurement on libesb.

`refine_shifts(cfg)` reads what EmSartRefine reads (emsart.cfg in refine
mode: the reconstruction OutVolumeFile, the tilt series, marker file, motive
list and the particle Reference) and measures, for every particle and every
usable projection, the particle's extra detector shift. The shifts go to
ShiftOutputFile in the ShiftFile layout that EmSARTSubVolumes reads as its
ShiftInputFile (`reconstruct_subvolumes`).

For each group of particles (EmSartRefine.cpp:697-1090: GroupMode ByGroup,
MaxDistance or MaxCount, plus the supporting particles of
SupportingReferences / SupportingMotiveLists) and projection:
- the reconstruction with the particles' cubes zeroed
  (Volume::RemoveSubVolume, Volume.cpp:565-645) is forward projected over
  the union of the particles' detector regions (ForwardProjectionROI);
- each particle's reference, rotated to its Euler angles (esb_rotate_volume,
  the reference's rot3d) and placed at the particle (esb_subvolume_geometry),
  is projected over its region; the sum is the model.
The volumes are read negated, as Volume::LoadFromFile (Volume.cpp:498-550)
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
sub-pixel estimate. Method "cc" projects through the reconstructor
(ForwardProjectionROI, with the per-slab CTF in CtfMode); method "lsq" uses
the plain ray integrals.

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


def hit_point(pg, x, y, z):
    """Projection::ComputeHitPoint (Projection.cpp:1051-1085) in float32: the
    foot of the normal from (x, y, z) on projection pg's detector plane,
    through its detector matrix (GetDetectorMatrix with os 1), each pixel
    coordinate truncated to int as the reference assigns it to an int2."""
    f = np.float32
    p = [f(x), f(y), f(z)]
    d = [f(a) for a in pg.detektor]
    n = [f(a) for a in pg.proj_norm]
    t = (n[0] * p[0] + n[1] * p[1]) + n[2] * p[2]
    t = t + (((-n[0]) * d[0] - n[1] * d[1]) - n[2] * d[2])
    t = abs(t)
    h = [t * (-n[k]) + p[k] for k in range(3)]
    M = [f(a) for a in pg.detector_matrix]
    u = ((M[0] * h[0] + M[1] * h[1]) + M[2] * h[2]) + f(1) * M[3]
    v = ((M[4] * h[0] + M[5] * h[1]) + M[6] * h[2]) + f(1) * M[7]
    return int(u), int(v)


def safe_dist(cfg: EmSartConfig) -> int:
    """EmSartRefine's safeDist, 100 + VoxelSizeSubVol * SizeSubVol * 2 +
    MaxShift * 2 evaluated in float and truncated (EmSartRefine.cpp:830)."""
    f = np.float32
    return int(f(100) + f(cfg.VoxelSizeSubVol) * f(cfg.SizeSubVol) * f(2) + f(int(cfg.MaxShift) * 2))


def particle_roi(pg, m, vg, vs, safe, mag_inv):
    """A particle's detector region as EmSartRefine.cpp:815-847 forms it:
    the hit point of the particle centre (bbMin + (coord + shift - 1) * vs +
    vs / 2, in float), as ints, through the inverse magnification anisotropy
    (MatrixVector3Mul of the 3 x 3 matrix on (x, y, 1)), then
    floor - safeDist .. ceil + safeDist; the minima clamped at 0, the maxima
    not (the projection kernels clip them to the detector). Returns
    (x_min, y_min, x_max, y_max)."""
    f = np.float32
    bmin = [f(a) for a in vg.bbox_min]
    vs = [f(a) for a in vs]
    c = [(bmin[k] + ((f(m[7 + k]) + f(m[10 + k])) - f(1)) * vs[k]) + f(0.5) * vs[k] for k in range(3)]
    hx, hy = hit_point(pg, *c)
    A = [f(a) for a in np.asarray(mag_inv, np.float32).ravel()]
    x = (A[0] * f(hx) + A[1] * f(hy)) + A[2] * f(1)
    y = (A[3] * f(hx) + A[4] * f(hy)) + A[5] * f(1)
    return (max(int(math.floor(x)) - safe, 0), max(int(math.floor(y)) - safe, 0),
            int(math.ceil(x)) + safe, int(math.ceil(y)) + safe)


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


def _distance(a, b):
    """MotiveList::GetDistance (MotiveList.cpp:121-130): float distance of two
    particles' coordinates."""
    d = (a[7:10] - b[7:10]).astype(np.float32)
    return np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])))


def global_index(motl, i):
    """MotiveList::GetGlobalIdx (MotiveList.cpp:254-263): the first row equal
    to row i in every field."""
    return int(np.flatnonzero((motl == motl[i]).all(axis=1))[0])


def group_count(motl, mode):
    """MotiveList::GetGroupCount (MotiveList.cpp:233-245): the distinct
    classNo values for ByGroup, one group per particle otherwise."""
    if mode == "ByGroup":
        return len(dict.fromkeys(motl[:, 19].tolist()))
    return motl.shape[0]


def group_members(motl, group, mode, max_distance=0.0, group_size=1):
    """MotiveList::GetNeighbours(index, mode, maxDist, groupSize)
    (MotiveList.cpp:132-230): the rows of a group, its leader first.
    ByGroup: the particles of the group-th classNo in order of first
    appearance; MaxDistance: the particle, then every other within
    max_distance in row order; MaxCount: the group_size nearest particles,
    ordered by (distance, row)."""
    n = motl.shape[0]
    if mode == "ByGroup":
        classes = list(dict.fromkeys(motl[:, 19].tolist()))
        if group < 0 or group >= len(classes):
            return []
        return [i for i in range(n) if motl[i, 19] == classes[group]]
    if mode == "MaxDistance":
        md = np.float32(max_distance)
        return [group] + [i for i in range(n) if i != group and _distance(motl[i], motl[group]) <= md]
    if mode == "MaxCount":
        order = sorted((float(_distance(motl[i], motl[group])), i) for i in range(n))
        return [i for _, i in order[:min(group_size, n)]]
    raise ValueError(f"GroupMode {mode!r}")


def support_members(leader, support_lists, max_distance):
    """MotiveList::GetNeighbours(index, maxDist, supporters)
    (MotiveList.cpp:184-205): (list number, row) of every supporting particle
    within max_distance of the leader."""
    md = np.float32(max_distance)
    return [(s, j) for s, lst in enumerate(support_lists) for j in range(lst.shape[0])
            if _distance(lst[j], leader) <= md]


def groups(motl, mode, processed, max_distance=0.0, group_size=1, only=None):
    """The groups EmSartRefine measures, in its order (EmSartRefine.cpp:
    697-730): (group number, member rows, leader's global index). A MaxCount
    or MaxDistance group whose leader already received a shift is skipped;
    `processed` is read as the caller updates it. only: the group numbers
    to consider (default all)."""
    for group in (range(group_count(motl, mode)) if only is None else only):
        members = group_members(motl, group, mode, max_distance, group_size)
        if not members:
            continue
        lead = global_index(motl, members[0])
        if mode in ("MaxCount", "MaxDistance") and processed[lead]:
            continue
        yield group, members, lead


def shift_receivers(motl, members, mode, speed_up):
    """Global indices that get a group's shift in one projection, in the
    order EmSartRefine.cpp:1024-1086 stores them: every member (ByGroup), or
    the members within speed_up of the leader and then the leader."""
    if mode == "ByGroup":
        return [global_index(motl, k) for k in members]
    out, min_dist = [], {}  # minDistOfProcessedParticles, reset per projection
    for k in members[1:]:
        g2 = global_index(motl, k)
        d = _distance(motl[members[0]], motl[k])
        if d <= np.float32(speed_up) and d < min_dist.get(g2, np.float32(1.0e8)):
            out.append(g2)
            min_dist[g2] = d
    out.append(global_index(motl, members[0]))
    return out


def _remove_radius(size, cfg):
    """The half width EmSartRefine passes to Volume::RemoveSubVolume: size /
    (VoxelSize.x / VoxelSizeSubVol) / 2 in float, truncated."""
    adjust = np.float32(np.float32(cfg.VoxelSize[0]) / np.float32(cfg.VoxelSizeSubVol))
    return int(np.float32(np.float32(size) / adjust) / np.float32(2.0))


def _remove_subvolume(vol, m, radius, saved):
    """Volume::RemoveSubVolume (Volume.cpp:565-645) at the particle's
    position + shift (float sum truncated to int, 1-based): zero the cube of
    half width radius, keeping its contents in `saved`."""
    dims = vol.shape[::-1]
    lo = [int(np.float32(m[7 + k] + m[10 + k])) - 1 - radius for k in range(3)]
    box = [(max(lo[k], 0), min(lo[k] + 2 * radius, dims[k])) for k in range(3)]
    if any(b[1] <= b[0] for b in box):
        return
    region = vol[box[2][0]:box[2][1], box[1][0]:box[1][1], box[0][0]:box[0][1]]
    saved.append((region, region.clone()))
    region.zero_()


def _cc_shift(R, vg, i, vol, parts_roi, roi, bufs, max_shift, multi, maps):
    """GetDisplacement of projection i (EmSartRefine.cpp:825-980): the holey
    reconstruction's projection over the union region goes through Compare;
    the particles' projections (each over its region) are the model; both
    through GetDisplacement. Projections are the reconstructor's
    (ForwardProjectionROI: with CTF in CtfMode). bufs: a residual image and
    the reconstructor's projection buffer. Returns the shift (x, y) as the
    ShiftFile stores it, and the correlation maximum."""
    residual, proj = bufs
    rec = R.rec
    rec.reset_projections()
    rec.forward_projection_roi(vg, vol, i, roi)
    rec.compare(vg, R.prepared[i], i)
    residual.copy_(proj)
    rec.reset_projections()
    for sub, rot, r in parts_roi:
        rec.forward_projection_roi(sub, rot, i, r)
    cmap, cmulti = maps
    # the model stays in the projection buffer (the reference copies it to
    # projSubVols_d first, CopyProjectionToSubVolumeProjection)
    (sx, sy), value = rec.cc_displacement(residual, proj, max_shift, multi, cmap, cmulti)
    return sx, sy, value


def write_relations(path, relations, cc_values):
    """The `<ShiftOutputFile>.relations` text EmSartRefine writes
    (EmSartRefine.cpp:1104-1116): per particle "particleNr; particleNrInTomo;
    particleNrInTomo; obtainedShiftFromID; CCValue" (the second number
    written twice, as the reference does), integers as ints and the value as
    a C++ stream formats a float."""
    with open(path, "w") as f:
        for r, v in zip(relations, cc_values):
            f.write(f"{int(r[0])}; {int(r[1])}; {int(r[1])}; {int(r[3])}; {'%g' % float(np.float32(v))}\n")


def refine_shifts(cfg: EmSartConfig, write: bool = True, iterations: int = 10, particles=None, method: str = "cc"):
    """Extra shifts [projection][motive][2] of every particle (the layout
    `fileio.read_shift_file` returns); written to cfg.ShiftOutputFile when
    `write`.

    The groups of cfg.GroupMode (EmSartRefine.cpp:697-1090): each group's
    particles (and the supporting particles within MaxDistanceSupport of its
    leader) are cut out of the reconstruction and their rotated references
    projected together as the model; the measured shift goes to every member
    (ByGroup) or to the leader and the members within SpeedUpDistance of it
    (MaxDistance, MaxCount; a particle that received a shift is not a leader
    later). particles: the group numbers to process (default all; rows of
    the motive list for MaxDistance and MaxCount). Projections marked
    unusable in the marker file and groups whose region misses a projection
    keep zero shifts there.

    method: "cc" (the reference's cross-correlation peak, integer shifts;
    (-1000, -1000) stored where no positive correlation is found, which
    EmSARTSubVolumes then leaves out) or "lsq" (sub-pixel least squares, for
    groups of one particle without supporting particles; iterations bounds
    its Gauss-Newton steps)."""
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
    # negated, Volume::Invert); so it does for the references
    vol = torch.from_numpy(np.ascontiguousarray(-volf.astype(np.float32))).to(dev)
    S = cfg.SizeSubVol

    def load_reference(path, size=None):
        r, _ = F.read_em(path)
        if size is not None and r.shape != (size, size, size):
            raise ValueError(f"{path}: reference {r.shape} is not SizeSubVol^3 = {size}^3")
        if len(set(r.shape)) != 1:
            raise ValueError(f"{path}: reference {r.shape} is not a cube")
        return torch.from_numpy(np.ascontiguousarray(-r.astype(np.float32))).to(dev)

    ref = load_reference(cfg.Reference, S)
    sup_refs = [load_reference(pth) for pth in cfg.SupportingReferences]
    motl = F.read_motive_list(cfg.MotiveList, cfg.ScaleMotivelistPosition, cfg.ScaleMotivelistShift)
    sup_lists = [F.read_motive_list(pth, cfg.ScaleMotivelistPosition, cfg.ScaleMotivelistShift)
                 for pth in cfg.SupportingMotiveLists]
    if len(sup_lists) < len(sup_refs):
        raise ValueError("every supporting reference needs its supporting motive list")
    n_part, n_proj = motl.shape[0], len(R.tilt)
    index_list = E.projection_index_list(E.PLT_NORMAL, R.tilt, R.good.astype(np.int32))
    vs = np.array(cfg.VoxelSize, np.float32)
    safe = safe_dist(cfg)
    extra = np.zeros((n_proj, n_part, 2), np.float32)
    max_shift = int(cfg.MaxShift)
    multi = bool(cfg.MultiPeakDetection)
    mode = cfg.GroupMode
    speed_up = np.float32(cfg.SpeedUpDistance)
    dump = method == "cc" and len(cfg.CCMapFileName) > 3
    cc_maps, cc_multi = {}, {}
    bufs = (torch.zeros((H, W), device=dev), R.rec.views()[0])  # residual, the projection buffer
    cmap = torch.zeros((4 * max_shift, 4 * max_shift), device=dev) if dump else None
    cmulti = torch.zeros((4 * max_shift, 4 * max_shift), device=dev) if dump and multi else None
    proj = torch.zeros((H, W), device=dev)
    dist = torch.zeros((H, W), device=dev)
    target = torch.zeros((H, W), device=dev)
    out = torch.zeros(8, dtype=torch.float64, device=dev)
    processed = np.zeros(n_part, bool)
    # groupRelations per particle: particleNr, particleNrInTomo, tomoNr,
    # obtainedShiftFromID; and CCValue (EmSartRefine.cpp:74-81, zeroed)
    relations = np.zeros((n_part, 4), np.int64)
    rel_cc = np.zeros(n_part, np.float32)
    for group, members, lead in groups(motl, mode, processed, cfg.MaxDistance, cfg.GroupSize, particles):
        receivers = shift_receivers(motl, members, mode, speed_up)
        support = support_members(motl[lead], sup_lists[:len(sup_refs)], cfg.MaxDistanceSupport) if sup_refs else []
        if method == "lsq" and (len(members) > 1 or support):
            raise ValueError("method 'lsq' fits groups of one particle without supporting particles")
        # the particles' rotated references and their boxes; the holey volume
        saved = []
        parts = []
        for k in members:
            m = motl[k]
            rot = torch.empty_like(ref)
            E.rotate_volume(ref, rot, E.rotation_matrix(m[16], m[17], m[18]))
            parts.append((m, rot, E.subvolume_geometry(S, cfg.VoxelSizeSubVol, vg, m[7:10], m[10:13])))
            _remove_subvolume(vol, m, _remove_radius(S, cfg), saved)
        for s_idx, j in support:
            m = sup_lists[s_idx][j]
            sref = sup_refs[s_idx]
            rot = torch.empty_like(sref)
            E.rotate_volume(sref, rot, E.rotation_matrix(m[16], m[17], m[18]))
            size = sref.shape[0]
            parts.append((m, rot, E.subvolume_geometry(size, cfg.VoxelSizeSubVol, vg, m[7:10], m[10:13])))
            _remove_subvolume(vol, m, _remove_radius(size, cfg), saved)
        for i in index_list:
            i = int(i)
            c_full = E.set_constant_values(R.pg[i], vg)
            # the model: every particle projected over its own region; the
            # reconstruction over the union of the regions, which starts as
            # (W, H)..(0, 0) (EmSartRefine.cpp:799-800, 838-847)
            x0, y0, x1, y1 = W, H, 0, 0
            parts_roi = []
            for m, rot, sub in parts:
                r = particle_roi(R.pg[i], m, vg, vs, safe, R.mag_inv)
                x0, y0, x1, y1 = min(x0, r[0]), min(y0, r[1]), max(x1, r[2]), max(y1, r[3])
                parts_roi.append((sub, rot, r))
            roi = (x0, y0, min(x1, W), min(y1, H))
            if method == "cc":
                # an empty union is measured as the reference measures it:
                # nothing is projected, GetDisplacement of the images as they
                # are (no positive correlation: the shift (-1000, -1000))
                sx, sy, cc_value = _cc_shift(R, vg, i, vol, parts_roi, roi, bufs, max_shift, multi, (cmap, cmulti))
                shift = np.array([-sx, -sy], np.float32)  # the file holds the shift; the extra shift is its negation
                if dump:
                    cc_maps.setdefault(i, []).append(cmap.cpu().numpy().copy())
                    if multi:
                        cc_multi.setdefault(i, []).append(cmulti.cpu().numpy().copy())
            else:
                if roi[2] <= roi[0] or roi[3] <= roi[1]:
                    continue
                m, rot, sub = parts[0]
                proj.zero_()
                E.forward_project(c_full, vol, proj, dist, roi=roi, fast=True)
                target.zero_()
                target[y0:y1, x0:x1] = R.prepared[i][y0:y1, x0:x1] - proj[y0:y1, x0:x1]
                s = _fit_shift(E.set_constant_values(R.pg[i], sub), rot, target, roi, iterations,
                               float(cfg.MaxShift), out)
                if s is None:
                    continue
                # the fitted model moves the particle's image by -s; the
                # extra shift that moves it back is -s
                shift = (-s).astype(np.float32)
            # EmSartRefine.cpp:1024-1086: the group's shift to its particles;
            # the relations name the group (ByGroup) or the leader, and are
            # kept for every receiver but a MaxCount / MaxDistance leader
            for g2 in receivers:
                extra[i, g2] = shift
                if mode != "ByGroup":
                    processed[g2] = True
                if method == "cc" and (mode == "ByGroup" or g2 != lead):
                    mm = motl[g2]
                    relations[g2] = (int(mm[3]), int(mm[5]), int(mm[4]), group if mode == "ByGroup" else lead)
                    rel_cc[g2] = cc_value
        for region, keep in reversed(saved):
            region.copy_(keep)
        if write:  # the shifts so far, in case the run stops (EmSartRefine.cpp:1091-1095)
            F.write_shift_file(cfg.ShiftOutputFile, np.moveaxis(-extra, -1, 0))
    if write:
        # the file holds the measured displacement (ShiftFile::SetValue);
        # EmSARTSubVolumes reads it negated as the extra shift
        F.write_shift_file(cfg.ShiftOutputFile, np.moveaxis(-extra, -1, 0))
        if method == "cc":
            write_relations(cfg.ShiftOutputFile + ".relations", relations, rel_cc)
        # one slice per group (EmSartRefine.cpp:986-1010)
        for i, maps in cc_maps.items():
            F.write_em(f"{cfg.CCMapFileName}{i}.em", np.stack(maps))
        for i, maps in cc_multi.items():
            F.write_em(f"{cfg.CCMapFileName}Multi_{i}.em", np.stack(maps))
    return extra
