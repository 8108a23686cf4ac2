"""EmSART's reconstruction run (EmSart.cpp main, SART and WBP) on libesb.

`reconstruct(cfg)` reads the tilt series, marker file and CTF file named by
an `EmSartConfig` (emsart.cfg), prepares every usable projection on the GPU
(Reconstructor::PrepareProjection), runs SART (or WBP: one back-projection
per projection of the filtered images, EmSart.cpp:575-583, 624-629) and
writes the volume as EmSart.cpp:694-813 does (negated FP32, or FP16 when
FP16Volume and WriteVolumeAsFP16 are set). `reconstruct_subvolumes(cfg)`
is EmSartSubVolumes' run: the particle boxes of a motive list with their
per-tilt extra shifts. Every computation runs in the library's CUDA
kernels; this module only moves files and buffers.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import emsart as E
from . import fileio as F
from .config import EmSartConfig

_PIX = {np.dtype(np.float32): "float32", np.dtype(np.int16): "int16", np.dtype(np.uint16): "uint16",
        np.dtype(np.int32): "int32", np.dtype(np.uint32): "uint32"}


@dataclass
class _Run:
    rec: object
    pg: object
    vg: object
    markers: object
    tilt: np.ndarray
    good: np.ndarray
    prepared: object
    stats: list
    pixel_nm: float
    tc: object
    dev: object
    W: int
    H: int
    mag_inv: np.ndarray  # the inverse magnification anisotropy, 3 x 3 row-major


def _rank_world(rank, world):
    """This process's rank and the number of ranks: the arguments, else
    torch.distributed's when it is initialised, else one rank."""
    if rank is not None and world is not None:
        return int(rank), int(world)
    try:
        import torch.distributed as dist

        if dist.is_available() and dist.is_initialized():
            return dist.get_rank(), dist.get_world_size()
    except ImportError:
        pass
    return 0, 1


def _setup(cfg: EmSartConfig, variant: int, rank: int = 0) -> _Run:
    """Files in, geometry, reconstructor and the prepared projections
    (EmSart.cpp / EmSartSubVolumes.cpp up to the reconstruction loop). Rank r
    runs on CudaDeviceID[r] (the reference's CudaDeviceIDs[mpi_offset +
    mpi_host_rank], EmSartSubVolumes.cpp:297-299, on one node), on device r
    when the list is shorter."""
    import torch

    ids = list(cfg.CudaDeviceID or [])
    dev = torch.device("cuda", ids[rank] if rank < len(ids) else rank)
    torch.cuda.set_device(dev)
    stack, pixel_nm = F.read_stack(cfg.ProjectionFile)
    if stack.dtype not in _PIX:
        raise TypeError("Projections have wrong data type: supported types are: short, ushort, int, uint and float.")
    n, H, W = stack.shape
    md = F.read_markers(cfg.MarkerFile, cfg.ReferenceMarker)
    if md.projection_count != n:
        raise ValueError(f"marker file has {md.projection_count} projections, the stack {n}")
    markers = md.markers()
    tc = E.TiltConfig(cfg.AddTiltAngle, cfg.AddTiltXAngle, cfg.UseFixPsiAngle, cfg.PsiAngle, cfg.PhiAngle)
    pg = E.projection_geometry(markers, W, H, tc)
    vg = E.volume_geometry(cfg.RecDimensions, cfg.VoxelSize, cfg.VolumeShift)
    amount, angle = cfg.MagAnisotropy
    mag = E.mag_aniso_matrix(amount, angle, W, H)
    # GetMagAnistropyMatrix(1.0f / amount, ...): the reciprocal in float
    mag_inv = E.mag_aniso_matrix(float(np.float32(1.0) / np.float32(amount)), angle, W, H)
    defocus = F.read_ctf(cfg.CtfFile).ravel() if cfg.CtfMode else None
    rc = E.ReconConfig(W, H, n, lambda_=cfg.Lambda, oversampling=cfg.OverSampling, ctf_mode=cfg.CtfMode,
                       cut_length=cfg.CutLength, dim_length=cfg.DimLength, crop=cfg.Crop, crop_dim=cfg.CropDim,
                       projection_scale_factor=cfg.ProjectionScaleFactor, pixel_size_nm=pixel_nm, cs_mm=cfg.Cs,
                       voltage_kv=cfg.Voltage, amp_contrast=0.0, ctf_slice_thickness_nm=cfg.CTFSliceThickness,
                       ctf_beta_fac=cfg.CTFBetaFac, wiener_noise_level=cfg.WienerFilterNoiseLevel,
                       phase_flip_only=cfg.PhaseFlipOnly, ignore_z_shift_for_ctf=cfg.IgnoreZShiftForCTF,
                       switch_ctf_direction=cfg.SwitchCTFDirectionForIMOD, volume_shift=cfg.VolumeShift,
                       add_tilt_angle=cfg.AddTiltAngle, variant=variant)
    tilt = markers.tilt_angle
    rec = E.Reconstructor(rc, pg, tilt, defocus, mag, mag_inv)
    good = md.good()
    # PrepareProjection for every usable projection (EmSart.cpp:534-572)
    prepared = torch.zeros((n, H, W), dtype=torch.float32, device=dev)
    stats = []
    psi = markers.rotation_psi
    for i in range(n):
        if not good[i]:
            stats.append(None)
            continue
        raw = torch.from_numpy(np.ascontiguousarray(stack[i])).to(dev)
        pc = dict(wbp=int(cfg.WBP), normalization=cfg.ProjectionNormalization,
                  correct_bad_pixels=int(cfg.CorrectBadPixels), bad_pixel_value=cfg.BadPixelValue,
                  mirror_y=int(cfg.ProjectionFile.rfind(".dm4") >= 0), skip_filter=int(cfg.SkipFilter),
                  lp=float(cfg.fourFilterLP), hp=float(cfg.fourFilterHP), lps=float(cfg.fourFilterLPS),
                  hps=float(cfg.fourFilterHPS), dose_weighting=int(cfg.DoseWeighting),
                  accumulated_dose=float(cfg.AccumulatedDose[i]) if cfg.DoseWeighting else 0.0,
                  pixel_size_nm=pixel_nm, down_weight_tilts=int(cfg.DownWeightTiltsForWBP),
                  tilt_deg=float(tilt[i]), psi_deg=float(psi[i] if psi is not None else 0.0),
                  wbp_filter=cfg.WBPFilter)
        stats.append(rec.prepare_projection(raw, prepared[i], **pc))
    return _Run(rec, pg, vg, markers, tilt, good, prepared, stats, pixel_nm, tc, dev, W, H, mag_inv)


def reconstruct(cfg: EmSartConfig, write: bool = True, variant: int = E.VARIANT_FAST, graphs: bool = True):
    """Runs the configured reconstruction; returns the volume as written
    ([z][y][x], numpy) and the Reconstructor statistics per projection."""
    import torch

    R = _setup(cfg, variant)
    rec, vg, dev = R.rec, R.vg, R.dev
    index_list = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, R.tilt, R.good.astype(np.int32))
    vol = torch.zeros(tuple(int(d) for d in cfg.RecDimensions[::-1]), device=dev,
                      dtype=torch.float16 if cfg.FP16Volume else torch.float32)
    if cfg.WBP:  # one back-projection of every filtered projection (EmSart.cpp:575-583, 624-651)
        proj_v, _, _ = rec.views()
        for index in index_list:
            proj_v.copy_(R.prepared[int(index)])
            rec.back_projection(vg, vol, int(index), 1.0)
    else:
        rec.enable_graphs(graphs)
        rec.sart(vg, vol, R.prepared, index_list, iterations=cfg.Iterations, sirt_count=cfg.SIRTCount,
                 volume_is_empty=True)
    torch.cuda.synchronize()
    # output (EmSart.cpp:694-813): FP32 volumes are negated (Volume::Invert),
    # FP16 volumes too when converted to float (convertVolumeFP16ToFP32,
    # BackProjectionSquareOS.cu:1296-1323), FP16 output is written as stored
    if cfg.FP16Volume and cfg.WriteVolumeAsFP16:
        out = vol.cpu().numpy()
    else:
        out = _negated(vol, dev)
    rec.close()
    if write:
        F.write_volume(cfg.OutVolumeFile, out, R.pixel_nm, cfg.VoxelSize[0])
    return out, R.stats


def _negated(vol, dev):
    import torch

    neg = torch.empty(vol.shape, dtype=torch.float32, device=dev)
    E.convert_volume(vol, neg, negate=True)
    torch.cuda.synchronize()
    return neg.cpu().numpy()


@dataclass
class SubvolumeBatch:
    """One batch of EmSartSubVolumes' particle loop on one rank."""
    parts: list  # motive-list indices of this rank's particles
    sub: list  # VolGeom of each particle's box
    pair: object  # ProjGeom[len(parts) * n_proj]: detector frames with the particle's extra shift
    active: np.ndarray  # [particle][projection]: |extra shift| < MaxShift - 0.5


def subvolume_batches(cfg: EmSartConfig, markers, tc, vg, W: int, H: int, rank: int = 0, world: int = 1):
    """The host side of EmSartSubVolumes' particle loop
    (EmSartSubVolumes.cpp:611-668) for one rank: the motive list in batches of
    BatchSize, each batch split over the ranks (distributed.batch_particles),
    and per particle its box placement (Volume::PositionInSpace) and the
    detector frames with its extra shifts. No device work."""
    from .distributed import batch_particles

    motl = F.read_motive_list(cfg.MotiveList, cfg.ScaleMotivelistPosition, cfg.ScaleMotivelistShift)
    shifts = F.read_shift_file(cfg.ShiftInputFile)  # [projection][motive][2]
    n_proj = len(markers.tilt_angle)
    out = []
    for parts in batch_particles(motl.shape[0], max(1, cfg.BatchSize), rank, world):
        sub = []
        pair = (L.ProjGeom * (len(parts) * n_proj))()
        active = np.zeros((len(parts), n_proj), np.uint8)
        for k, p in enumerate(parts):
            m = motl[p]
            sub.append(E.subvolume_geometry(cfg.SizeSubVol, cfg.VoxelSizeSubVol, vg, m[7:10], m[10:13]))
            es = shifts[:, p, :]  # [projection][2]
            g = E.projection_geometry(markers, W, H, tc, extra_shift=es)
            for i in range(n_proj):
                pair[k * n_proj + i] = g[i]
            active[k] = np.sqrt((es.astype(np.float32) ** 2).sum(1)) < np.float32(cfg.MaxShift - 0.5)
        out.append(SubvolumeBatch(parts, sub, pair, active))
    return out


def reconstruct_subvolumes(cfg: EmSartConfig, write: bool = True, batched: bool = True,
                           variant: int = E.VARIANT_FAST, rank: int | None = None, world: int | None = None):
    """EmSartSubVolumes' run (EmSartSubVolumes.cpp:611-705): weighted
    back-projection of a SizeSubVol^3 box around every particle of the motive
    list, each projection shifted by the particle's extra shift from the
    shift file (tilts with |shift| >= MaxShift - 0.5 are left out), BatchSize
    particles per pass, every box written negated to
    SubVolPath + <particle index coding> + ".em". With several ranks (the
    arguments, or torch.distributed's) each batch is split over them as the
    reference's MPI run splits it; the projections are replicated and no
    collective is needed. Returns {file name: box} of this rank's
    particles."""
    import torch

    rank, world = _rank_world(rank, world)
    R = _setup(cfg, variant, rank)
    rec, vg, dev = R.rec, R.vg, R.dev
    motl = F.read_motive_list(cfg.MotiveList, cfg.ScaleMotivelistPosition, cfg.ScaleMotivelistShift)
    index_list = E.projection_index_list(E.PLT_NORMAL, R.tilt, R.good.astype(np.int32))
    S = cfg.SizeSubVol
    out = {}
    for b in subvolume_batches(cfg, R.markers, R.tc, vg, R.W, R.H, rank, world):
        boxes = [torch.zeros((S, S, S), dtype=torch.float32, device=dev) for _ in b.parts]
        rec.subvolume_wbp(vg, b.sub, b.pair, boxes, R.prepared, index_list, active=b.active, batched=batched)
        torch.cuda.synchronize()
        for k, p in enumerate(b.parts):
            name = cfg.SubVolPath + F.index_coding(motl[p], cfg.NamingConvention == 1) + ".em"
            box = _negated(boxes[k], dev)
            out[name] = box
            if write:
                F.write_em(name, box)
    rec.close()
    return out
