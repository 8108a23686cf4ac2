"""Multi-process paths: z-slab SART with a per-projection all-reduce, and
particle sharding of the sub-volume reconstruction.

World size 2 over gloo on 127.0.0.1. The CPU tests run the driver of
artiatomi_b200.distributed on the oracle (one slab per process) and check it
against the same decomposition emulated in one process, bit for bit (the
all-reduce of two float images is one float addition per pixel), and run
the particle split of reconstruct.subvolume_batches on two ranks, each
back-projecting its particles on the oracle, against the one-rank run. The
GPU test runs the library's z-slab SART (Reconstructor.sart_zslab, the C
entry esb_sart_run_zslab with a torch.distributed all-reduce callback) in two
processes on the one GPU with gloo (host-side reduction: no kernel waits on
another process) and checks them against the same decomposition run in one
process on the GPU.
"""
import os
import socket
import tempfile

import numpy as np
import pytest

from tests.helpers import rel_l2, small_case

DIMS, N_PROJ, W, H = (48, 40, 20), 5, 48, 48
CFG = dict(lambda_=0.5, oversampling=2)


def _case():
    return small_case(dims=DIMS, n_proj=N_PROJ, W=W, H=H, seed=21, n_ell=10, shift=1.0, psi=0.2)


def _projections(case):
    from tests.test_parity_recon import _projections as P

    return P(case)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleSlab:
    """The driver's slab adapter over the CPU oracle (tests only)."""

    def __init__(self, orc, vo, vol):
        import torch

        self.orc, self.vo, self.vol = orc, vo, vol
        self.proj = torch.from_numpy(orc.proj)
        self.dist = torch.from_numpy(orc.dist)

    def reset(self):
        self.orc.reset()

    def forward(self, index, volume_is_empty):
        self.orc.forward_projection(self.vo, self.vol, 0, index, volume_is_empty)

    def compare(self, real, index):
        self.orc.compare(self.vo, real, index)

    def residual(self):
        return self.orc.proj.copy()

    def back_project(self, index, sirt_count, residual):
        self.orc.back_projection(self.vo, self.vol, 0, index, float(sirt_count), img=residual)

    def synchronize(self):
        pass


def _ctf_setup(ctf):
    """(reconstructor config, defocus table) of the case, with or without
    3-D CTF (2.5 nm slabs: several per slab of the volume)."""
    if not ctf:
        return dict(CFG), None
    from tests.test_parity_fast import _defocus
    from tests.test_parity_recon import _ctf_cfg

    return dict(_ctf_cfg(W), **CFG), _defocus(N_PROJ, 15)


def _oracle_slab(case, part, count, ctf=False):
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    cfgd, defocus = _ctf_setup(ctf)
    vo = G.volume_geometry(DIMS, count=count, part=part)
    vol = np.zeros((int(vo.dim[2]), DIMS[1], DIMS[0]), np.float32)
    orc = OracleReconstructor(cfgd, W, H, case["og"], case["tilt"], defocus)
    return OracleSlab(orc, vo, vol)


def _emulate(slabs, projections, il, iterations, sirt):
    """The z-slab loop with the all-reduce done in-process (float32 sums)."""
    n = len(il)
    empty = True
    for _ in range(iterations):
        for s in range((n + sirt - 1) // sirt):
            res = {}
            for i in range(sirt):
                if s * sirt + i >= n:
                    continue
                index = int(il[s * sirt + i])
                for S in slabs:
                    S.reset()
                    S.forward(index, empty)
                for S in slabs:
                    S.synchronize()
                for name in ("proj", "dist"):
                    tot = getattr(slabs[0], name).clone()
                    for S in slabs[1:]:
                        tot = tot + getattr(S, name)
                    for S in slabs:
                        getattr(S, name).copy_(tot)
                for S in slabs:
                    S.compare(projections[index], index)
                res[i] = [S.residual() for S in slabs]
            for i in range(sirt):
                if s * sirt + i >= n:
                    continue
                empty = False
                index = int(il[s * sirt + i])
                for k, S in enumerate(slabs):
                    S.back_project(index, sirt, res[i][k])


def _worker_oracle(rank, world, port, outdir):
    import torch.distributed as dist

    import artiatomi_b200 as E
    from artiatomi_b200.distributed import ZSlabSart

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = _case()
        projs = _projections(case)
        il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
        S = _oracle_slab(case, rank, world)
        ZSlabSart(S).run(projs, il, iterations=2, sirt_count=2)
        np.save(os.path.join(outdir, f"slab{rank}.npy"), S.vol)
    finally:
        dist.destroy_process_group()


def test_zslab_sart_two_ranks_matches_emulation():
    import torch.multiprocessing as mp

    import artiatomi_b200 as E

    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker_oracle, args=(2, _free_port(), d), nprocs=2, join=True)
        got = [np.load(os.path.join(d, f"slab{r}.npy")) for r in range(2)]
    case = _case()
    projs = _projections(case)
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    slabs = [_oracle_slab(case, r, 2) for r in range(2)]
    _emulate(slabs, projs, il, 2, 2)
    for r in range(2):
        assert np.abs(slabs[r].vol).max() > 0
        np.testing.assert_array_equal(got[r], slabs[r].vol)
    # against the undivided volume: the slabs only differ where the
    # interpolation crosses the slab boundary (each slab clamps at its own
    # faces, as in the reference's MPI runs); 1.4e-3 on this case
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    orc = OracleReconstructor(CFG, W, H, case["og"], case["tilt"])
    full = np.zeros(case["vol"].shape, np.float32)
    orc.sart(G.volume_geometry(DIMS), full, 0, projs, il, 2, 2)
    assert rel_l2(np.concatenate(got, 0), full) <= 5e-3


def test_particle_shards_cover_every_particle_once():
    from artiatomi_b200.distributed import batch_particles, shard_particles

    for n, world in ((7, 2), (10, 3), (1, 4), (0, 2)):
        parts = [shard_particles(n, r, world) for r in range(world)]
        flat = sorted(p for ps in parts for p in ps)
        assert flat == list(range(n))
    for n, batch, world in ((11, 4, 2), (9, 6, 3), (5, 3, 2), (3, 8, 4), (6, 1, 1)):
        per_rank = [batch_particles(n, batch, r, world) for r in range(world)]
        assert all(len(b) == (n + batch - 1) // batch for b in per_rank)
        flat = sorted(p for b in per_rank for ps in b for p in ps)
        assert flat == list(range(n))
        for r in range(world):
            for k, ps in enumerate(per_rank[r]):
                b0 = k * batch
                assert all(b0 <= p < b0 + batch for p in ps)
                if batch % world == 0:
                    # the reference's motlIdx = batch + pInBatch + mpi_part
                    ref = [b0 + q + r for q in range(0, batch, world) if b0 + q + r < n]
                    assert ps == ref
    with pytest.raises(ValueError):
        batch_particles(4, 2, 2, 2)


# -- particle-sharded sub-volumes -------------------------------------------

SUB_N, SUB_S = 7, 12


def _write_subvolume_dataset(d):
    """tilt series, markers, motive list, shift file and config of a small
    EmSartSubVolumes run; returns the oracle-prepared projections."""
    from pathlib import Path

    from tests.test_reconstruct import H as RH
    from tests.test_reconstruct import N as NP
    from tests.test_reconstruct import W as RW
    from tests.test_reconstruct import _dataset
    from artiatomi_b200 import fileio as F
    from artiatomi_b200.config import EmSartConfig
    from oracle.driver import prepare_projection

    d = Path(d)
    raw, tilt, psi, og, vo = _dataset(d, wbp=True)
    rng = np.random.default_rng(13)
    motl = np.zeros((SUB_N, 20), np.float32)
    motl[:, 3] = np.arange(1, SUB_N + 1)
    motl[:, 7:10] = np.stack([rng.uniform(18, 46, SUB_N), rng.uniform(18, 46, SUB_N), rng.uniform(8, 16, SUB_N)], 1)
    motl[:, 10:13] = rng.uniform(-1, 1, (SUB_N, 3))
    F.write_motive_list(str(d / "motl.em"), motl)
    F.write_shift_file(str(d / "shifts.em"), rng.uniform(-1.8, 1.8, (2, NP, SUB_N)).astype(np.float32))
    (d / "sub").mkdir(exist_ok=True)
    text = (d / "emsart.cfg").read_text() + f"""SizeSubVol = {SUB_S}
VoxelSizeSubVol = 1
MotiveList = {d / 'motl.em'}
SubVolPath = {d / 'sub'}/
ShiftInputFile = {d / 'shifts.em'}
BatchSize = 4
MaxShift = 2
ScaleMotivelistShift = 1
ScaleMotivelistPosition = 1
"""
    (d / "emsart_sub.cfg").write_text(text)
    cfg = EmSartConfig.from_text(text, subvolumes=True)
    pc = dict(wbp=1, normalization=cfg.ProjectionNormalization, correct_bad_pixels=1,
              bad_pixel_value=cfg.BadPixelValue, skip_filter=int(cfg.SkipFilter), lp=float(cfg.fourFilterLP),
              hp=float(cfg.fourFilterHP), lps=float(cfg.fourFilterLPS), hps=float(cfg.fourFilterHPS),
              wbp_filter=cfg.WBPFilter)
    prepared = np.stack([prepare_projection(raw[i], max(RW, RH), dict(pc, tilt_deg=float(tilt[i]),
                                                                      psi_deg=float(psi[i])))[0]
                         for i in range(NP)])
    np.save(d / "prepared.npy", prepared)


def _oracle_vg(v):
    from oracle import geometry as G

    a = lambda x: np.asarray(list(x), np.float32)  # noqa: E731
    return G.VolGeom(a(v.bbox_min), a(v.bbox_max), a(v.bbox_rcp), a(v.dim), a(v.voxel_size), float(v.z_shift),
                     a(v.full_dim), a(v.full_bbox_min), a(v.full_bbox_max))


def _subvolumes_on_oracle(d, rank, world):
    """reconstruct_subvolumes' batches for this rank, each particle box
    back-projected by the oracle from the library's own geometry."""
    from pathlib import Path

    import artiatomi_b200 as E
    from artiatomi_b200 import fileio as F
    from artiatomi_b200.config import EmSartConfig
    from artiatomi_b200.reconstruct import _rank_world, subvolume_batches
    from oracle.driver import OracleReconstructor
    from tests.test_reconstruct import H as RH
    from tests.test_reconstruct import W as RW

    d = Path(d)
    rank, world = _rank_world(rank, world)
    cfg = EmSartConfig.from_text((d / "emsart_sub.cfg").read_text(), subvolumes=True)
    md = F.read_markers(cfg.MarkerFile, cfg.ReferenceMarker)
    markers = md.markers()
    tc = E.TiltConfig(cfg.AddTiltAngle, cfg.AddTiltXAngle, cfg.UseFixPsiAngle, cfg.PsiAngle, cfg.PhiAngle)
    vg = E.volume_geometry(cfg.RecDimensions, cfg.VoxelSize, cfg.VolumeShift)
    n_proj = len(markers.tilt_angle)
    prepared = np.load(d / "prepared.npy")
    orc = OracleReconstructor(dict(lambda_=cfg.Lambda, oversampling=cfg.OverSampling, cut_length=cfg.CutLength,
                                   dim_length=cfg.DimLength), RW, RH, None, markers.tilt_angle, precision=1)
    il = E.projection_index_list(E.PLT_NORMAL, markers.tilt_angle)
    boxes, batches = {}, []
    for b in subvolume_batches(cfg, markers, tc, vg, RW, RH, rank, world):
        batches.append(list(b.parts))
        pair = [[{"det": list(g.detektor), "u": list(g.u_pitch), "v": list(g.v_pitch), "n": list(g.proj_norm),
                  "detMat": list(g.detector_matrix)} for g in b.pair[k * n_proj:(k + 1) * n_proj]]
                for k in range(len(b.parts))]
        bo = [np.zeros((SUB_S,) * 3, np.float32) for _ in b.parts]
        orc.subvolume_wbp(_oracle_vg(vg), [_oracle_vg(v) for v in b.sub], pair, bo, prepared, il, active=b.active)
        for k, p in enumerate(b.parts):
            boxes[p] = bo[k]
    return boxes, batches


def _worker_subvolumes(rank, world, port, d):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        boxes, batches = _subvolumes_on_oracle(d, None, None)  # rank and world from torch.distributed
        np.savez(os.path.join(d, f"boxes{rank}.npz"), batches=np.array(repr(batches)),
                 **{f"p{p}": b for p, b in boxes.items()})
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_reconstruct_subvolumes_particle_sharding_two_ranks():
    import torch.multiprocessing as mp

    with tempfile.TemporaryDirectory() as d:
        _write_subvolume_dataset(d)
        mp.spawn(_worker_subvolumes, args=(2, _free_port(), d), nprocs=2, join=True)
        got = [np.load(os.path.join(d, f"boxes{r}.npz")) for r in range(2)]
        single, single_batches = _subvolumes_on_oracle(d, 0, 1)
    # BatchSize 4 over 2 ranks: the reference's split within each batch
    assert eval(str(got[0]["batches"])) == [[0, 2], [4, 6]]
    assert eval(str(got[1]["batches"])) == [[1, 3], [5]]
    assert single_batches == [[0, 1, 2, 3], [4, 5, 6]]
    seen = []
    for g in got:
        for key in g.files:
            if key == "batches":
                continue
            p = int(key[1:])
            seen.append(p)
            assert np.abs(single[p]).max() > 0
            np.testing.assert_array_equal(g[key], single[p])
    assert sorted(seen) == list(range(SUB_N))


def _worker_gpu(rank, world, port, outdir, ctf):
    import torch
    import torch.distributed as dist

    import artiatomi_b200 as E
    from artiatomi_b200.distributed import torch_allreduce

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = _case()
        projs = torch.from_numpy(_projections(case)).cuda()
        il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
        vg = E.volume_geometry(DIMS, subvol_count=world, subvol=rank)
        vol = torch.zeros((int(vg.dim[2]), DIMS[1], DIMS[0]), device="cuda")
        cfgd, defocus = _ctf_setup(ctf)
        rec = E.Reconstructor(E.ReconConfig(W, H, N_PROJ, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"],
                              defocus)
        empty = rec.sart_zslab(vg, vol, projs, il, 2, 2, torch_allreduce())
        assert not empty
        torch.cuda.synchronize()
        np.save(os.path.join(outdir, f"slab{rank}.npy"), vol.cpu().numpy())
        rec.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("ctf", [False, True])
def test_zslab_sart_two_ranks_on_gpu(ctf):
    """esb_sart_run_zslab in two processes (one slab each, the all-reduce
    over gloo) equals the decomposition run in one process; with CTF each
    rank filters its own slab images before the sum."""
    import torch
    import torch.multiprocessing as mp

    import artiatomi_b200 as E
    from artiatomi_b200.distributed import GpuSlab

    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker_gpu, args=(2, _free_port(), d, ctf), nprocs=2, join=True)
        got = [np.load(os.path.join(d, f"slab{r}.npy")) for r in range(2)]
    case = _case()
    projs = torch.from_numpy(_projections(case)).cuda()
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    slabs = []
    for r in range(2):
        vg = E.volume_geometry(DIMS, subvol_count=2, subvol=r)
        vol = torch.zeros((int(vg.dim[2]), DIMS[1], DIMS[0]), device="cuda")
        cfgd, defocus = _ctf_setup(ctf)
        rec = E.Reconstructor(E.ReconConfig(W, H, N_PROJ, variant=E.VARIANT_FAST, **cfgd), case["pg"], case["tilt"],
                              defocus)
        slabs.append(GpuSlab(rec, vg, vol))
    _emulate(slabs, projs, il, 2, 2)
    torch.cuda.synchronize()
    for r in range(2):
        np.testing.assert_array_equal(got[r], slabs[r].vol.cpu().numpy())
    # and the oracle's decomposition, at the fast-kernel SART tolerance
    oslabs = [_oracle_slab(case, r, 2, ctf) for r in range(2)]
    _emulate(oslabs, projs.cpu().numpy(), il, 2, 2)
    for r in range(2):
        assert rel_l2(got[r], oslabs[r].vol) <= 1e-3
