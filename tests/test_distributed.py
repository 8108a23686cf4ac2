"""Multi-process paths: z-slab SART with a per-projection all-reduce, and
particle sharding of the sub-volume reconstruction.

World size 2 over gloo on 127.0.0.1. The CPU tests run the driver of
artiatomi_b200.distributed on the oracle (one slab per process) and check it
against the same decomposition emulated in one process, bit for bit (the
all-reduce of two float images is one float addition per pixel). The GPU
test runs two processes on the one GPU with gloo (host-side reduction: no
kernel waits on another process) and checks them against the same
decomposition run in one process on the GPU.
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


def _oracle_slab(case, part, count):
    from oracle import geometry as G
    from oracle.driver import OracleReconstructor

    vo = G.volume_geometry(DIMS, count=count, part=part)
    vol = np.zeros((int(vo.dim[2]), DIMS[1], DIMS[0]), np.float32)
    orc = OracleReconstructor(CFG, W, H, case["og"], case["tilt"])
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
    from artiatomi_b200.distributed import shard_particles

    for n, world in ((7, 2), (10, 3), (1, 4)):
        parts = [shard_particles(n, r, world) for r in range(world)]
        flat = sorted(p for ps in parts for p in ps)
        assert flat == list(range(n))


def _worker_gpu(rank, world, port, outdir):
    import torch
    import torch.distributed as dist

    import artiatomi_b200 as E
    from artiatomi_b200.distributed import GpuSlab, ZSlabSart

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = _case()
        projs = torch.from_numpy(_projections(case)).cuda()
        il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
        vg = E.volume_geometry(DIMS, subvol_count=world, subvol=rank)
        vol = torch.zeros((int(vg.dim[2]), DIMS[1], DIMS[0]), device="cuda")
        rec = E.Reconstructor(E.ReconConfig(W, H, N_PROJ, variant=E.VARIANT_FAST, **CFG), case["pg"], case["tilt"])
        ZSlabSart(GpuSlab(rec, vg, vol)).run(projs, il, iterations=2, sirt_count=2)
        np.save(os.path.join(outdir, f"slab{rank}.npy"), vol.cpu().numpy())
        rec.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_zslab_sart_two_ranks_on_gpu():
    import torch
    import torch.multiprocessing as mp

    import artiatomi_b200 as E
    from artiatomi_b200.distributed import GpuSlab

    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker_gpu, args=(2, _free_port(), d), nprocs=2, join=True)
        got = [np.load(os.path.join(d, f"slab{r}.npy")) for r in range(2)]
    case = _case()
    projs = torch.from_numpy(_projections(case)).cuda()
    il = E.projection_index_list(E.PLT_RANDOM_START_ZERO_TILT, case["tilt"])
    slabs = []
    for r in range(2):
        vg = E.volume_geometry(DIMS, subvol_count=2, subvol=r)
        vol = torch.zeros((int(vg.dim[2]), DIMS[1], DIMS[0]), device="cuda")
        rec = E.Reconstructor(E.ReconConfig(W, H, N_PROJ, variant=E.VARIANT_FAST, **CFG), case["pg"], case["tilt"])
        slabs.append(GpuSlab(rec, vg, vol))
    _emulate(slabs, projs, il, 2, 2)
    torch.cuda.synchronize()
    for r in range(2):
        np.testing.assert_array_equal(got[r], slabs[r].vol.cpu().numpy())
    # and the oracle's decomposition, at the fast-kernel SART tolerance
    oslabs = [_oracle_slab(case, r, 2) for r in range(2)]
    _emulate(oslabs, projs.cpu().numpy(), il, 2, 2)
    for r in range(2):
        assert rel_l2(got[r], oslabs[r].vol) <= 1e-3
