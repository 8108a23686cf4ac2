"""Multi-process reconstruction: z-slab SART and particle-sharded sub-volumes.

One process per GPU with torch.distributed for the plumbing.

* ``Reconstructor.sart_zslab`` with ``torch_allreduce``: the reference's MPI
  scheme for one tomogram larger than one GPU (Volume(dim, count, part),
  Volume.cpp:82-114; EmSart.cpp:579-675 with the projections summed over
  ranks) inside the library (esb_sart_run_zslab): one all-reduce of the
  slab's projection and ray lengths per projection, on the reconstructor's
  stream. ``ZSlabSart`` is the same loop in Python over an adapter, which
  runs it on the CPU oracle in the tests. Rank r holds z-slab r of the volume.
  For every projection each rank forward-projects its slab (line integrals
  and ray lengths through the slab), the projection and the ray-length image
  are summed over ranks with one all-reduce, every rank forms the same
  residual and back-projects it into its own slab. With CTF the slab images
  of each rank are filtered before the sum, which is the same as filtering
  the sum: the filter is linear.
* ``batch_particles``: EmSartSubVolumes' particles split over ranks
  (EmSartSubVolumes.cpp:611-668), used by reconstruct.reconstruct_subvolumes;
  the projections are replicated and no collective is needed.

The driver talks to a reconstructor through a small adapter, so the same
loop runs on the GPU library (``GpuSlab``) and, for tests without a GPU, on
the CPU oracle (in tests only).
"""
from __future__ import annotations

from typing import Sequence


class GpuSlab:
    """Adapter over ``emsart.Reconstructor`` for one rank's slab."""

    def __init__(self, rec, vg, vol):
        self.rec, self.vg, self.vol = rec, vg, vol
        self.proj, self.dist, _ = rec.views()

    def reset(self):
        self.rec.reset_projections()

    def forward(self, index: int, volume_is_empty: bool):
        self.rec.forward_projection(self.vg, self.vol, index, volume_is_empty)

    def compare(self, real, index: int):
        self.rec.compare(self.vg, real, index)

    def residual(self):
        return self.proj.clone()

    def back_project(self, index: int, sirt_count: int, residual):
        self.proj.copy_(residual)
        self.rec.back_projection(self.vg, self.vol, index, float(sirt_count))

    def synchronize(self):
        import torch

        torch.cuda.synchronize()


class ZSlabSart:
    """SART over the z-slabs of one volume, one slab per rank."""

    def __init__(self, slab, group=None):
        self.slab = slab
        self.group = group

    def _allreduce(self, t):
        import torch.distributed as dist

        if dist.is_initialized() and dist.get_world_size(self.group) > 1:
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)

    def run(self, projections: Sequence, index_list: Sequence[int], iterations: int, sirt_count: int,
            volume_is_empty: bool = True) -> bool:
        """EmSart.cpp:579-675 on this rank's slab; every rank calls it with the
        same arguments (the collectives are matched in order). Returns the
        updated volume_is_empty flag."""
        n = len(index_list)
        steps = (n + sirt_count - 1) // sirt_count
        S = self.slab
        for _ in range(iterations):
            for s in range(steps):
                residuals = {}
                for i in range(sirt_count):
                    if s * sirt_count + i >= n:
                        continue
                    index = int(index_list[s * sirt_count + i])
                    S.reset()
                    S.forward(index, volume_is_empty)
                    S.synchronize()
                    self._allreduce(S.proj)
                    self._allreduce(S.dist)
                    S.compare(projections[index], index)
                    residuals[i] = S.residual()
                for i in range(sirt_count):
                    if s * sirt_count + i >= n:
                        continue
                    volume_is_empty = False
                    index = int(index_list[s * sirt_count + i])
                    S.back_project(index, sirt_count, residuals[i])
        S.synchronize()
        return volume_is_empty


def torch_allreduce(group=None):
    """The all-reduce callback of Reconstructor.sart_zslab over
    torch.distributed: the sum is enqueued on the reconstructor's stream
    (NCCL: no host synchronisation; gloo reduces CUDA tensors through the
    host)."""

    def allreduce(buf, stream):
        import torch
        import torch.distributed as dist

        if not dist.is_initialized() or dist.get_world_size(group) == 1:
            return
        with torch.cuda.stream(stream):
            dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)

    return allreduce


def batch_particles(n_particles: int, batch_size: int, rank: int, world: int) -> list[list[int]]:
    """This rank's particles, batch by batch (EmSartSubVolumes.cpp:611-668):
    the motive list in batches of batch_size; in each batch rank r takes
    batch + r, batch + r + world, ... With batch_size a multiple of world
    this is the reference's split exactly. Otherwise the reference's
    index batch + pInBatch + rank runs past the batch end into the next batch
    (and past its per-batch box array), so those particles would be done
    twice; here every rank stops at its batch's end and each particle is
    reconstructed once."""
    if batch_size < 1 or world < 1 or not 0 <= rank < world:
        raise ValueError("batch_particles: invalid batch size, rank or world size")
    out = []
    for b0 in range(0, n_particles, batch_size):
        end = min(b0 + batch_size, n_particles)
        out.append(list(range(b0 + rank, end, world)))
    return out


def shard_particles(n_particles: int, rank: int, world: int) -> list[int]:
    """All particles of this rank (batch_particles with one batch)."""
    return batch_particles(n_particles, max(1, n_particles), rank, world)[0] if n_particles else []
