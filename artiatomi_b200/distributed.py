"""Multi-process reconstruction: z-slab SART and particle-sharded sub-volumes.

One process per GPU with torch.distributed for the plumbing.

* ``ZSlabSart``: the reference's MPI scheme for one tomogram larger than one
  GPU (Volume(dim, count, part), Volume.cpp:82-114; EmSart.cpp:579-675 with
  the projections summed over ranks). Rank r holds z-slab r of the volume.
  For every projection each rank forward-projects its slab (line integrals
  and ray lengths through the slab), the projection and the ray-length image
  are summed over ranks with one all-reduce, every rank forms the same
  residual and back-projects it into its own slab. With CTF the slab images
  of each rank are filtered before the sum, which is the same as filtering
  the sum: the filter is linear.
* ``shard_particles``: EmSartSubVolumes' particles split over ranks
  (EmSartSubVolumes.cpp:614-668); the projections are replicated and no
  collective is needed.

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


def shard_particles(n_particles: int, rank: int, world: int) -> list[int]:
    """Particles of this rank: round-robin over ranks, as the reference
    splits each batch (EmSartSubVolumes.cpp:614-668)."""
    return [p for p in range(n_particles) if p % world == rank]
