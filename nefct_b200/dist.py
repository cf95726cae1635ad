"""View-sharded projection across ranks (one process per GPU).

The projector shards naturally by views: each rank projects its contiguous
block of views (no communication), and the transpose of a view-sharded
sinogram is the sum over ranks of each rank's partial volume -- one
all-reduce of the volume (NCCL over NVLink on GPUs; any torch.distributed
backend works, gloo on CPU).  Independent scans need no communication at
all (``bench.py --gpus N`` runs one scan per rank).
"""
from __future__ import annotations

from typing import Callable

import numpy as np
import torch
import torch.distributed as dist

from . import ops

__all__ = ["view_shard", "ShardedProjector"]


def view_shard(nv: int, rank: int, world: int) -> slice:
    """Contiguous, balanced block of views of ``rank`` (sizes differ by <= 1)."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(nv, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


class ShardedProjector:
    """Projector over the views of this rank.

    forward(vol)    -> this rank's sinogram block [nv_rank, nb, na]
    backward(sino)  -> the full transpose: local partial volume summed over
                       the process group (every rank gets the result)
    gather(sino)    -> the full sinogram on every rank (all-gather)

    ``forward_fn(vol, geom, flags)`` / ``backward_fn(sino, geom, flags)``
    default to the CUDA operators; any pair with the same contract works.
    """

    def __init__(self, geom: ops.ConeBeam, flags: int = 0, group=None,
                 forward_fn: Callable | None = None, backward_fn: Callable | None = None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.full = geom
        self.views = view_shard(geom.nv, self.rank, self.world)
        self.local = geom.subset(np.arange(geom.nv)[self.views])
        self.flags = flags
        self.forward_fn = forward_fn or ops.cb_forward
        self.backward_fn = backward_fn or ops.cb_backward

    def forward(self, vol: torch.Tensor) -> torch.Tensor:
        return self.forward_fn(vol, self.local, self.flags)

    def backward(self, sino_local: torch.Tensor) -> torch.Tensor:
        part = self.backward_fn(sino_local, self.local, self.flags)
        dist.all_reduce(part, op=dist.ReduceOp.SUM, group=self.group)
        return part

    def gather(self, sino_local: torch.Tensor) -> torch.Tensor:
        sizes = [view_shard(self.full.nv, r, self.world) for r in range(self.world)]
        nmax = max(s.stop - s.start for s in sizes)
        pad = torch.zeros((nmax,) + tuple(sino_local.shape[1:]), dtype=sino_local.dtype,
                          device=sino_local.device)
        pad[: sino_local.shape[0]] = sino_local
        bufs = [torch.empty_like(pad) for _ in range(self.world)]
        dist.all_gather(bufs, pad, group=self.group)
        return torch.cat([b[: s.stop - s.start] for b, s in zip(bufs, sizes)], 0)
