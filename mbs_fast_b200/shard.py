"""Orientation sharding across ranks (one process per GPU).

Orientations are independent units of the PO diffraction path: each rank
diffracts a contiguous range of them into its own Mueller accumulator, and the
only exchange is one sum of the accumulators at the end.  The ranges follow
the reference's multi-device split, begin = start + n*dev/N,
end = start + n*(dev+1)/N (src/cuda/GpuDiffraction.cu:4224-4226), so a batch
gives the same per-range work whether it runs on N devices of one process or
N ranks.
"""
from __future__ import annotations

import numpy as np


def orientation_range(n_orient: int, rank: int, world: int, start: int = 0) -> tuple[int, int]:
    """(begin, count) of this rank's contiguous orientation range."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} of {world}")
    if n_orient < 0:
        raise ValueError("negative orientation count")
    begin = start + (n_orient * rank) // world
    end = start + (n_orient * (rank + 1)) // world
    return begin, end - begin


def reduce_mueller(local, group=None):
    """Sum the ranks' Mueller accumulators in place (torch.distributed
    all-reduce; device tensors over NCCL, host tensors over gloo) and return
    the summed array.  numpy arrays are wrapped without copying."""
    import torch
    import torch.distributed as dist
    t = torch.from_numpy(local) if isinstance(local, np.ndarray) else local
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return local


def diffract_sharded(handler, batch, local_m: np.ndarray, local_m_noshadow=None,
                     precision: int = 0, rank: int = 0, world: int = 1, group=None) -> bool:
    """HandleOrientationsToLocalGpu over this rank's range of `batch`, then the
    all-rank sum into local_m (and local_m_noshadow).  Every rank takes the
    same collective steps whatever its range holds; a rank whose call fails
    still joins the reduction and the failure is agreed on by all ranks."""
    import torch
    import torch.distributed as dist
    begin, count = orientation_range(batch.n_orient, rank, world)
    part = np.zeros_like(local_m)
    part_ns = np.zeros_like(local_m_noshadow) if local_m_noshadow is not None else None
    ok = True
    if count > 0:
        ok = handler.handle_orientations_to_local_gpu(batch, part, part_ns, start=begin,
                                                      count=count, precision=precision)
    multi = dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1
    if multi:
        flag = torch.tensor([0 if ok else 1], dtype=torch.int32)
        dist.all_reduce(flag, op=dist.ReduceOp.MAX, group=group)
        ok = int(flag.item()) == 0
    reduce_mueller(part, group)
    if part_ns is not None:
        reduce_mueller(part_ns, group)
    if not ok:
        return False
    local_m += part
    if local_m_noshadow is not None:
        local_m_noshadow += part_ns
    return True
