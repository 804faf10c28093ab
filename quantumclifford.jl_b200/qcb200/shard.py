"""Shot sharding across ranks (one process per GPU).

Frame sampling shards by shots with no collective in the sampling itself:
rank r runs the whole circuit on its own shot range starting at
``shard_offset(r, shots_per_rank)``, a multiple of 1024 (the Philox noise
counters use the global 1024-shot group and 32-shot column, so the union of
the shards is one run over all the shots).  ``gather_record_planes`` puts the
shards' record planes back together on every rank (an all-gather, only when
the caller wants the whole record), ``max_over_ranks`` gives the job's time
as the slowest rank's.
"""
from __future__ import annotations

import numpy as np

SHOT_GROUP = 1024


def shard_offset(rank: int, shots_per_rank: int) -> int:
    """First shot of rank `rank` when every rank runs `shots_per_rank` shots."""
    return rank * ((shots_per_rank + SHOT_GROUP - 1) // SHOT_GROUP * SHOT_GROUP)


def gather_record_planes(planes: np.ndarray, shots_per_rank: int, group=None) -> np.ndarray:
    """All-gather the ranks' record planes (uint32 [nbits, ceil(shots/32)] each)
    into the planes of the whole run, in rank order.  Ranks must run the same
    number of shots; shard offsets are multiples of 1024, so rank r's words
    start at word r * ceil(shots/1024) * 32 of the whole record."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    t = torch.from_numpy(np.ascontiguousarray(planes).view(np.int32))
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    stride = shard_offset(1, shots_per_rank) // 32
    nbits, words = planes.shape
    out = np.zeros((nbits, stride * (world - 1) + words), dtype=np.uint32)
    for r, p in enumerate(parts):
        out[:, r * stride:r * stride + words] = p.numpy().view(np.uint32)
    return out


def max_over_ranks(values, group=None, device=None):
    """Element-wise maximum of a list of floats over the ranks."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return [float(x) for x in t.cpu()]
