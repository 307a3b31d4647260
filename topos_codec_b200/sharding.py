"""Frame sharding across ranks (one process per GPU).

Frames are independent in the intra path, so ranks never exchange coded data:
each rank codes its own frames (seeded by rank), and the only collective is
the reduction of the measured times, where the slowest rank decides the
job's time.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def rank_frames(rank: int, frames_per_rank: int) -> List[Tuple[int, int]]:
    """(seed, frame index) of the frames a rank codes; disjoint across ranks."""
    return [(rank, i) for i in range(frames_per_rank)]


def max_over_ranks(values: Sequence[float], device=None) -> List[float]:
    """Element-wise maximum of per-rank measurements (identity on one rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()
