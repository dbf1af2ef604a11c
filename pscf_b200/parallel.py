"""Instance-parallel execution over ranks (one process per GPU).

SCFT instances (sweep points, candidate phases, Jacobian columns) are
independent, so a job is split into contiguous shards, one per rank, with
no collective on the data path; only the per-instance scalar results are
gathered at the end (all_gather_object over the process group: NCCL on
GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple


def shard(n: int, rank: int, world: int) -> Tuple[int, int]:
    """[begin, end) of rank's contiguous share of n items (sizes differ by <= 1)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    q, r = divmod(n, world)
    begin = rank * q + min(rank, r)
    return begin, begin + q + (1 if rank < r else 0)


def solve_sharded(items: Sequence, solve: Callable[[Sequence], List[dict]], group=None) -> List[dict]:
    """Run `solve` on this rank's shard of `items` and return every rank's
    results in the global order (list of per-instance dicts)."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    b, e = shard(len(items), rank, world)
    mine = solve(items[b:e]) if e > b else []
    if world == 1:
        return list(mine)
    gathered: List[List[dict]] = [None] * world  # type: ignore
    dist.all_gather_object(gathered, list(mine), group=group)
    out: List[dict] = []
    for part in gathered:
        out.extend(part)
    return out
