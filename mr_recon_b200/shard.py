"""Data-parallel plumbing for one process per GPU.

The NUFFT / CG-SENSE path shards by problem: slices of an uneven batch (and
replicas of a problem) are independent, so ranks exchange nothing on the
data path (the reference has no multi-GPU path). What ranks do share is
bookkeeping: which slices each rank solves, and the job time, which is the
maximum of the ranks' device times.
"""

from __future__ import annotations

from typing import List, Sequence, Tuple

import torch

__all__ = ["shard_slices", "max_over_ranks", "gather_slices"]


def shard_slices(costs: Sequence[float], world: int, rank: int) -> Tuple[int, int]:
    """Contiguous slice range [begin, end) of ``rank`` out of ``world`` that
    balances the summed cost (e.g. coils x samples per slice): rank r takes
    the slices whose cumulative cost midpoint falls in [r, r+1) * total/world.
    Every slice goes to exactly one rank; ranks may get none when there are
    fewer slices than ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    n = len(costs)
    total = float(sum(costs))
    if n == 0:
        return 0, 0
    if total <= 0.0:
        b = n * rank // world
        return b, n * (rank + 1) // world
    owner: List[int] = []
    acc = 0.0
    for c in costs:
        mid = acc + 0.5 * float(c)
        owner.append(min(world - 1, int(mid * world / total)))
        acc += float(c)
    begin = next((i for i, o in enumerate(owner) if o >= rank), n)
    end = next((i for i, o in enumerate(owner) if o > rank), n)
    return begin, end


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar over the default process group (the
    value itself without one). Used for job times: the slowest rank sets it."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    backend = dist.get_backend()
    dev = device if device is not None else (torch.device("cuda") if backend == "nccl" else torch.device("cpu"))
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_slices(local: Sequence[torch.Tensor], begin: int, end: int, n_total: int) -> List[torch.Tensor]:
    """The per-slice results of every rank, in slice order, on every rank.
    ``local`` holds this rank's results for slices [begin, end) (tensors of
    any shape, one per slice). Without a process group it returns ``local``.
    The exchange is a host-side all_gather of objects: bookkeeping after a
    solve, not part of the data path."""
    import torch.distributed as dist
    if len(local) != end - begin:
        raise ValueError("one result per local slice is needed")
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(local)
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (int(begin), [t.detach().cpu() for t in local]))
    out: List = [None] * n_total
    for b, ts in parts:
        for i, t in enumerate(ts):
            out[b + i] = t
    if any(t is None for t in out):
        raise RuntimeError("the ranks' slice ranges do not cover the batch")
    return out
