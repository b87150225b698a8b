"""Replica sharding of the batched forms across the ranks of a job (one process per GPU).

Independent systems and independent right-hand-side columns need no communication: each rank
takes its share, solves it on its own GPU with its own hierarchies, and only the timing (and,
when asked, the results) meet on rank 0. The reference has no batched form; its one data-parallel
split is the row partition of a single system (BCMGX/src/utility/distribuite.cu).

* systems_of_rank(nsys, rank, world): systems k = rank, rank + world, ... (round robin, so that
  uneven system sizes spread evenly);
* columns_of_rank(k, rank, world): a contiguous slice of the k right-hand-side columns (the
  first k % world ranks take one more), so that each rank's block keeps the column order;
* gather_in_order(local, index, total, world): every rank's (index, item) pairs gathered on all
  ranks and put back into single-rank order.
"""
from __future__ import annotations


def systems_of_rank(nsys: int, rank: int, world: int) -> list[int]:
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return list(range(rank, nsys, world))


def columns_of_rank(k: int, rank: int, world: int) -> range:
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(k, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def gather_in_order(local, index, total: int, world: int):
    """local[i] is the item of global index index[i]; returns the list of all `total` items in
    global order on every rank (torch.distributed all_gather_object; any backend)."""
    if len(local) != len(index):
        raise ValueError("one index per item")
    if world <= 1:
        out = [None] * total
        for i, it in zip(index, local):
            out[i] = it
        return out
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, list(zip(index, local)))
    out = [None] * total
    seen = 0
    for part in parts:
        for i, it in part:
            if out[i] is not None:
                raise RuntimeError(f"item {i} came from two ranks")
            out[i] = it
            seen += 1
    if seen != total:
        raise RuntimeError(f"{total - seen} items missing after the gather")
    return out
