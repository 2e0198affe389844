"""Query sharding across ranks (one process per GPU).

A query's hits depend only on that query and the library: masklevel, the hit order and the
E-values are all per query.  So whole queries shard across ranks with no exchange on the data
path.  Each rank searches a contiguous run of the queries, and the outfmt-6 text joins in query
order on rank 0.  That is one gather of text at the end, not a collective inside the search.
"""
from __future__ import annotations

from typing import Callable, Sequence


def shard_bounds(lengths: Sequence[int], world: int) -> list[tuple[int, int]]:
    """Contiguous [start, end) query ranges, one per rank, with about equal bases each (whole
    queries; a rank may get none when there are fewer queries than ranks)."""
    if world < 1:
        raise ValueError("world must be at least 1")
    n = len(lengths)
    total = sum(lengths)
    bounds, start, acc = [], 0, 0
    for r in range(world):
        if r == world - 1:
            end = n
        else:
            target = total * (r + 1) / world
            end = start
            while end < n and (acc + lengths[end] <= target or end == start):
                acc += lengths[end]
                end += 1
                if acc >= target:
                    break
        bounds.append((start, end))
        start = end
    return bounds


def search_sharded(search_text: Callable[[list, list], str], queries: list, ids: list, group=None) -> str | None:
    """Run `search_text(queries, ids) -> outfmt-6 text` on this rank's shard and return the whole
    text, in query order, on rank 0 (None elsewhere).  Without an initialised process group this
    is a single-rank search."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return search_text(queries, ids)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    b, e = shard_bounds([len(q) for q in queries], world)[rank]
    text = search_text(queries[b:e], ids[b:e]) if e > b else ""
    parts = [None] * world if rank == 0 else None
    dist.gather_object(text, parts, dst=0, group=group)
    return "".join(parts) if rank == 0 else None
