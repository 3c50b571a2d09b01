"""Sharding a batched ensemble over GPUs, one process per GPU.

The reference runs one system on one device and has no multi-device code.
Independent systems are the only unit that shards here: each rank takes a
share of the ensemble and advances it as one batched engine on its own GPU,
with no exchange during a stride.  Shares are balanced by the
longest-processing-time rule on a cost per system (the atom count: pairs, mesh
points and constraint units all grow in proportion), and per-system reports
come back to every rank with one host-side all-gather at the end.
"""

from __future__ import annotations

import heapq
from typing import Any, Sequence


def lpt_partition(costs: Sequence[float], parts: int) -> list[list[int]]:
    """Indices of `costs` in `parts` groups: largest first, each to the group
    with the least total so far (ties to the lowest group).  The largest group
    total is within 4/3 - 1/(3 parts) of the best possible split.  Each group
    lists its indices in ascending order, so every rank builds the same batch
    layout from the same ensemble."""
    if parts < 1:
        raise ValueError("parts must be at least 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, g) for g in range(parts)]
    groups: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        load, g = heapq.heappop(heap)
        groups[g].append(i)
        heapq.heappush(heap, (load + float(costs[i]), g))
    return [sorted(g) for g in groups]


def rank_share(costs: Sequence[float], rank: int, world: int) -> list[int]:
    """The ensemble indices rank `rank` of `world` advances."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return lpt_partition(costs, world)[rank]


def gather_by_system(local: dict[int, Any], world: int) -> dict[int, Any]:
    """Every rank's {system index: report} merged on every rank (one
    all-gather of host objects over the default process group; with one rank
    the reports come back as they are).  A system reported by two ranks is an
    error."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist

    parts: list[Any] = [None] * world
    dist.all_gather_object(parts, dict(local))
    merged: dict[int, Any] = {}
    for part in parts:
        for k, v in part.items():
            if k in merged:
                raise RuntimeError(f"system {k} reported by two ranks")
            merged[k] = v
    return merged
