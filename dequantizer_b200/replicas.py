"""Instance-level replicas across ranks (one process per GPU).

The hot path has no exchange step inside one graph: independent instances
(e.g. a batch of annealing problems) are sharded across ranks and their
host-side results gathered at the end. Nothing here touches device memory of
another rank; the only collectives are on small host objects, over whatever
backend the process group uses (NCCL on GPUs, gloo on CPU).
"""

from typing import Any, Dict, List, Sequence

import torch.distributed as dist


def shard(n_items: int, world: int, rank: int) -> range:
    """Contiguous, balanced block of item indices owned by ``rank``."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad world / rank")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shard_weighted(costs: Sequence[float], world: int, rank: int) -> List[int]:
    """Greedy longest-processing-time assignment of items with uneven costs
    (e.g. instances of different node counts); deterministic on every rank."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0.0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda j: (load[j], j))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def gather_results(local: Dict[int, Any]) -> Dict[int, Any]:
    """Merges per-rank {item index: result} dicts on every rank."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return dict(local)
    parts: List[Dict[int, Any]] = [None] * dist.get_world_size()  # type: ignore[list-item]
    dist.all_gather_object(parts, local)
    merged: Dict[int, Any] = {}
    for p in parts:
        overlap = merged.keys() & p.keys()
        if overlap:
            raise RuntimeError(f"items {sorted(overlap)[:5]} reported by more than one rank")
        merged.update(p)
    return merged
