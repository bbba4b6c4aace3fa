"""Independent KKT systems spread over GPUs, one process per GPU.

The batched workloads (many optimal-control systems, or one system per
sample in differentiation) have no coupling between systems. So they shard
by system with no exchange on the data path. Every rank factors and solves
its own share in one batch handle on its own GPU. The per-system results
(inertia, backward errors) are gathered on the host at the end. The
reference factors such systems one after another, each with its own
SparseLDL (include/sparse_ldl.h:65-118).

The partition is deterministic, so every rank computes the same one
without communicating. Systems go to ranks largest first, each to the rank
with the least work so far (ties to the lower rank). Each rank then keeps
its systems in their original order.
"""

from __future__ import annotations

from typing import Callable, Sequence

__all__ = ["partition_systems", "shard_systems", "gather_by_system"]


def partition_systems(costs: Sequence[float], world: int) -> list[list[int]]:
    """Indices of the systems of each of ``world`` ranks, balanced by cost
    (e.g. factorization flops, or the size for chain-structured systems).
    The largest share exceeds the smallest by at most the largest cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    loads = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    for i in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        parts[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(p) for p in parts]


def shard_systems(systems: Sequence, rank: int, world: int,
                  cost: Callable[[object], float] = lambda q: q.n):
    """This rank's (indices, systems) under :func:`partition_systems`."""
    idx = partition_systems([cost(q) for q in systems], world)[rank]
    return idx, [systems[i] for i in idx]


def gather_by_system(local_items: Sequence, local_indices: Sequence[int], num_systems: int,
                     group=None) -> list:
    """Every rank's per-system items, in the original system order, on every
    rank (host objects through torch.distributed.all_gather_object; with
    one process, the local items)."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        pairs = [(list(local_indices), list(local_items))]
    else:
        pairs = [None] * dist.get_world_size(group)
        dist.all_gather_object(pairs, (list(local_indices), list(local_items)), group=group)
    missing = object()
    out = [missing] * num_systems
    seen = 0
    for idx, items in pairs:
        if len(idx) != len(items):
            raise ValueError("each index needs one item")
        for i, it in zip(idx, items):
            if out[i] is not missing:
                raise ValueError(f"system {i} reported by two ranks")
            out[i] = it
            seen += 1
    if seen != num_systems:
        raise ValueError(f"{num_systems - seen} systems missing from the gather")
    return out
