"""Spreading independent BA instances over several GPUs (replicas only).

One BA on one (n, k) fits one B200, so several GPUs run independent
instances (different (n, k) pairs and seeded starts), one process per GPU,
with no collective on the data path.  This module holds the host-side logic:
the assignment of instances to ranks (longest processing time first, by the
per-iteration work of the factored engine) and the merge of the per-rank
results.  The reference has no multi-GPU path (backend/main_BAA.cu runs one
(n, k) per process).
"""
from __future__ import annotations

from typing import Sequence


def instance_cost(n: int, k: int) -> float:
    """Relative per-iteration work of one instance: the dense half iterate
    (2^(n-1) entries) times the contraction width, which grows with the
    number of split terms (k + 1)."""
    return float(1 << (n - 1)) * (k + 1)


def partition(instances: Sequence[tuple[int, int]], world: int) -> list[list[int]]:
    """Indices of `instances` ((n, k) pairs) per rank: the costliest first,
    each to the least loaded rank (ties to the lowest rank), so that every
    rank gets a deterministic, disjoint share and the loads differ by at most
    one instance's cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(instances)), key=lambda i: (-instance_cost(*instances[i]), i))
    load = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += instance_cost(*instances[i])
    for share in out:
        share.sort()
    return out


def merge(per_rank: Sequence[Sequence[tuple[int, dict]]], count: int) -> list[dict]:
    """Per-instance results in instance order from the ranks' (index, result)
    lists; every index must appear exactly once."""
    out: list[dict | None] = [None] * count
    for share in per_rank:
        for i, res in share:
            if out[i] is not None:
                raise ValueError(f"instance {i} reported twice")
            out[i] = res
    missing = [i for i, r in enumerate(out) if r is None]
    if missing:
        raise ValueError(f"instances without a result: {missing}")
    return out  # type: ignore[return-value]


def gather(local: list[tuple[int, dict]], count: int, group=None) -> list[dict] | None:
    """Collects every rank's (index, result) list on rank 0 through
    torch.distributed (any backend) and merges them; other ranks get None."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    objs = [None] * world if dist.get_rank(group) == 0 else None
    dist.gather_object(local, objs, dst=0, group=group)
    if dist.get_rank(group) != 0:
        return None
    return merge(objs, count)
