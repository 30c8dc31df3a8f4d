"""Replica sharding across GPUs (one process per GPU, torch.distributed).

Independent replicas (ensembles, Richardson triples, calibrate_dt candidates) need no communication while
they run: each rank advances its own shard in its own engine, and the per-replica results are gathered
once at the end. A single system is not split across GPUs (no spatial decomposition), so the step loop
has no collective.
"""
from __future__ import annotations

import heapq

import numpy as np


def shard_replicas(sizes, world):
    """Assign replicas to `world` ranks, largest first to the least-loaded rank (ties to the lower rank).
    Returns one sorted index list per rank; deterministic, every replica exactly once."""
    order = sorted(range(len(sizes)), key=lambda r: (-int(sizes[r]), r))
    heap = [(0, k) for k in range(world)]
    shards = [[] for _ in range(world)]
    for r in order:
        load, k = heapq.heappop(heap)
        shards[k].append(r)
        heapq.heappush(heap, (load + int(sizes[r]), k))
    return [sorted(s) for s in shards]


def gather_results(local, world, group=None):
    """Merge {replica index: result} dictionaries from every rank onto every rank, in replica order."""
    import torch.distributed as dist
    if world == 1:
        return dict(sorted(local.items()))
    out = [None] * world
    dist.all_gather_object(out, local, group=group)
    merged = {}
    for part in out:
        for k, v in part.items():
            if k in merged:
                raise ValueError(f"replica {k} reported by two ranks")
            merged[k] = v
    return dict(sorted(merged.items()))


def run_sharded(systems, forces, dts, steps, record_every=0, rank=0, world=1, tpa=None):
    """Advance this rank's shard of the replicas on its GPU and gather (positions, velocities, drift) of all
    replicas on every rank."""
    from .ensemble import ReplicaEnsemble
    shard = shard_replicas([s.n for s in systems], world)[rank]
    local = {}
    if shard:
        ens = ReplicaEnsemble([systems[r] for r in shard], forces, [dts[r] for r in shard], tpa=tpa)
        ens.run(steps, record_every)
        for k, (p, v) in enumerate(ens.state()):
            local[shard[k]] = (np.asarray(p), np.asarray(v), ens.drift(k))
    return gather_results(local, world)
