"""Replica sharding across ranks: the host logic of the multi-GPU path, run as world_size-2 gloo process
groups on the CPU (each replica exactly once, balanced, results gathered in replica order)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from devinproj_b200.sharding import gather_results, shard_replicas


def test_shard_replicas_covers_each_replica_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = (4 * np.clip(np.rint((np.exp(rng.uniform(np.log(256), np.log(32000), 768)) / 4) ** (1 / 3)), 4, 20)
             ** 3).astype(int)
    for world in (1, 2, 4, 8):
        shards = shard_replicas(sizes, world)
        flat = sorted(r for s in shards for r in s)
        assert flat == list(range(len(sizes)))
        loads = [sizes[s].sum() for s in shards]
        assert max(loads) - min(loads) <= sizes.max()
        assert shards == shard_replicas(sizes, world)   # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        shard = shard_replicas(sizes, world)[rank]
        # stand-in for a GPU run: each replica's "result" is a deterministic function of its index
        local = {r: (np.full(3, float(r)), float(sizes[r])) for r in shard}
        merged = gather_results(local, world)
        q.put((rank, sorted(merged), [merged[r][1] for r in sorted(merged)]))
    finally:
        dist.destroy_process_group()


def test_gather_results_world_size_two_gloo():
    sizes = [256, 32000, 500, 864, 4000, 13500, 2048]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, sizes, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = [q.get(timeout=10) for _ in range(world)]
    for rank, keys, vals in got:
        assert keys == list(range(len(sizes)))
        assert vals == [float(s) for s in sizes]


def test_gather_results_rejects_a_replica_reported_twice(monkeypatch):
    import torch.distributed as dist
    assert gather_results({2: 1, 0: 5}, 1) == {0: 5, 2: 1}

    def fake_all_gather_object(out, obj, group=None):
        out[0] = {1: "a"}
        out[1] = {1: "b"}
    monkeypatch.setattr(dist, "all_gather_object", fake_all_gather_object)
    with pytest.raises(ValueError):
        gather_results({1: "a"}, 2)
