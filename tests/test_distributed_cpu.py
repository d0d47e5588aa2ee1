"""Multi-process (world_size 2, gloo, CPU) coverage of the replica path:
instances sharded across ranks, host results gathered on every rank."""

import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from dequantizer_b200.replicas import gather_results, shard, shard_weighted


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n_items, costs, out_q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard_weighted(costs, world, rank)
        # each instance's "result": a deterministic function of its index,
        # computed only by the owning rank
        local = {i: float(np.sin(i) * costs[i]) for i in mine}
        merged = gather_results(local)
        out_q.put((rank, sorted(mine), merged))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_gather():
    world, n = 2, 64
    rng = np.random.default_rng(0)
    costs = [float(c) for c in rng.integers(100, 1001, n)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = sorted(i for _, mine, _ in results for i in mine)
    assert owned == list(range(n))
    for _, _, merged in results:
        assert sorted(merged) == list(range(n))
        assert all(abs(merged[i] - np.sin(i) * costs[i]) < 1e-12 for i in range(n))
    loads = [sum(costs[i] for i in mine) for _, mine, _ in results]
    assert max(loads) / min(loads) < 1.05


def test_shard_blocks_cover_items():
    for n in (0, 1, 7, 64):
        for world in (1, 2, 3, 8):
            got = [i for r in range(world) for i in shard(n, world, r)]
            assert got == list(range(n))
