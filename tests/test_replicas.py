"""Replica dispatch over several ranks (the multi-GPU plan: one process per GPU, each matching its
own pairs), exercised with world_size 2 over gloo on the CPU."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from fasterstereocuda_b200 import replicas


def test_shard_partitions_every_pair_once():
    for n in (0, 1, 5, 64, 65):
        for world in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, world) for r in range(world)]
            items = [i for p in parts for i in p]
            assert items == list(range(n))
            sizes = [len(p) for p in parts]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, n_pairs, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = replicas.shard(n_pairs, rank, world)
        # each rank "matches" its pairs: a per-pair value that depends only on the pair index
        results = {i: (i * 2654435761) % 1000003 for i in mine}
        replicas.barrier(world)
        elapsed = replicas.max_over_ranks(0.25 * (rank + 1), world)
        gathered = replicas.gather_to_rank0(results, world, rank)
        replicas.barrier(world)
        q.put((rank, elapsed, gathered))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_time_and_gather():
    world, n_pairs = 2, 7
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, n_pairs, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        rank, elapsed, gathered = q.get(timeout=120)
        out[rank] = (elapsed, gathered)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the timing agreed on is the slowest rank's, on every rank
    assert out[0][0] == out[1][0] == 0.5
    # rank 0 holds every pair's result exactly once, in rank order
    assert out[1][1] is None
    merged = {}
    for part in out[0][1]:
        assert not set(part) & set(merged)
        merged.update(part)
    assert sorted(merged) == list(range(n_pairs))
    assert merged == {i: (i * 2654435761) % 1000003 for i in range(n_pairs)}


def test_single_rank_needs_no_process_group():
    assert not torch.distributed.is_initialized()
    assert replicas.max_over_ranks(1.5, 1) == 1.5
    assert replicas.gather_to_rank0({"a": 1}, 1, 0) == [{"a": 1}]
    replicas.barrier(1)
