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


def test_bench_launches_one_rank_per_gpu_and_shards_the_pairs():
    """bench.py --gpus 2 without a launcher starts two ranks (torch.distributed.run), splits each
    step's pairs between them and reports the slowest rank's time; --dry-run keeps CUDA out (gloo)."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    env = {k: v for k, v in os.environ.items() if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR",
                                                            "MASTER_PORT")}
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--gpus", "2", "--dry-run", "--batch", "8"],
                       capture_output=True, text=True, env=env, timeout=300, cwd=root)
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    out = json.loads(lines[0])
    assert out["n_gpus"] == 2 and out["pairs_per_step"] == 16
    assert out["shards"] == [[0, 8], [8, 16]]
    assert out["ms_per_step"] >= 40.0  # rank 1's 40 ms, the maximum over ranks
    # a launcher that started fewer ranks than --gpus asks for is refused
    env1 = dict(env, WORLD_SIZE="1", RANK="0", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(root / "bench.py"), "--gpus", "2", "--dry-run"], capture_output=True,
                       text=True, env=env1, timeout=120, cwd=root)
    assert r.returncode == 2 and "ranks were launched" in r.stderr
