"""Replica dispatch over several GPUs of one node.

Stereo pairs are independent and the scans of one pair are whole-row / whole-column sequential,
so the matching path does not shard below a pair: N processes (one per GPU, launched by
torchrun) each match their own contiguous share of the pair list with their own matchers. Ranks
meet only to agree on timing (a barrier on both sides of a timed region, the maximum of the
per-rank elapsed times) and, optionally, to collect results on rank 0. No collective touches
the matching itself.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> range:
    """The contiguous slice of `n_items` pairs that `rank` of `world` matches (sizes differ by at
    most one; ranks past the end get an empty range)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(max(n_items, 0), world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Maximum of a per-rank value (an elapsed time) over all ranks; `device` is the rank's CUDA
    device under NCCL, None (CPU) under gloo."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_rank0(obj, world: int, rank: int):
    """Every rank's `obj` as a list on rank 0 (None elsewhere); `[obj]` with one rank."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world if rank == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
