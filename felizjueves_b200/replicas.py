"""Replicas over ranks: one process per GPU, each building the same workload.

The Fock build does not shard (every rank builds its own J, K, G from its own
density), so N GPUs run N independent replicas and the only collectives are
the timing plumbing: a barrier on each side of the timed region and the
maximum of the per-rank times.  NCCL carries them on GPUs; gloo carries them
in the CPU tests.
"""

from __future__ import annotations

from datetime import timedelta


def init(world: int, backend: str = "nccl", timeout_s: float = 120.0):
    """The process group for `world` > 1 ranks (env:// rendezvous from
    RANK / WORLD_SIZE / MASTER_ADDR / MASTER_PORT), or None for one rank.  A
    short timeout makes a rank that never arrives end the others' next
    collective with an error instead of a wait."""
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the slowest replica's time);
    `value` itself with one rank.  Every rank must call it, in the same
    order as its other collectives."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def finish(dist) -> None:
    if dist is not None:
        dist.destroy_process_group()
