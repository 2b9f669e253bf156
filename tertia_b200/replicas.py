"""Replicas: one independent march per GPU, one process per GPU.

A march does not shard: layer i needs layer i+1, and each transverse
transform couples the whole layer.  N GPUs therefore run N independent
marches (seeds, parameter scans, finite-difference probes) with no collective
in the data path.  The only cross-rank steps are the bookkeeping of a timed
run: a barrier on both sides of the timed region, the maximum of the per-rank
device times, and the whole-job rate (the units of all ranks over that
maximum).  The launcher (torchrun) sets RANK, WORLD_SIZE and LOCAL_RANK;
NCCL carries the bookkeeping between GPUs, gloo on the host.
"""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init(world: int, local: int, backend: str = "nccl", timeout_s: float = 300.0) -> None:
    """Join the process group (nothing to do for a single process)."""
    if world <= 1:
        return
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int, device: str = "cuda") -> float:
    """The maximum of x over the ranks (device: where the reduction tensor
    lives, "cuda" with NCCL, "cpu" with gloo)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, ms_max: float) -> float:
    """Units per second of the whole job: every rank processed units_per_rank
    in at most ms_max milliseconds."""
    return world * units_per_rank / (ms_max / 1e3)


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
