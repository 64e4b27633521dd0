"""Multi-GPU bookkeeping: one process per GPU, no data-path collective.

A single Wigner instance does not shard usefully (a pencil decomposition
would move the whole state across NVLink twice per step, more than the HBM
sweep it replaces), so N GPUs run N independent replicas, or split a set of
independent instances (``shard``).  The only collectives are on timing and
bookkeeping scalars: the maximum of the ranks' device times and sums of
per-rank counts.  They work with any torch.distributed backend (NCCL on the
GPUs, gloo on the host for the tests).
"""
import os

import torch


def rank_info():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def _initialized():
    import torch.distributed as dist
    return dist.is_available() and dist.is_initialized()


def _reduce(value, op):
    import torch.distributed as dist
    if not _initialized() or dist.get_world_size() == 1:
        return float(value)
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend() == "nccl" else torch.device("cpu")
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value):
    """Maximum of ``value`` over all ranks (the job's time is its slowest rank's)."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX)


def sum_over_ranks(value):
    """Sum of ``value`` over all ranks."""
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM)


def barrier():
    """All ranks meet (no-op without a process group)."""
    import torch.distributed as dist
    if _initialized() and dist.get_world_size() > 1:
        dist.barrier()


def shard(items, rank, world_size):
    """This rank's share of independent work items: every item exactly once
    over the ranks, sizes differing by at most one."""
    return list(items)[rank::world_size]
