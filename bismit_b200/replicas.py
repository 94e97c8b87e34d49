"""Replica sharding across ranks (one process per GPU).

One area's cycle has no exchange step, so several GPUs run independent
replicas (areas, batch instances or server sessions) with no collective on
the data path. What the ranks share is bookkeeping: each rank's replica
seeds, and the whole job's timing, which is the slowest rank's. These helpers
hold that logic; they take any initialised torch.distributed process group
(NCCL on GPUs, gloo on the host) and work without one for a single rank.
"""
import os


def dist_env():
    """(world_size, rank, local_rank) from the launcher's environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def replica_seed(seed, rank):
    """Growth seed of rank `rank`'s replica: distinct per rank, and rank 0's
    equals a single-process run's."""
    return int(seed) + 1000 * int(rank)


def frame_seed(seed, rank):
    """Input-frame seed of rank `rank`'s replica."""
    return int(seed) + int(rank)


def _reduce(x, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, device="cpu"):
    """The slowest rank's figure (times of a step that every rank runs)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.MAX, device)


def sum_over_ranks(x, device="cpu"):
    """The whole job's total (work every rank does on its own replica)."""
    import torch.distributed as dist
    return _reduce(x, dist.ReduceOp.SUM, device)


def job_throughput(units_per_rank, ms_per_rank, device="cpu"):
    """Units per second of the whole job: every rank's units over the slowest
    rank's time (weak scaling)."""
    total = sum_over_ranks(units_per_rank, device)
    ms = max_over_ranks(ms_per_rank, device)
    return total / (ms / 1e3)
