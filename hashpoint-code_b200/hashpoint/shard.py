"""Replicas across GPUs: one process per GPU, views sharded, no data-path collective.

Views are independent, so with N ranks every rank renders its own views
(weak scaling: a rank's camera set is seeded by its rank) and nothing is
exchanged while rendering.  The only collective is the timing reduction after
the timed region: the job's time is the slowest rank's.
"""
import torch
import torch.distributed as dist


def view_seed(base_seed, rank):
    """Camera seed of a rank's view set (rank 0 keeps the single-GPU workload)."""
    return int(base_seed) + 1000 * int(rank)


def max_over_ranks(value, device=None):
    """The largest `value` over all ranks (the value itself without a process group)."""
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rays_per_s(rays_per_rank, ms_per_step_this_rank, device=None):
    """Whole-job throughput: all ranks' rays over the slowest rank's step time."""
    world = dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1
    ms = max_over_ranks(ms_per_step_this_rank, device)
    return rays_per_rank * world / (ms * 1e-3), ms
