"""Multi-GPU replicas: pairs are independent, so N GPUs run N copies of the solve, one process
per GPU, with no collective on the data path.  The only cross-rank traffic is timing plumbing:
a barrier around the timed region and the maximum of the ranks' elapsed times."""
import torch
import torch.distributed as dist


def pair_seed(rank, i, stride=1000):
    """Seed of pair i on rank `rank`: every rank solves its own, distinct pairs."""
    return stride * rank + i


def max_over_ranks(x, device=None):
    """Maximum of a float over all ranks (the identity without a process group)."""
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_rank, world, elapsed_max_s):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / elapsed_max_s
