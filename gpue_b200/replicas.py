"""Independent solves on several GPUs: one process per GPU, whole solves per
rank, no collective on the data path.  Only timing crosses ranks: a job's
device time is the maximum over its ranks, and its rate is the work of all
ranks over that time.  The caller owns the torch.distributed process group
(NCCL between GPUs; gloo works the same way on CPU)."""


def shard(n, world, rank):
    """Indices of the solves rank `rank` of `world` runs: every world-th one,
    so mixed sizes spread evenly over the ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d outside a world of %d" % (rank, world))
    return list(range(rank, n, world))


def max_over_ranks(value, dist=None, device="cpu"):
    """The maximum of a per-rank float over all ranks (itself with no group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device="cpu"):
    """The sum of a per-rank float over all ranks (itself with no group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def job_rate(units_this_rank, seconds_this_rank, dist=None, device="cpu"):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    units = sum_over_ranks(units_this_rank, dist, device)
    secs = max_over_ranks(seconds_this_rank, dist, device)
    return units / secs, units, secs
