"""Replica plumbing for more than one GPU.

One boundary-value solve does not shard without a distributed LU, and
requests (incidence directions, frequencies, meshes) are independent, so N
GPUs run N replicas: each rank takes its share of the units and no data
crosses between ranks.  The only collective steps are a barrier before the
timed region and one reduction after it (the slowest rank's time, the units
of all ranks), taken in the same order on every rank.
"""
import torch


def shard(n_units, rank, world):
    """Indices of the units rank `rank` of `world` processes: round robin, so a
    stream keeps its arrival order on every rank and shares differ by one at most."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    return list(range(rank, n_units, world))


def reduce_timing(elapsed, units, device="cpu"):
    """(max of `elapsed` over ranks, sum of `units` over ranks).  `elapsed` is a
    list of times (each reduced by max: one slowest rank per quantity), `units`
    a list of counts (each summed).  With no process group, the local values."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(x) for x in elapsed], [float(x) for x in units]
    t = torch.tensor([float(x) for x in elapsed], dtype=torch.float64, device=device)
    u = torch.tensor([float(x) for x in units], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()], [float(x) for x in u.tolist()]
