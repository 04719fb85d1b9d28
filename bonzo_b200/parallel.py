"""Multi-GPU layout of a batched sweep: one process per GPU (torchrun), the
sweep's instances partitioned across ranks with no data-path collective.

An uneven parameter sweep is a set of independent runs, so ranks never
exchange state; per-instance dt is local to the instance.  The global sweep of
`per_rank` x world instances is drawn rank by rank: rank r owns the instances
drawn from seed + r (weak scaling -- per-GPU work is fixed as the number of
GPUs grows).  The only collectives are the timing barrier and the max of the
per-rank elapsed times.
"""


def rank_seed(seed, rank):
    """Seed of the instances rank `rank` owns."""
    return int(seed) + int(rank)


def sweep_shard(per_rank, seed, rank):
    """Parameter sets (bonzo_b200.problems.blast_batch_params) of rank `rank`."""
    from .problems import blast_batch_params
    return blast_batch_params(per_rank, rank_seed(seed, rank))


def max_over_ranks(value, dist=None, device=None):
    """Max of a per-rank scalar (elapsed milliseconds) over all ranks."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device=None):
    """Sum of a per-rank count (zones processed) over all ranks."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
