"""Multi-GPU plumbing: one process per GPU, estimations sharded across ranks.

Estimations are independent, so ranks share no data: each rank runs its own share of the
work (weak scaling) and the only collectives are barriers and the max of the per-rank
device times (the job's time).  No collective sits on the data path.
"""


def shard(n_items, rank, world):
    """Indices of the estimations rank `rank` runs (round-robin over ranks)."""
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    return list(range(rank, n_items, world))


def estimation_seed(rank, k, stride=100_000):
    """Bootstrap seed of the k-th estimation of a rank: distinct across ranks and steps."""
    return rank * stride + k


def max_over_ranks(value, dist=None, device=None):
    """The maximum of a per-rank float over all ranks (identity without a process group)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
