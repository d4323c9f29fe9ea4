"""Replica bookkeeping for runs with one independent grid per GPU.

The solver keeps a whole grid resident on one GPU (the reference's MPI pencil
decomposition, set up in src/initialize_mpi_nonperiodic.f90, is not needed for grids that fit in one GPU's
memory).  N GPUs therefore run N independent replicas: each rank steps its own
seeded grid and nothing is exchanged on the data path.  The only cross-rank
operations are the barrier around a timed region and the maximum of the ranks'
device times, which sets the whole job's throughput.
"""


def replica_seed(base, rank):
    """Seed of the synthetic initial field of `rank` (independent replicas)."""
    return int(base) + int(rank)


def max_over_ranks(value, dist=None, device="cpu"):
    """Maximum of a float over all ranks of the default process group.

    `dist` is ``torch.distributed`` (or None for a single process); `device` is
    where the reduction tensor lives ("cuda" for NCCL, "cpu" for gloo).  Every
    rank must call this the same number of times in the same order."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(cells, steps, ms, world):
    """Whole-job Mcell-steps/s: every rank advanced `cells` cells by `steps`
    steps, and the slowest rank took `ms` milliseconds."""
    if ms <= 0:
        raise ValueError("elapsed time must be positive")
    return world * cells * steps / (ms / 1e3) / 1e6
