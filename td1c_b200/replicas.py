"""Replica bookkeeping of a multi-GPU run: one independent propagation per rank.

The path does not shard (one atom's RHS reduces over all its pairs on one
GPU), so `bench.py --gpus N` runs N replicas, one per rank, with no
data-path collective.  What the ranks share is the timing: every rank
measures its own elapsed time on its device, the job's time is the maximum
over ranks, and the job's throughput is the simulated time of all replicas
divided by that maximum.  Each replica starts from its own seeded state.
"""
AU2FS = 0.02418884254  # femtoseconds per atomic unit of time, td1c's value (mod_const.F90:21)


def replica_seed(base_seed, rank):
    """Seed of rank `rank`'s synthetic initial state."""
    return int(base_seed) + int(rank)


def max_over_ranks(seconds, dist=None, device=None):
    """The job's elapsed time: the maximum of every rank's `seconds` (all ranks call this at the
    same point).  `device` is where the reduction tensor lives: the rank's GPU for NCCL, None
    (CPU) for gloo.  Without an initialised process group the local value is returned."""
    if dist is None or not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(seconds)
    import torch
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, steps, dt_au, seconds):
    """fs of simulated time per second of the whole job: `world` replicas of `steps` steps of
    `dt_au` each, in the job's elapsed `seconds` (weak scaling: per-GPU work fixed)."""
    return world * steps * dt_au * AU2FS / seconds
