"""Several GPUs as replicas: one process per GPU, each simulating its own phonon configurations.

The reference's only multi-GPU form is independent work per GPU with host-side averaging
(single_simulator.cuh:238-297: per-GPU threads, each running a share of the phonon
configurations, the patterns summed on the host).  Here each rank is one process with its own
context; rank r draws its configurations from seed + r * seed_stride, and the ranks' patterns are
summed with one all-reduce per simulation.  Nothing crosses between GPUs inside the slice loop.
Timing takes the maximum over ranks.
"""
from __future__ import annotations

import numpy as np

SEED_STRIDE = 1000


def rank_seed(seed: int, rank: int) -> int:
    """Phonon seed of `rank`: distinct configurations on every rank."""
    return int(seed) + SEED_STRIDE * int(rank)


def for_rank(params, rank: int):
    """A copy of `params` whose phonon seed is the rank's."""
    q = params.copy()
    q.pn_seed = rank_seed(params.pn_seed, rank)
    return q


def sum_patterns(pattern, dist=None):
    """Sum a rank's pattern over all ranks in place (a torch tensor; NCCL on GPUs, gloo on CPU).
    The sum of n ranks' patterns of equal weight 1/c is the pattern of all n*c configurations
    scaled by n; `mean_weight` undoes the factor."""
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(pattern)
    return pattern


def mean_weight(dist=None) -> float:
    """Weight that turns the summed pattern into the average over every rank's configurations."""
    if dist is not None and dist.is_initialized():
        return 1.0 / dist.get_world_size()
    return 1.0


def max_over_ranks(value: float, device=None, dist=None) -> float:
    """The largest of a per-rank time (ms) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def as_numpy(pattern) -> np.ndarray:
    return pattern.detach().cpu().numpy() if hasattr(pattern, "detach") else np.asarray(pattern)
