"""Range-sharded MSM over the ranks of a torch.distributed process group.

The reference's multi-GPU MSM (multigpu-msm.cuh:87-114) gives every device a
share of the windows, which replicates every point's scalar on every device
and needs a window-split precompute.  Here the points are split by range:
rank k of N takes points [k n / N, (k + 1) n / N), runs its MSM on its own
GPU (lzk_msm_g1 / lzk_msm_g2), and the one exchange step is an all-gather of
the N partial results (one Jacobian point per rank: 96 B for G1, 192 B for
G2; NCCL over NVLink for device tensors).  Every rank then adds the N
partials on its device as an MSM with unit scalars over their affine forms,
so all ranks hold the same result.  A rank may pass the whole base array or
only its own range (the memory-saving form: key tables stay sharded).
"""
import numpy as np
import torch

from . import msm
from .synth import FR_ONE


def shard_range(n, rank, world):
    """the point range [lo, hi) of `rank` among `world` ranks"""
    return (n * rank) // world, (n * (rank + 1)) // world


def _gpu_msm(group, scalars, bases, window_bits):
    return msm.msm(group, scalars, bases, window_bits=window_bits)


def _gpu_sum(group, parts):
    aff = msm.to_affine(group, parts)
    ones = torch.from_numpy(np.tile(FR_ONE, (parts.shape[0], 1)).view(np.int64))
    return msm.msm(group, ones.to(parts.device), aff)


def sharded_msm(group, scalars, bases, pg=None, window_bits=0, local_msm=None, local_sum=None):
    """sum_i scalars[i] * bases[i] over all n points, computed by range
    across the ranks of `pg`.  scalars: all n scalars (n, 4); bases: all n
    points, or only this rank's range [lo, hi).  Returns the Jacobian result
    (same on every rank).  local_msm(group, scalars, bases, window_bits) and
    local_sum(group, jacobian_points) replace the per-rank device operations
    (defaults: lzk_msm_g1/g2 and the unit-scalar MSM over lzk_g*_to_affine)."""
    import torch.distributed as dist
    world = dist.get_world_size(pg)
    rank = dist.get_rank(pg)
    n = scalars.shape[0]
    lo, hi = shard_range(n, rank, world)
    mine = bases[lo:hi] if bases.shape[0] == n else bases
    if mine.shape[0] != hi - lo:
        raise ValueError(f"rank {rank}: expected {hi - lo} bases (range [{lo}, {hi})), got {mine.shape[0]}")
    part = (local_msm or _gpu_msm)(group, scalars[lo:hi], mine, window_bits).contiguous()
    parts = [torch.empty_like(part) for _ in range(world)]
    dist.all_gather(parts, part, group=pg)
    return (local_sum or _gpu_sum)(group, torch.stack(parts))
