"""Multi-GPU plumbing for the rigid-contact step: one process per GPU.

Worlds never interact (cross-world pairs are filtered out,
newton/_src/geometry/broad_phase_common.py:176-177), so the path shards by
worlds with no data-path collective:

* weak scaling: every rank simulates its own full scene (the benchmark's
  default: 4096 worlds per GPU);
* strong scaling: the ranks split one scene into contiguous world ranges
  balanced by cost (sum of bodies^2 per world: broad-phase pairs and
  contacts grow with the square of the body count).

Collectives are used only for run metrics and timing: max over ranks of the
elapsed time and of the max penetration / joint violation (torch.distributed,
NCCL on GPUs, gloo on CPU).
"""

from __future__ import annotations

import numpy as np


def world_costs(bodies_per_world) -> np.ndarray:
    n = np.asarray(bodies_per_world, dtype=np.float64)
    return n * n + n


def partition_worlds(costs, world_size: int) -> list[tuple[int, int]]:
    """Split worlds [0, W) into `world_size` contiguous ranges of near-equal total cost.

    Greedy on the prefix sum: range r ends where the running cost first reaches
    (r + 1) / world_size of the total; every range is non-empty when W >= world_size.
    """
    c = np.asarray(costs, dtype=np.float64)
    W = c.size
    if world_size <= 0:
        raise ValueError("world_size must be positive")
    if W < world_size:
        raise ValueError(f"cannot split {W} worlds over {world_size} ranks")
    prefix = np.cumsum(c)
    total = prefix[-1]
    bounds = [0]
    for r in range(1, world_size):
        cut = int(np.searchsorted(prefix, total * r / world_size, side="left")) + 1
        cut = max(cut, bounds[-1] + 1)            # non-empty
        cut = min(cut, W - (world_size - r))      # leave one world for each remaining rank
        bounds.append(cut)
    bounds.append(W)
    return [(bounds[r], bounds[r + 1]) for r in range(world_size)]


def shard_range(rank: int, world_size: int, bodies_per_world) -> tuple[int, int]:
    return partition_worlds(world_costs(bodies_per_world), world_size)[rank]


def max_over_ranks(values, dist=None, device=None):
    """Element-wise max of `values` (a float or a sequence of floats) over all ranks
    (identity without an initialised process group)."""
    import torch

    if dist is None:
        import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return values
    scalar = np.isscalar(values)
    t = torch.tensor([values] if scalar else list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out = t.cpu().tolist()
    return out[0] if scalar else out
