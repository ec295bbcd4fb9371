"""Running the path on several GPUs: independent replicas.

One process per GPU.  A single field does not shard (it fits one GPU and its
transforms need no exchange that one GPU cannot do locally), so several GPUs
run independent replicas or disjoint member lists of an ensemble, with no
collective on the data path.  ``torch.distributed`` is used for the barrier
around a timed region and the max over ranks of its duration only.
"""

from __future__ import annotations

import math
from typing import List, Sequence

import torch
import torch.distributed as dist


def world() -> tuple:
    """(rank, world size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (e.g. the device time of a timed region)."""
    _, n = world()
    if n == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, max_ms: float, n_ranks: int) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest
    rank's time."""
    return n_ranks * units_per_rank / (max_ms / 1e3)


def member_cost(N: int, n_scalars: int = 0) -> float:
    """Relative cost of one ensemble member's step (N^2 log N transforms for
    theta and for each passive scalar)."""
    return N * N * math.log2(N) * (1.0 + 0.9 * n_scalars)


def shard_members(costs: Sequence[float], rank: int, n_ranks: int) -> List[int]:
    """Indices of the members this rank advances: longest-processing-time
    assignment (members by decreasing cost, each to the least loaded rank,
    ties to the lower rank), deterministic so that every rank computes the
    same partition without communicating."""
    if not 0 <= rank < n_ranks:
        raise ValueError(f"rank {rank} outside [0, {n_ranks})")
    load = [0.0] * n_ranks
    owner = [0] * len(costs)
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]
