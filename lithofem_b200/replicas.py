"""Host-side logic of the multi-GPU runs: one process per GPU, independent
work per rank, no data-path collective.

A single mesh is assembled by one GPU (the reference has no intra-problem
multi-GPU, README.md:165-168); several meshes (the batched workload) or
k-parallel groups shard across ranks like the reference's process-per-task
sweeps (driver.py:258-311).  The only collectives are the timing and unit
reductions of the benchmark, over whatever backend the process group has
(NCCL on GPUs, gloo in the CPU tests).
"""

from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> list[int]:
    """Round-robin share of items 0..n_items-1 for one rank."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    return list(range(rank, n_items, world))


def _reduce(value: float, dist, device, op) -> float:
    import torch
    if dist is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """The slowest rank's time (the benchmark reports the max over ranks)."""
    return _reduce(value, dist, device, None if dist is None else dist.ReduceOp.MAX)


def sum_over_ranks(value: float, dist=None, device="cpu") -> float:
    """Units processed by all ranks together."""
    return _reduce(value, dist, device, None if dist is None else dist.ReduceOp.SUM)
