"""Codeword sharding across GPUs (one process per GPU).

Codewords are independent, so a simulation splits the codeword index range
across ranks with no data-path exchange: rank r draws its data and noise from
Philox counters [start, start + count) of the same seed, so the union of the
ranks' work is exactly what one GPU would simulate.  The only collective is
one sum of the per-SNR counters (codewords, iterations, bit errors, codeword
errors, uncoded errors) at the end, as run_LDPCsim.pl sums its processes'
reports (build/run_LDPCsim.pl:156-210).
"""
from __future__ import annotations

from typing import Tuple


def shard_range(total: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous share (start, count) of `total` codewords for `rank`."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of world %d" % (rank, world))
    start = total * rank // world
    end = total * (rank + 1) // world
    return start, end - start


def reduce_counters(counters, group=None):
    """Sum an integer counter tensor over all ranks (in place) and return it."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(counters, op=dist.ReduceOp.SUM, group=group)
    return counters


def weak_shard(n_per_rank: int, rank: int, world: int) -> Tuple[int, int]:
    """Weak scaling: every rank simulates `n_per_rank` codewords per SNR point,
    and rank r takes counters [r * n_per_rank, (r + 1) * n_per_rank) of the
    global index range of `world * n_per_rank` codewords."""
    return shard_range(n_per_rank * world, rank, world)


def max_over_ranks(value: float, device=None, group=None) -> float:
    """Largest `value` over all ranks (a step's device time: the job ends when
    its slowest rank does)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def finish_run(counters, elapsed_ms: float, group=None):
    """End of a timed run on every rank: per-SNR counters summed over ranks
    (a copy; the rank's own counters are left as they are) and the elapsed
    device time as the maximum over ranks.  Every rank must call it, in the
    same order relative to its other collectives."""
    total = reduce_counters(counters.clone(), group)
    return total, max_over_ranks(elapsed_ms, counters.device, group)
