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
